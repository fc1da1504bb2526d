"""Build script for libgfgpu.so (sm_100a) and the test-side oracle.

Compiles every CUDA translation unit under geoflow_b200/csrc with nvcc for
sm_100a, in parallel, and links them into geoflow_b200/libgfgpu.so (in the
source tree, so it travels with the repository).  `build_oracle()` builds
the C oracle (oracle/_build) and, given a reference checkout, the
reference's own code (oracle/_ref); those are test infrastructure only.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgfgpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-O3", "--expt-relaxed-constexpr",
                     "-I" + str(ROOT / "include")]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    deps = [src] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "gfgpu.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build_lib(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    """Compile and link libgfgpu.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    srcs = _sources()
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(o, s)]

    def compile_one(so):
        s, o = so
        cmd = [nvcc] + NVCC_FLAGS + ["-c", str(s), "-o", str(o)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {s.name}:\n{r.stderr[-4000:]}")
        if verbose:
            print(f"compiled {s.name}", file=sys.stderr)
        return o

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            list(ex.map(compile_one, todo))
    if force or todo or not LIB.exists():
        cmd = [nvcc] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return LIB


def build_oracle(reference: str | None = None) -> None:
    """Build the C oracle and, given a reference checkout, oracle/_ref.

    `reference` (or the GEOFLOW_REFERENCE environment variable) is the root of
    a NOAA-GSL/GeoFLOW checkout; without one only the C oracle is built.
    """
    od = ROOT / "oracle"
    r = subprocess.run(["make", "-C", str(od)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr[-4000:])
    ref = reference or os.environ.get("GEOFLOW_REFERENCE")
    if not ref:
        return
    if not os.path.isdir(os.path.join(ref, "src", "cdg")):
        raise RuntimeError(f"no reference sources under {ref}")
    r = subprocess.run(["make", "-C", str(od), "-j", "4", "ref", f"REF={ref}"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle/_ref build failed:\n" + r.stderr[-4000:])


if __name__ == "__main__":
    build_lib(force="--force" in sys.argv, verbose=True)
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    build_oracle(args[0] if args else None)
    print(LIB)
