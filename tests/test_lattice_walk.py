"""Box-lattice index arithmetic on the host (tests/cpp/test_lattice_walk.cu):
the multiply-shift division and the lattice-point copy enumeration that the
lattice-order kernels (smoother passes, assembly, box gather-scatter) use,
checked against integer division and against the element-to-lattice map,
for 2-d and 3-d boxes, p = 1..8, every periodic combination (single-element
periodic directions included) and rows longer than a block.  Runs on the CPU;
the GPU tests check the same kernels against the oracle and the CSR path."""
import shutil
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_lattice_walk_host(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "test_lattice_walk"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets",
                    str(ROOT / "tests" / "cpp" / "test_lattice_walk.cu"),
                    "-o", str(exe)], check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "lattice walk ok" in r.stdout
