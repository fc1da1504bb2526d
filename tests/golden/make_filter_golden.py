"""Generates tests/golden/ref_filters.npz from the reference's own code.

Runs in the build container only: it calls oracle/_ref/libgfref.so, built
from the reference's GLLBasis sources by `make -C oracle ref`, whose
gfr_boyd_filter / gfr_projection_filter compute the 1-d filter matrices as
GBoydFilter::init and GProjectionFilter::init do (F column-major).
Keys: boyd_p{p}_d{pdelta}_s{strength}, proj_p{p}_d{pdelta}_s{strength}.
Usage: python tests/golden/make_filter_golden.py
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402

P = C.POINTER(C.c_double)
STRENGTHS = (0.0, 0.25, 1.0)


def cases():
    for p in range(2, 12):
        n = p + 1
        for pdelta in (1, 2, 3):
            for st in STRENGTHS:
                if 0 < n - pdelta - 1 < n:
                    yield "boyd", p, pdelta, st
                # the reference's GLLBasis asserts on a p = 1 low basis
                if pdelta <= (n - 1) // 2 and n - pdelta - 1 >= 2:
                    yield "proj", p, pdelta, st


def main():
    ref = oracle.load_ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libgfref.so missing: run `make -C oracle ref` first")
    out = {}
    for kind, p, pdelta, st in cases():
        F = np.zeros((p + 1) ** 2)
        fn = ref.gfr_boyd_filter if kind == "boyd" else ref.gfr_projection_filter
        assert fn(p, pdelta, C.c_double(st), F.ctypes.data_as(P)) == 0
        out[f"{kind}_p{p}_d{pdelta}_s{st}"] = F
    dst = Path(__file__).resolve().parent / "ref_filters.npz"
    np.savez_compressed(dst, **out)
    print(f"wrote {dst} ({len(out)} matrices)")


if __name__ == "__main__":
    main()
