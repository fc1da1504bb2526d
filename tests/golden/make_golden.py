"""Generates tests/golden/ref_gll_gmtk.npz from the reference's own code.

Runs in the build container only (it needs oracle/_ref/libgfref.so, which is
compiled from the reference's GLLBasis and GMTK sources by `make -C oracle
ref`).  The fixture holds:
  gll_p{p}_{xi,w,D}   GLLBasis<long double,double>(p) nodes, weights, D
                      (column-major), p = 2..16
  gmtk_{which}_{u,A,B,C,y,N,Ne}
                      GMTK tensor products on seeded inputs, which =
                      0 I2_X_D1, 1 D2_X_I1, 2 I3_X_I2_X_D1, 3 I3_X_D2_X_I1,
                      4 D3_X_I2_X_I1, 5 D2_X_D1, 6 D3_X_D2_X_D1
Usage: python tests/golden/make_golden.py
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402

P = C.POINTER(C.c_double)


def main():
    ref = oracle.load_ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libgfref.so missing: run `make -C oracle ref` first")
    out = {}
    for p in range(2, 17):
        n = p + 1
        xi, w, D = np.zeros(n), np.zeros(n), np.zeros(n * n)
        ref.gfr_gll(p, xi.ctypes.data_as(P), w.ctypes.data_as(P), D.ctypes.data_as(P))
        out[f"gll_p{p}_xi"], out[f"gll_p{p}_w"], out[f"gll_p{p}_D"] = xi, w, D
    rng = np.random.default_rng(20261203)
    N = np.array([4, 5, 6], dtype=np.uint64)
    Ne = 3
    for which in range(7):
        three = which in (2, 3, 4, 6)
        nn = int(N[0] * N[1] * (N[2] if three else 1))
        ne = 1 if which in (5, 6) else Ne
        u = rng.standard_normal(nn * ne)
        A = rng.standard_normal(int(N[0] * N[0]) if which not in (1, 3, 4) else
                                int(N[1] * N[1]) if which in (1, 3) else int(N[2] * N[2]))
        B = rng.standard_normal(int(N[1] * N[1]))
        Cm = rng.standard_normal(int(N[2] * N[2]))
        y = np.zeros(nn * ne)
        Nc = (C.c_size_t * 3)(*[int(v) for v in N])
        rc = ref.gfr_gmtk(which, A.ctypes.data_as(P), B.ctypes.data_as(P), Cm.ctypes.data_as(P),
                          Nc, C.c_size_t(ne), u.ctypes.data_as(P), y.ctypes.data_as(P))
        assert rc == 0
        for k, v in (("u", u), ("A", A), ("B", B), ("C", Cm), ("y", y)):
            out[f"gmtk_{which}_{k}"] = v
        out[f"gmtk_{which}_N"] = N.astype(np.int64)
        out[f"gmtk_{which}_Ne"] = np.array([ne])
    dst = Path(__file__).resolve().parent / "ref_gll_gmtk.npz"
    np.savez_compressed(dst, **out)
    print(dst, len(out))


if __name__ == "__main__":
    main()
