"""Spectral filters (sem/gboyd_filter.ipp, sem/gprojection_filter.ipp).

CPU: the 1-d filter matrices of gf_filter_matrix against the reference's
own GLLBasis-based construction (tests/golden/ref_filters.npz, made by
tests/golden/make_filter_golden.py from oracle/_ref; and live when
oracle/_ref is built), 1e-12 relative; projection properties (idempotent at
strength 1, keeps polynomials of the low order); argument checks.
GPU: the in-place filter (gf_filter_apply, a matrix per direction) against
the oracle's GMTK products, 1e-13; filtered RK stepping equals stepping then
filtering, bit for bit.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from geoflow_b200 import _abi as A
from geoflow_b200.sem import filter_matrix

GOLDEN = Path(__file__).parent / "golden" / "ref_filters.npz"
KIND = {"boyd": A.GF_FILTER_BOYD, "proj": A.GF_FILTER_PROJECTION}


def parse(key):
    kind, p, d, s = key.split("_")
    return KIND[kind], int(p[1:]), int(d[1:]), float(s[1:])


def test_filter_matrices_match_reference_fixture():
    gold = np.load(GOLDEN)
    assert len(gold.files) >= 100
    for key in gold.files:
        kind, p, pdelta, st = parse(key)
        F = filter_matrix(kind, p, pdelta, st).ravel(order="F")
        ref = gold[key]
        assert np.max(np.abs(F - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref))), key


def test_filter_matrices_match_live_reference():
    ref = O.load_ref()
    if ref is None:
        pytest.skip("oracle/_ref not built here")
    P = C.POINTER(C.c_double)
    for p in (3, 7, 11):
        for pdelta in (1, 2):
            for st in (0.4, 1.0):
                F = np.zeros((p + 1) ** 2)
                assert ref.gfr_boyd_filter(p, pdelta, C.c_double(st), F.ctypes.data_as(P)) == 0
                ours = filter_matrix(A.GF_FILTER_BOYD, p, pdelta, st).ravel(order="F")
                assert np.max(np.abs(ours - F)) <= 1e-12 * max(1.0, np.max(np.abs(F)))
                if pdelta > p // 2 or p - pdelta < 2:  # invalid, or a p = 1 low basis
                    continue
                assert ref.gfr_projection_filter(p, pdelta, C.c_double(st),
                                                 F.ctypes.data_as(P)) == 0
                ours = filter_matrix(A.GF_FILTER_PROJECTION, p, pdelta, st).ravel(order="F")
                assert np.max(np.abs(ours - F)) <= 1e-12 * max(1.0, np.max(np.abs(F)))


@pytest.mark.parametrize("p,pdelta", [(4, 1), (7, 2), (8, 3), (2, 1)])
def test_projection_filter_properties(p, pdelta):
    F = filter_matrix(A.GF_FILTER_PROJECTION, p, pdelta, 1.0)
    assert np.allclose(F @ F, F, atol=1e-12)
    xi, _, _ = O.gll(p)
    v = xi ** (p - pdelta) - 0.3 * xi + 1.0  # degree p - pdelta
    assert np.allclose(F @ v, v, atol=1e-12)
    half = filter_matrix(A.GF_FILTER_PROJECTION, p, pdelta, 0.5)
    assert np.allclose(half, 0.5 * F + 0.5 * np.eye(p + 1), atol=1e-13)


def test_filter_matrix_rejects_bad_arguments():
    lib = A.load()
    F = np.zeros(64)
    assert lib.gf_filter_matrix(A.GF_FILTER_BOYD, 7, 7, 0.5, A.ptr(F)) == A.GF_ERR_ARG  # ifilter 0
    assert lib.gf_filter_matrix(A.GF_FILTER_BOYD, 7, 2, 1.5, A.ptr(F)) == A.GF_ERR_ARG
    assert lib.gf_filter_matrix(A.GF_FILTER_PROJECTION, 7, 4, 0.5, A.ptr(F)) == A.GF_ERR_ARG
    assert lib.gf_filter_matrix(7, 7, 2, 0.5, A.ptr(F)) == A.GF_ERR_ARG


# ------------------------------------------------------------------ GPU ----

def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("dim,ne,p", [(3, [2, 3, 2], 5), (3, [2, 2, 2], 7), (2, [3, 4], 6)])
def test_filter_apply_matches_oracle_gmtk(ctx, dim, ne, p):
    from geoflow_b200 import GBoydFilter, GProjectionFilter, GridBox, Problem
    g = GridBox(dim, ne, p)
    prob = Problem(ctx, g)
    rng = np.random.default_rng(p)
    u = [rng.standard_normal(g.ndof()) for _ in range(2)]
    lib, Ne, n = O.load(), g.nelems, p + 1
    col = lambda m: np.ascontiguousarray(m.ravel(order="F"))
    for flt in (GBoydFilter(prob, [1, 2, 1][:dim], [0.3, 0.6, 0.9][:dim]),
                GProjectionFilter(prob, 1, 0.5, istate=[1])):
        ut = [dev(a) for a in u]
        flt.apply(ut)
        for j in range(2):
            if flt.istate and j not in flt.istate:
                assert np.array_equal(ut[j].cpu().numpy(), u[j])
                continue
            F = flt.F
            y1, y2 = np.zeros(g.ndof()), np.zeros(g.ndof())
            if dim == 3:
                y3 = np.zeros(g.ndof())
                lib.gfo_I3_X_I2_X_D1(O.dp(col(F[0])), O.dp(u[j]), n, n, n, Ne, O.dp(y1))
                lib.gfo_I3_X_D2_X_I1(O.dp(col(F[1].T)), O.dp(y1), n, n, n, Ne, O.dp(y2))
                lib.gfo_D3_X_I2_X_I1(O.dp(col(F[2].T)), O.dp(y2), n, n, n, Ne, O.dp(y3))
                ref = y3
            else:
                lib.gfo_I2_X_D1(O.dp(col(F[0])), O.dp(u[j]), n, n, Ne, O.dp(y1))
                lib.gfo_D2_X_I1(O.dp(col(F[1].T)), O.dp(y1), n, n, Ne, O.dp(y2))
                ref = y2
            got = ut[j].cpu().numpy()
            assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.gpu
def test_filtered_stepping_equals_step_then_filter(ctx):
    """GBurgers.step(filters=[f]) = for each step: advance one step, then
    f.apply in place (GMConv::step_impl's order), bit for bit."""
    import torch
    from geoflow_b200 import GBoydFilter, GBurgers, GridBox, Problem
    g = GridBox(3, [3, 2, 2], 5, periodic=[1, 1, 1])
    prob = Problem(ctx, g, dirichlet_mask=False)
    rng = np.random.default_rng(9)
    u0 = [0.2 * rng.standard_normal(g.ndof()) for _ in range(3)]
    f = GBoydFilter(prob, 2, 0.5)
    B = GBurgers(prob, A.GF_EQN_BURGERS, 0.02, scheme=A.GF_RK3)
    ua = [dev(a) for a in u0]
    B.step(ua, None, dt=1e-3, nsteps=3, filters=[f])
    ub = [dev(a) for a in u0]
    for _ in range(3):
        B.step(ub, None, dt=1e-3, nsteps=1)
        f.apply(ub)
    for a, b in zip(ua, ub):
        assert torch.equal(a, b)
    # out of place leaves the input untouched
    uc = [dev(a) for a in u0]
    uo = [torch.empty_like(a) for a in uc]
    f.apply(uc, None, uo)
    assert torch.equal(uc[0], dev(u0[0])) and not torch.equal(uo[0], uc[0])
