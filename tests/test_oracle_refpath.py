"""Pins the C oracle to the reference's own path code: the box grid's mass
and mask, GGFX::doOp, GHelmholtz::opVec_prod, GAdvect::apply, GCG::solve and
GBurgers stepped by GExRKStepper, compiled from the reference sources
(oracle/ref/ref_path.cpp) into the committed fixture
tests/golden/ref_path.npz.  The bar is bit-identity: same inputs, same
operation order, same IEEE results.  When oracle/_ref is built here the
live reference is compared as well."""
import numpy as np
import pytest

import oracle as O

GRIDS = {"2d_dir": (2, [4, 3], 4, [0, 0]), "2d_per": (2, [4, 3], 4, [1, 1]),
         "3d_dir": (3, [2, 3, 2], 3, [0, 0, 0]), "3d_per": (3, [2, 2, 3], 4, [1, 1, 1])}
CGS = {"2d_none_inf": (2, [4, 4], 5), "2d_jac_euc": (2, [4, 4], 5),
       "3d_none_euc": (3, [3, 2, 2], 4), "3d_jac_inf": (3, [3, 2, 2], 4),
       "3d_jac_maxit": (3, [3, 2, 2], 4)}
SCHEME = {(1, 0): 1, (2, 0): 2, (3, 0): 3, (4, 0): 4, (2, 1): 22, (3, 1): 33}


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def same(a, b):
    return np.array_equal(bits(a), bits(b))


@pytest.mark.parametrize("tag", list(GRIDS))
def test_grid_mass_mask_mult_bit_exact(refpath, tag):
    dim, ne, p, per = GRIDS[tag]
    o = O.OracleBox(dim, ne, p, periodic=per)
    k = f"grid_{tag}_"
    assert same(o.mass, refpath[k + "mass"])
    assert same(o.mask, refpath[k + "mask"])
    assert same(1.0 / o.mult(), refpath[k + "imult"])


@pytest.mark.parametrize("tag", list(GRIDS))
@pytest.mark.parametrize("op", range(4))
def test_ggfx_doop_bit_exact(refpath, tag, op):
    dim, ne, p, per = GRIDS[tag]
    o = O.OracleBox(dim, ne, p, periodic=per)
    k = f"grid_{tag}_"
    assert same(o.dss(refpath[k + "u"].copy(), op), refpath[k + f"dss{op}"])


@pytest.mark.parametrize("tag", list(GRIDS))
def test_helmholtz_and_advect_bit_exact(refpath, tag):
    dim, ne, p, per = GRIDS[tag]
    o = O.OracleBox(dim, ne, p, periodic=per)
    k = f"grid_{tag}_"
    u, q, pv = refpath[k + "u"], refpath[k + "q"], refpath[k + "pv"]
    assert same(o.helmholtz(u, p=0.7, q_vec=q), refpath[k + "helm_s"])
    assert same(o.helmholtz(u, p_vec=pv, q_vec=q), refpath[k + "helm_v"])
    c = list(refpath[k + "c"])
    assert same(o.advect(u, c), refpath[k + "adv"])


@pytest.mark.parametrize("tag", list(CGS))
def test_cg_iterates_bit_exact(refpath, tag):
    """Same solution bits, residual history and GCGERR code; the iteration
    count the reference's get_iteration_count() reports is iterations + 1
    (solvers/gcg.hpp:75), stored here as iterations."""
    dim, ne, p = CGS[tag]
    o = O.OracleBox(dim, ne, p, periodic=[0] * dim)
    k = f"cg_{tag}_"
    rc_r, it_r, maxit, norm, pc = (int(v) for v in refpath[k + "info"])
    x = np.zeros(o.N)
    rc, it, res = o.cg_solve(refpath[k + "b"], x, p=1.0, q_vec=np.ones(o.N),
                             xb=np.zeros(o.N), maxit=maxit, normtype=norm, tol=1e-10,
                             dinv=refpath[k + "dinv"] if pc else None)
    assert (rc, it) == (rc_r, it_r)
    assert same(x, refpath[k + "x"]) and same(res, refpath[k + "res"])
    if tag.endswith("maxit"):
        assert rc == 1  # GCGERR_NOCONVERGE (gcg.ipp:339-341)


def _rk_tags(refpath):
    return sorted({k[3:-5] for k in refpath.files if k.startswith("rk_") and k.endswith("_info")})


def test_rk_fixture_has_all_schemes(refpath):
    tags = _rk_tags(refpath)
    assert len(tags) == 22


@pytest.mark.parametrize("i", range(22))
def test_rk_stepping_bit_exact(refpath, i):
    tag = _rk_tags(refpath)[i]
    k = f"rk_{tag}_"
    dim, p, order, ssp, kind, nsteps = (int(v) for v in refpath[k + "info"])
    ne = [int(v) for v in refpath[k + "ne"]]
    dt = float(refpath[k + "dt"][0])
    o = O.OracleBox(dim, ne, p, periodic=[1] * dim)
    u = [a.copy() for a in refpath[k + "u0"]]
    c = [np.full(o.N, 1.0 - 0.5 * d) for d in range(dim)] if kind == 0 else None
    o.rk_advance(kind, 0.01, SCHEME[(order, ssp)], u, c=c, dt=dt, nsteps=nsteps)
    for a, b in zip(u, refpath[k + "u"]):
        assert same(a, b), tag


def test_config1_full_200_steps_bit_exact(refpath):
    """The 2-d periodic advection case at full length: 16^2 elements, p = 4,
    c = (1, 0.5), nu = 0.01, RK4, dt = 1e-4, 200 steps."""
    o = O.OracleBox(2, [16, 16], 4, periodic=[1, 1])
    u = [refpath["cfg1_u0"].copy()]
    o.rk_advance(0, 0.01, 4, u, c=[np.ones(o.N), np.full(o.N, 0.5)], dt=1e-4, nsteps=200)
    assert same(u[0], refpath["cfg1_u200"])


def test_live_reference_matches_oracle_if_built():
    if O.load_refpath(2) is None or O.load_refpath(3) is None:
        pytest.skip("oracle/_ref/libgfref{2,3}.so not built (reference checkout absent)")
    rng = np.random.default_rng(7)
    for dim, ne, p in ((2, [3, 5], 6), (3, [2, 2, 1], 5)):
        for per in ([0] * dim, [1] * dim):
            r = O.RefBox(dim, ne, p, periodic=per)
            o = O.OracleBox(dim, ne, p, periodic=per)
            assert same(r.mass(), o.mass) and same(r.mask(), o.mask)
            u = rng.standard_normal(o.N)
            for op in range(4):
                assert same(r.dss(u.copy(), op), o.dss(u.copy(), op))
            q = 0.5 + rng.random(o.N)
            assert same(r.helmholtz(u, p=1.3, q_vec=q), o.helmholtz(u, p=1.3, q_vec=q))


@pytest.mark.parametrize("tag,dim,ne,p", [("2d", 2, [5, 4], 5), ("3d", 3, [3, 3, 2], 4)])
def test_cg_tight_bit_exact(refpath, tag, dim, ne, p):
    o = O.OracleBox(dim, ne, p, periodic=[0] * dim)
    k = f"cgt_{tag}_"
    x = np.zeros(o.N)
    q = np.ones(o.N)
    rc, it, _ = o.cg_solve(refpath[k + "b"], x, p=1.0, q_vec=q, xb=np.zeros(o.N), maxit=2000,
                           normtype=O.NORM_INF, tol=1e-13, dinv=1.0 / o.helmholtz_diag(1.0, q))
    assert (rc, it) == tuple(int(v) for v in refpath[k + "info"])
    assert same(x, refpath[k + "x"])


def test_config3_small_box_100_steps_bit_exact(refpath):
    """The 3-d Burgers configuration (its initial velocity, nu = 1e-3,
    SSP-RK3 at CFL 0.3, 100 steps) on a 3^3-element p = 5 periodic box."""
    o = O.OracleBox(3, [3] * 3, 5, periodic=[1] * 3, length=[2 * np.pi] * 3)
    u = [a.copy() for a in refpath["cfg3s_u0"]]
    o.rk_advance(1, 1e-3, 33, u, dt=float(refpath["cfg3s_dt"][0]), nsteps=100)
    for a, b in zip(u, refpath["cfg3s_u100"]):
        assert same(a, b)
