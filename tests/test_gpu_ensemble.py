"""Ensembles (gf_ensemble_*): many independent problems advanced by one
persistent launch per RK stage or CG iteration.  The CG runs FP32
iterations restarted from the FP64 residual (mixed; inner_tol 1e-4 by
default) or FP64 iterations.

Acceptance:
  * RK members (icosahedral spheres of mixed level and order): every
    member's state after the ensemble steps is bit-identical to gf_rk_advance
    on that member alone (FP64 and FP32, RK1..RK4, advection and heat), for
    every launch shape, tuned or set by hand.  gf_rk_advance is pinned to the
    reference's compiled GBurgers/GExRKStepper on the icosahedral sphere by
    test_gpu_icos.py, so the chain reaches the reference.
  * CG members (2-d Dirichlet boxes of mixed size and order, FP32
    iterations with FP64 refinement): each member converges; its FP64
    residual mask*DSS_Sum(b - A x), recomputed by the oracle, is at most
    1.05 x tol x norm(b) (the solver's own stop test, EUC norm; FP64
    iterations stop on the recurrence residual, and the true one is held
    to 2 x tol); the
    solution matches the oracle's FP64 Jacobi-PCG solution (solved to 1e-14)
    within 1e-8 relative (the members' condition numbers are below 1e4, so
    a 1e-10 relative residual bounds the error near 1e-6 in theory; observed
    differences are far smaller).  Runs repeat bit for bit.
"""
import numpy as np
import pytest
import torch

import oracle as O
from geoflow_b200 import CGTraits, Ensemble, GBurgers, GridBox, IcosGrid, Problem, GFError
from geoflow_b200 import _abi as A
from geoflow_b200 import workloads as W

pytestmark = pytest.mark.gpu

ICOS = [(0, 3), (1, 4), (1, 5), (0, 6), (2, 3), (0, 9)]
BOXES = [(4, 3), (6, 5), (8, 8), (5, 4), (3, 7), (7, 6)]


@pytest.fixture(scope="module")
def icos_members(ctx):
    out = []
    for k, (level, p) in enumerate(ICOS):
        g = IcosGrid(level, p)
        prob = g.problem(ctx)
        lat0, lon0 = 0.3 * k - 0.6, 0.9 * k
        u0 = W.icos_cosine_bell(g.xyz, lat0, lon0)
        c = W.icos_solid_body_wind(g.xyz, alpha=0.2 * k)
        out.append((g, prob, u0, c))
    return out


def _run_single(prob, u0, c, dt, nsteps, dtype, eqn, nu, scheme):
    u = [torch.from_numpy(u0).to("cuda", dtype)]
    cc = [torch.from_numpy(a).to("cuda", dtype) for a in c] if eqn == A.GF_EQN_ADVECT else None
    GBurgers(prob, eqn, nu, scheme=scheme).step(u, cc, dt=dt, nsteps=nsteps)
    return u[0].cpu().numpy()


def _run_ensemble(E, members, dts, nsteps, dtype, eqn, nu, scheme):
    us = [torch.from_numpy(m[2]).to("cuda", dtype) for m in members]
    cs = [[torch.from_numpy(a).to("cuda", dtype) for a in m[3]] for m in members]
    E.advance(us, cs if eqn == A.GF_EQN_ADVECT else None, dt=dts, nsteps=nsteps, eqn=eqn, nu=nu,
              scheme=scheme)
    return [u.cpu().numpy() for u in us]


def _dts(members):
    return [0.2 / (m[0].p ** 2 * 2 ** m[0].level) for m in members]


@pytest.mark.parametrize("nu", [1e-3, 0.0])  # general kernel; prescribed-velocity fast path
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("scheme,nsteps", [(A.GF_RK4, 3), (A.GF_RK4, 4), (A.GF_RK2, 2),
                                           (A.GF_RK3, 3), (A.GF_RK1, 1)])
def test_rk_members_bit_identical_to_single(ctx, icos_members, dtype, scheme, nsteps, nu):
    E = Ensemble(ctx, [m[1] for m in icos_members])
    assert E.kind == A.GF_ENS_RK
    dts = _dts(icos_members)
    got = _run_ensemble(E, icos_members, dts, nsteps, dtype, A.GF_EQN_ADVECT, nu, scheme)
    for k, m in enumerate(icos_members):
        ref = _run_single(m[1], m[2], m[3], dts[k], nsteps, dtype, A.GF_EQN_ADVECT, nu, scheme)
        assert np.array_equal(got[k], ref), (k, ICOS[k])
        assert not np.array_equal(ref, m[2].astype(ref.dtype))  # the state moved


def test_rk_heat_members_bit_identical(ctx, icos_members):
    E = Ensemble(ctx, [m[1] for m in icos_members])
    dts = [1e-4] * len(icos_members)
    got = _run_ensemble(E, icos_members, dts, 3, torch.float64, A.GF_EQN_HEAT, 0.05, A.GF_RK4)
    for k, m in enumerate(icos_members):
        ref = _run_single(m[1], m[2], m[3], dts[k], 3, torch.float64, A.GF_EQN_HEAT, 0.05, A.GF_RK4)
        assert np.array_equal(got[k], ref), k


@pytest.mark.parametrize("threads,bps,team", [(64, 0, 8), (128, 2, 16), (512, 1, 32),
                                              (256, 0, None)])
def test_rk_launch_shape_does_not_change_bits(ctx, icos_members, threads, bps, team):
    members = icos_members
    dts = _dts(members)
    ref = [_run_single(m[1], m[2], m[3], dts[k], 2, torch.float32, A.GF_EQN_ADVECT, 0.0,
                       A.GF_RK4) for k, m in enumerate(members)]
    E = Ensemble(ctx, [m[1] for m in members])
    tb = None if team is None else {n: team for n in range(3, 11)}
    try:
        E.set_shape(threads, bps, tb, dtype=torch.float32)
    except GFError:
        pytest.skip("shape does not fit this device")
    got = _run_ensemble(E, members, dts, 2, torch.float32, A.GF_EQN_ADVECT, 0.0, A.GF_RK4)
    for k in range(len(members)):
        assert np.array_equal(got[k], ref[k]), k


def test_rk_tuned_shape_is_recorded_and_exact(ctx, icos_members):
    members = icos_members
    dts = _dts(members)
    E = Ensemble(ctx, [m[1] for m in members])
    _run_ensemble(E, members, dts, 1, torch.float32, A.GF_EQN_ADVECT, 0.0, A.GF_RK4)
    E.tune(torch.float32, reps=2)
    sh = E.shape(torch.float32)
    assert sh["tuned"] and sh["blocks"] > 0 and sh["threads"] in (64, 128, 256, 512)
    assert set(sh["team_by_n"]) == {m[0].n for m in members}
    got = _run_ensemble(E, members, dts, 2, torch.float32, A.GF_EQN_ADVECT, 0.0, A.GF_RK4)
    for k, m in enumerate(members):
        ref = _run_single(m[1], m[2], m[3], dts[k], 2, torch.float32, A.GF_EQN_ADVECT, 0.0,
                          A.GF_RK4)
        assert np.array_equal(got[k], ref), k
    assert E.launches() > 0


def test_rk_nonfinite_member_reported(ctx, icos_members):
    members = icos_members[:3]
    E = Ensemble(ctx, [m[1] for m in members])
    us = [torch.from_numpy(m[2]).to("cuda") for m in members]
    us[1][5] = float("nan")
    cs = [[torch.from_numpy(a).to("cuda") for a in m[3]] for m in members]
    with pytest.raises(GFError) as ei:
        E.advance(us, cs, dt=1e-3, nsteps=1)
    assert ei.value.code == A.GF_ERR_NONFINITE


# ---- CG ----
@pytest.fixture(scope="module")
def box_members(ctx):
    out = []
    for k, (ne, p) in enumerate(BOXES):
        g = GridBox(2, [ne, ne], p)
        prob = Problem(ctx, g)
        box = O.OracleBox(2, [ne, ne], p)
        f = W.helmholtz2d_rhs(box.xyz, seed=100 + k)
        b = box.mass * f
        out.append((g, prob, box, b))
    return out


def _traits(**kw):
    t = CGTraits()
    t.maxit, t.normtype, t.tol = 20000, A.GF_NORM_EUC, 1e-10
    t.precond, t.precision, t.relative = A.GF_PRECOND_JACOBI, A.GF_CG_MIXED, 1
    for k, v in kw.items():
        setattr(t, k, v)
    return t


def _solve(E, members, traits):
    bs = [torch.from_numpy(m[3]).to("cuda") for m in members]
    xs = [torch.zeros_like(b) for b in bs]
    rc, it, nrm, st = E.solve(bs, xs, traits, p=1.0, q=1.0)
    return rc, it, nrm, st, [x.cpu().numpy() for x in xs]


def _euc(box, v):
    return float(np.sqrt(np.sum(v * v) / box.N))


CG_MODES = {"mixed": {}, "mixed_inner_1e-3": {"inner_tol": 1e-3},
            "fp64": {"precision": A.GF_CG_FP64}}


@pytest.mark.parametrize("mode", list(CG_MODES))
def test_cg_members_converge_to_oracle(ctx, box_members, mode):
    E = Ensemble(ctx, [m[1] for m in box_members])
    assert E.kind == A.GF_ENS_CG
    rc, it, nrm, st, xs = _solve(E, box_members, _traits(**CG_MODES[mode]))
    assert rc == 0 and list(st) == [0] * len(box_members)
    for k, (g, prob, box, b) in enumerate(box_members):
        x = xs[k]
        r = b - box.helmholtz(x, p=1.0, q_vec=np.ones(box.N))
        box.dss(r, O.SUM)
        r *= box.mask
        if mode == "fp64":  # GCG's test on the recurrence residual; the true one near it
            assert nrm[k] <= 1e-10 * _euc(box, b), k
            assert _euc(box, r) <= 2e-10 * _euc(box, b), k
        else:  # the stop test is on the FP64 residual, which the oracle recomputes
            assert _euc(box, r) <= 1.05e-10 * _euc(box, b), k
            assert abs(nrm[k] - _euc(box, r)) <= 1e-3 * _euc(box, r) + 1e-14, k
        dinv = 1.0 / box.helmholtz_diag(1.0, np.ones(box.N))
        xr = np.zeros(box.N)
        rc0, _, _ = box.cg_solve(b, xr, p=1.0, q_vec=np.ones(box.N), xb=np.zeros(box.N),
                                 maxit=20000, normtype=O.NORM_EUC, tol=1e-14, dinv=dinv)
        assert np.max(np.abs(x - xr)) <= 1e-8 * np.max(np.abs(xr)), k
        assert it[k] > 0


def test_cg_repeats_bit_for_bit_and_after_tuning(ctx, box_members):
    E = Ensemble(ctx, [m[1] for m in box_members])
    r1 = _solve(E, box_members, _traits())
    r2 = _solve(E, box_members, _traits())
    for a, b in zip(r1[4], r2[4]):
        assert np.array_equal(a, b)
    assert list(r1[1]) == list(r2[1])
    E.tune(reps=2)
    assert E.shape()["tuned"]
    rc, it, nrm, st, xs = _solve(E, box_members, _traits())
    assert rc == 0 and list(st) == [0] * len(box_members)
    # partial sums are formed per 256-node lattice slice and folded in slice
    # order, so the launch shape changes no bit
    for k in range(len(box_members)):
        assert np.array_equal(xs[k], r1[4][k]), k
    assert list(it) == list(r1[1])
    E.set_shape(64, 1)
    r3 = _solve(E, box_members, _traits())
    for k in range(len(box_members)):
        assert np.array_equal(r3[4][k], r1[4][k]), k


def test_cg_maxit_reports_noconvergence(ctx, box_members):
    E = Ensemble(ctx, [m[1] for m in box_members[:3]])
    rc, it, nrm, st, xs = _solve(E, box_members[:3], _traits(maxit=3))
    assert rc == A.GF_CG_NOCONVERGE
    assert all(s == 1 for s in st)
    assert all(i <= 3 for i in it)


def test_cg_inf_norm_and_inner_tolerance(ctx, box_members):
    members = box_members[:4]
    E = Ensemble(ctx, [m[1] for m in members])
    rc, it, nrm, st, xs = _solve(E, members, _traits(normtype=A.GF_NORM_INF, inner_tol=1e-3))
    assert rc == 0
    for k, (g, prob, box, b) in enumerate(members):
        r = b - box.helmholtz(xs[k], p=1.0, q_vec=np.ones(box.N))
        box.dss(r, O.SUM)
        r *= box.mask
        assert np.max(np.abs(r)) <= 1.05e-10 * np.max(np.abs(b)), k


def test_members_of_both_kinds_are_rejected(ctx, icos_members, box_members):
    with pytest.raises(GFError):
        Ensemble(ctx, [icos_members[0][1], box_members[0][1]])
    g3 = GridBox(3, [2, 2, 2], 3)
    with pytest.raises(GFError):
        Ensemble(ctx, [Problem(ctx, g3)])
    E = Ensemble(ctx, [m[1] for m in box_members[:2]])
    with pytest.raises(GFError):
        _solve(E, box_members[:2], _traits(precond=A.GF_PRECOND_NONE))


def test_icos_classes_on_device_match_host(ctx):
    for level, p in [(1, 4), (2, 7)]:
        h = IcosGrid(level, p)
        d = IcosGrid(level, p, ctx=ctx)
        assert h.nclass == d.nclass
        for a in ("node_class", "class_ptr", "members"):
            assert np.array_equal(getattr(h, a), getattr(d, a)), a


def test_cg_members_match_single_problem_masked_solve(ctx, box_members):
    """The ensemble solves solve_impl(A, b, xb = 0, x): each member equals
    gf_cg_solve with a zero xb (1e-8) and keeps a zero Dirichlet boundary
    even from a nonzero initial guess."""
    from geoflow_b200 import GCG, GHelmholtz
    members = box_members[:4]
    E = Ensemble(ctx, [m[1] for m in members])
    bs = [torch.from_numpy(m[3]).to("cuda") for m in members]
    xs = [torch.full_like(b, 0.5) for b in bs]  # nonzero boundary in the initial guess
    rc, it, nrm, st = E.solve(bs, xs, _traits())
    assert rc == 0
    for k, (g, prob, box, b) in enumerate(members):
        x = xs[k].cpu().numpy()
        assert np.all(x[box.mask == 0] == 0.0)
        H = GHelmholtz(prob)
        H.set_Lap_scalar(1.0)
        H.set_mass_scalar(1.0)
        tr = _traits(precision=A.GF_CG_FP64, check_every=16)
        xr = torch.zeros_like(bs[k])
        GCG(tr, prob).solve(H, bs[k], torch.zeros_like(bs[k]), xr)
        xr = xr.cpu().numpy()
        assert np.max(np.abs(x - xr)) <= 1e-8 * np.max(np.abs(xr)), k


def test_single_problem_solve_without_xb_is_unmasked(ctx, box_members):
    """GCG::solve_impl(A, b, x) masks only when bbv_ is set, which the xb
    form does: without xb the solve is the unmasked (natural boundary)
    system, as the oracle's restatement with no mask."""
    from geoflow_b200 import GCG, GHelmholtz
    g, prob, box, b = box_members[1]
    H = GHelmholtz(prob)
    H.set_Lap_scalar(1.0)
    H.set_mass_scalar(1.0)
    x = torch.zeros(box.N, dtype=torch.float64, device="cuda")
    GCG(_traits(precision=A.GF_CG_FP64, normtype=A.GF_NORM_INF, relative=0, tol=1e-13),
        prob).solve(H, torch.from_numpy(b).to("cuda"), x)
    xo = np.zeros(box.N)
    dinv = 1.0 / box.helmholtz_diag(1.0, np.ones(box.N))
    rc, _, _ = box.cg_solve(b, xo, p=1.0, q_vec=np.ones(box.N), maxit=20000,
                            normtype=O.NORM_INF, tol=1e-13, dinv=dinv, use_mask=False)
    assert rc == 0
    x = x.cpu().numpy()
    assert np.max(np.abs(x[box.mask == 0])) > 0.1 * np.max(np.abs(x))  # boundary moved
    assert np.max(np.abs(x - xo)) <= 1e-10 * np.max(np.abs(xo))
