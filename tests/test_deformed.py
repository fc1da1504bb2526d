"""Deformed (GE_DEFORMED) and 2-d embedded (GE_2DEMBEDDED) elements: the
full-metric operators through the C ABI against the oracle on the same
caller-supplied geometry (per-node dXi/dX and Jac).

Tolerances: FP64 applies 1e-12 relative (max-norm), derivatives 1e-13,
advection / dudt 1e-11, FP32 apply 1e-5 (2-norm), constrain2sphere
bit-exact, one embedded RK1 Burgers step 1e-12.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle as O
from geoflow_b200 import GBurgers, GCG, CGTraits, GGFX, GHelmholtz, GridBox, Problem, _abi as A

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def host(t):
    return t.detach().cpu().numpy()


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def sphere_xyz(g, radius=1.3):
    """Node coordinates on a sphere from the 2-d box coordinates (as a
    lon/lat patch); only used by constrain2sphere."""
    lon = 0.4 + 1.2 * g.xyz[0]
    lat = -0.6 + 1.0 * g.xyz[1]
    return [radius * np.cos(lat) * np.cos(lon), radius * np.cos(lat) * np.sin(lon),
            radius * np.sin(lat)]


def make(ctx, dim, ne, p, kind, periodic=None, mask=True, structured=True, seed=0):
    """A box's elements and classes with a perturbed full metric."""
    g = GridBox(dim, ne, p, periodic=periodic)
    box = O.OracleBox(dim, ne, p, periodic=periodic)
    nxy = 3 if kind == "embedded" else dim
    rng = np.random.default_rng(seed)
    N = g.ndof()
    X = []
    for i in range(dim):
        row = []
        for k in range(nxy):
            base = box.dXidX[i] if i == k else np.zeros(N)
            row.append(base + 0.15 * np.max(box.dXidX[0]) * (rng.random(N) - 0.5))
        X.append(row)
    Jac = box.Jac * (0.7 + 0.6 * rng.random(N))
    od = O.OracleDef(box, X, Jac, nxy)
    xyz = sphere_xyz(g) if kind == "embedded" else None
    prob = Problem(ctx, g, dirichlet_mask=mask, structured=structured, geometry=kind,
                   node_geom=od.node_geom(), node_xyz=np.concatenate(xyz) if xyz else None)
    return g, prob, od, xyz


CASES = [(3, [2, 2, 2], 4, "deformed"), (3, [2, 1, 2], 7, "deformed"), (2, [3, 2], 5, "deformed"),
         (2, [3, 3], 4, "embedded"), (2, [2, 2], 8, "embedded")]


@pytest.mark.parametrize("dim,ne,p,kind", CASES)
def test_def_helmholtz_matches_oracle(ctx, dim, ne, p, kind):
    g, prob, od, _ = make(ctx, dim, ne, p, kind)
    rng = np.random.default_rng(3 + p)
    u = rng.standard_normal(g.ndof())
    qv = 0.5 + rng.random(g.ndof())
    pv = 0.5 + rng.random(g.ndof())
    for pscal, use_q, use_pv in ((1.0, False, False), (0.37, True, False), (1.0, True, True)):
        H = GHelmholtz(prob)
        H.set_Lap_scalar(dev(pv) if use_pv else pscal)
        if use_q:
            H.set_mass_scalar(dev(qv))
        uo = prob.zeros()
        H.opVec_prod(dev(u), None, uo)
        ref = od.helmholtz(u, p=pscal, p_vec=pv if use_pv else None, q_vec=qv if use_q else None)
        assert relerr(host(uo), ref) < 1e-12


@pytest.mark.parametrize("dim,ne,p,kind", [CASES[0], CASES[3]])
def test_def_helmholtz_fp32(ctx, dim, ne, p, kind):
    g, prob, od, _ = make(ctx, dim, ne, p, kind)
    u = np.random.default_rng(4).standard_normal(g.ndof())
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    uo = prob.zeros(torch.float32)
    H.opVec_prod(dev(u, torch.float32), None, uo)
    ref = od.helmholtz(u.astype(np.float32).astype(np.float64), q_vec=np.ones(g.ndof()))
    assert np.linalg.norm(host(uo) - ref) / np.linalg.norm(ref) < 1e-5


@pytest.mark.parametrize("dim,ne,p,kind", CASES)
def test_def_deriv_advect_dudt_match_oracle(ctx, dim, ne, p, kind):
    g, prob, od, _ = make(ctx, dim, ne, p, kind, periodic=[1] * dim, mask=False)
    lib = A.load()
    nxy = od.nxy
    rng = np.random.default_rng(8)
    u = rng.standard_normal(g.ndof())
    du = prob.zeros()
    for idir in range(1, nxy + 1):
        ctx.check(lib.gf_deriv(prob.handle, A.GF_F64, A.ptr(dev(u)), idir, A.ptr(du)))
        assert relerr(host(du), od.deriv(u, idir)) < 1e-13
    c = [rng.standard_normal(g.ndof()) for _ in range(nxy)]
    ct = [dev(a) for a in c]
    po = prob.zeros()
    ctx.check(lib.gf_advect_apply(prob.handle, A.GF_F64, A.ptr(dev(u)), nxy, A.ptr_array(ct),
                                  A.ptr(po)))
    assert relerr(host(po), od.advect(u, c)) < 1e-12
    for kind_eq, nst in ((0, 1), (1, nxy), (2, 1)):
        us = [rng.standard_normal(g.ndof()) for _ in range(nst)]
        B = GBurgers(prob, kind_eq, 0.013)
        B.nstate = nst
        out = prob.zeros(ncomp=nst)
        B.dudt([dev(a) for a in us], ct if kind_eq == 0 else None, out)
        ref = od.dudt(kind_eq, 0.013, us, c if kind_eq == 0 else None)
        for k in range(nst):
            assert relerr(host(out[k]), ref[k]) < 1e-11


@pytest.mark.parametrize("structured", [True, False])
def test_def_cg_converges_and_jacobi_agrees(ctx, structured):
    """Deformed 3-d Helmholtz: CG with and without the (full-metric)
    Jacobi preconditioner reach the same solution, and the oracle's
    assembled residual of that solution is at the tolerance."""
    g, prob, od, _ = make(ctx, 3, [3, 2, 2], 5, "deformed", structured=structured, seed=2)
    box = od.box
    rng = np.random.default_rng(12)
    f = rng.standard_normal(g.ndof())
    f = f[g.members[g.class_ptr[:-1]]][g.node_class]
    b = od.mass * f
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    xs = []
    for pre in (A.GF_PRECOND_NONE, A.GF_PRECOND_JACOBI):
        x = prob.zeros()
        cg = GCG(CGTraits(maxit=5000, tol=1e-12, precond=pre, normtype=A.GF_NORM_EUC, relative=1),
                 prob)
        assert cg.solve(H, dev(b), dev(0 * b), x) == 0
        xs.append(host(x))
    assert relerr(xs[1], xs[0]) < 1e-9
    # assembled, masked residual of the solution (oracle operator)
    r = b - od.helmholtz(xs[1], q_vec=np.ones(g.ndof()))
    box.dss(r, O.SUM)
    bb = b.copy()
    box.dss(bb, O.SUM)
    r *= box.mask
    bb *= box.mask
    assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(bb)


def test_constrain2sphere_bit_exact(ctx):
    g, prob, od, xyz = make(ctx, 2, [3, 2], 5, "embedded")
    lib = A.load()
    rng = np.random.default_rng(6)
    v = [rng.standard_normal(g.ndof()) for _ in range(3)]
    vt = [dev(a) for a in v]
    xt = [dev(a) for a in xyz]
    ctx.check(lib.gf_constrain2sphere(prob.handle, A.GF_F64, A.ptr_array(vt), A.ptr_array(xt)))
    ref = O.constrain2sphere(xyz, [a.copy() for a in v])
    for k in range(3):
        assert np.array_equal(host(vt[k]), ref[k])


def test_constrain2sphere_noop_off_the_sphere(ctx):
    g = GridBox(2, [2, 2], 3)
    prob = Problem(ctx, g)
    v = [dev(np.ones(g.ndof())) for _ in range(3)]
    A.load().gf_constrain2sphere(prob.handle, A.GF_F64, A.ptr_array(v), A.ptr_array(v))
    assert all(bool((t == 1.0).all()) for t in v)


def test_embedded_rk1_burgers_step_matches_composition(ctx):
    """One step_b(1) of 3-component Burgers on an embedded surface, with the
    stepper's constrain2sphere calls, against the same step composed from
    the oracle's pieces (gexrk_stepper.ipp:252-341)."""
    g, prob, od, xyz = make(ctx, 2, [3, 3], 4, "embedded", periodic=[1, 1], mask=False)
    rng = np.random.default_rng(10)
    u0 = [0.3 * rng.standard_normal(g.ndof()) for _ in range(3)]
    for a in u0:
        od.box.dss(a, O.SMOOTH)
    dt, nu = 1e-3, 0.02
    B = GBurgers(prob, A.GF_EQN_BURGERS, nu, scheme=A.GF_RK1)
    assert B.nstate == 3
    ut = [dev(a) for a in u0]
    B.step(ut, None, dt=dt, nsteps=1)
    # composition: u = constrain(S(uin)); K = S(F(u)); uout = S(uin + dt K); constrain(uout)
    u = [a.copy() for a in u0]
    for a in u:
        od.box.dss(a, O.SMOOTH)
    O.constrain2sphere(xyz, u)
    K = od.dudt(1, nu, u)
    for k in K:
        od.box.dss(k, O.SMOOTH)
    uo = [u0[k] + K[k] * dt for k in range(3)]
    for a in uo:
        od.box.dss(a, O.SMOOTH)
    O.constrain2sphere(xyz, uo)
    for k in range(3):
        assert relerr(host(ut[k]), uo[k]) < 1e-12


def test_adjoint_rejects_full_metric(ctx):
    g, prob, od, _ = make(ctx, 3, [2, 2, 2], 3, "deformed", periodic=[1, 1, 1], mask=False)
    lib = A.load()
    u = prob.zeros(ncomp=3)
    assert lib.gf_dudt_vjp(prob.handle, A.GF_F64, A.GF_EQN_BURGERS, 0.1, 3, A.ptr_array(u), None,
                           A.ptr_array(u), A.ptr_array(u)) == A.GF_ERR_ARG
