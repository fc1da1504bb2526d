"""Adjoint path (no reference counterpart): transpose and VJP kernels,
RK-step VJP and the checkpointed gradient, all through the C ABI.

Checks:
  * dot-product (transpose) tests <A v, w> = <v, A^T w> for the Helmholtz
    apply, DSS Sum/Smooth, the dudt VJP and the RK step VJP;
  * the full Jacobian of dudt (tiny 2-d case) against its VJP columns;
  * the gradient of J = 1/2 ||u(T) - u_obs||_M^2 against central finite
    differences (eps = 1e-6) on random directions, agreeing to 1e-6;
  * the gradient does not depend on the checkpoint interval (bit-exact);
  * torch.autograd.gradcheck through a torch.autograd.Function wrapper of
    the step VJP and of the gradient (the wrapper lives only here).
Tolerances are written at each assertion.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from geoflow_b200 import GBurgers, GMass, GridBox, Problem, _abi as A

pytestmark = pytest.mark.gpu

BURGERS, ADVECT, HEAT = A.GF_EQN_BURGERS, A.GF_EQN_ADVECT, A.GF_EQN_HEAT


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=torch.float64)


def vdot(a, b):
    return float(sum(torch.dot(x, y).item() for x, y in zip(a, b)))


def vnorm(a):
    return float(np.sqrt(sum(torch.dot(x, x).item() for x in a)))


def continuous(g, a):
    """The E-vector of a continuous field: every member of a class takes
    the value of the class's first member."""
    return a[g.members[g.class_ptr[:-1]]][g.node_class]


def fourier_field(g, rng, kmax=4, amp=0.1):
    """Seeded random Fourier series with wavenumbers <= kmax on the unit
    periodic box, scaled to max |u| = amp."""
    xs = g.xyz
    u = np.zeros(g.ndof())
    for _ in range(8):
        k = rng.integers(-kmax, kmax + 1, g.dim)
        ph = rng.uniform(0, 2 * np.pi)
        u += rng.standard_normal() * np.cos(2 * np.pi * sum(k[d] * xs[d] for d in range(g.dim)) + ph)
    return amp * continuous(g, u) / max(np.max(np.abs(u)), 1e-300)


def make(ctx, dim, ne, p, geometry="affine"):
    g = GridBox(dim, ne, p, periodic=[1] * dim)
    return g, Problem(ctx, g, dirichlet_mask=False, geometry=geometry)


def dudt(B, prob, u, c):
    out = prob.zeros(ncomp=B.nstate)
    B.dudt(u, c, out)
    return out


# ---------------------------------------------------------------- transposes
@pytest.mark.parametrize("dim,ne,p", [(3, [2, 2, 2], 4), (2, [3, 2], 6)])
def test_helmholtz_transpose_dot_product(ctx, dim, ne, p):
    g, prob = make(ctx, dim, ne, p)
    rng = np.random.default_rng(3)
    v, w = dev(rng.standard_normal(g.ndof())), dev(rng.standard_normal(g.ndof()))
    lib = A.load()
    Av, ATw = prob.zeros(), prob.zeros()
    ctx.check(lib.gf_helmholtz_apply(prob.handle, A.GF_F64, 0.7, None, 0.3, None, 1, A.ptr(v),
                                     A.ptr(Av)))
    ctx.check(lib.gf_helmholtz_apply_T(prob.handle, A.GF_F64, 0.7, 0.3, 1, A.ptr(w), A.ptr(ATw)))
    a, b = vdot([Av], [w]), vdot([v], [ATw])
    # tolerance: 1e-12 of |Av||w|
    assert abs(a - b) <= 1e-12 * vnorm([Av]) * vnorm([w])


@pytest.mark.parametrize("op", [A.GF_DSS_SUM, A.GF_DSS_SMOOTH])
@pytest.mark.parametrize("structured", [True, False])
def test_dss_transpose_dot_product(ctx, op, structured):
    g = GridBox(3, [3, 2, 2], 5, periodic=[1, 0, 1])
    prob = Problem(ctx, g, dirichlet_mask=False, structured=structured)
    rng = np.random.default_rng(4)
    v, w = dev(rng.standard_normal(g.ndof())), dev(rng.standard_normal(g.ndof()))
    lib = A.load()
    Sv, STw = v.clone(), w.clone()
    ctx.check(lib.gf_dss(prob.handle, A.GF_F64, op, A.ptr(Sv)))
    ctx.check(lib.gf_dss_T(prob.handle, A.GF_F64, op, A.ptr(STw)))
    # tolerance: 1e-13 of |Sv||w|
    assert abs(vdot([Sv], [w]) - vdot([v], [STw])) <= 1e-13 * vnorm([Sv]) * vnorm([w])


# ---------------------------------------------------------------- dudt VJP
DUDT_CASES = [(3, [2, 2, 2], 4, BURGERS), (3, [2, 1, 2], 6, ADVECT), (3, [2, 2, 1], 3, HEAT),
              (2, [3, 2], 5, BURGERS), (2, [2, 2], 7, ADVECT), (2, [3, 3], 4, HEAT),
              (3, [1, 1, 1], 11, BURGERS)]


@pytest.mark.parametrize("geometry", ["affine", "regular"])
@pytest.mark.parametrize("dim,ne,p,eqn", DUDT_CASES)
def test_dudt_vjp_dot_product(ctx, dim, ne, p, eqn, geometry):
    """dudt is at most quadratic in u, so the central difference with a
    unit step is its exact JVP: (F(u+v) - F(u-v)) / 2 = F'(u) v."""
    g, prob = make(ctx, dim, ne, p, geometry)
    rng = np.random.default_rng(100 + p)
    B = GBurgers(prob, eqn, 0.05)
    nc = B.nstate
    rnd = lambda: [dev(rng.standard_normal(g.ndof())) for _ in range(nc)]
    u, v, w = rnd(), rnd(), rnd()
    c = [dev(rng.standard_normal(g.ndof())) for _ in range(dim)] if eqn == ADVECT else None
    Fp = dudt(B, prob, [a + b for a, b in zip(u, v)], c)
    Fm = dudt(B, prob, [a - b for a, b in zip(u, v)], c)
    Jv = [(a - b) / 2 for a, b in zip(Fp, Fm)]
    JTw = prob.zeros(ncomp=nc)
    B.dudt_vjp(u if eqn == BURGERS else None, c, w, JTw)
    a, b = vdot(Jv, w), vdot(v, JTw)
    # tolerance: 1e-11 of |Jv||w| (the unit step's rounding is relative to |F|)
    scale = vnorm(Jv) * vnorm(w) + vnorm(Fp) * vnorm(w) * 1e-3
    assert abs(a - b) <= 1e-11 * scale, (a, b)


def test_dudt_vjp_full_jacobian_2d(ctx):
    """Tiny Burgers case: every column of F'(u) (exact central difference)
    equals the corresponding row of the VJP applied to unit vectors."""
    g, prob = make(ctx, 2, [2, 2], 2)
    rng = np.random.default_rng(5)
    B = GBurgers(prob, BURGERS, 0.1)
    n = g.ndof()
    u = [dev(rng.standard_normal(n)) for _ in range(2)]
    Jac = np.zeros((2 * n, 2 * n))
    for col in range(2 * n):
        v = prob.zeros(ncomp=2)
        v[col // n][col % n] = 1.0
        Fp = dudt(B, prob, [a + b for a, b in zip(u, v)], None)
        Fm = dudt(B, prob, [a - b for a, b in zip(u, v)], None)
        Jac[:, col] = np.concatenate([((a - b) / 2).cpu().numpy() for a, b in zip(Fp, Fm)])
    JT = np.zeros((2 * n, 2 * n))
    for row in range(2 * n):
        w = prob.zeros(ncomp=2)
        w[row // n][row % n] = 1.0
        out = prob.zeros(ncomp=2)
        B.dudt_vjp(u, None, w, out)
        JT[:, row] = np.concatenate([a.cpu().numpy() for a in out])
    # tolerance: 1e-12 of max |J| entrywise
    assert np.max(np.abs(JT.T - Jac)) <= 1e-12 * np.max(np.abs(Jac))


# ---------------------------------------------------------------- RK step VJP
def rk_step(B, u0, c, dt):
    u = [a.clone() for a in u0]
    B.step(u, c, dt=dt, nsteps=1)
    return u


@pytest.mark.parametrize("scheme", [1, 2, 3, 4, 22, 33, 34])
@pytest.mark.parametrize("eqn", [HEAT, BURGERS, ADVECT])
def test_rk_step_vjp_dot_product(ctx, scheme, eqn):
    g, prob = make(ctx, 3, [2, 2, 2], 4)
    rng = np.random.default_rng(scheme * 7 + eqn)
    B = GBurgers(prob, eqn, 0.02, scheme=scheme)
    nc = B.nstate
    u0 = [dev(fourier_field(g, rng, amp=0.5)) for _ in range(nc)]
    c = [dev(fourier_field(g, rng, amp=1.0)) for _ in range(3)] if eqn == ADVECT else None
    v = [dev(rng.standard_normal(g.ndof())) for _ in range(nc)]
    w = [dev(rng.standard_normal(g.ndof())) for _ in range(nc)]
    dt = 2e-3
    # the heat and advection steps are linear: a unit central step is exact
    eps = 1e-4 if eqn == BURGERS else 1.0
    Gp = rk_step(B, [a + eps * b for a, b in zip(u0, v)], c, dt)
    Gm = rk_step(B, [a - eps * b for a, b in zip(u0, v)], c, dt)
    Jv = [(a - b) / (2 * eps) for a, b in zip(Gp, Gm)]
    lam = [a.clone() for a in w]
    B.step_vjp(u0, c, dt, lam)
    a, b = vdot(Jv, w), vdot(v, lam)
    # tolerance: 1e-11 (linear) / 1e-8 (Burgers, FD truncation and
    # rounding at eps = 1e-4) of |Jv||w|
    tol = 1e-8 if eqn == BURGERS else 1e-11
    assert abs(a - b) <= tol * vnorm(Jv) * vnorm(w), (a, b)


# ---------------------------------------------------------------- gradient
def misfit(B, prob, mass, u0, obs, dt, nsteps):
    u = [a.clone() for a in u0]
    B.step(u, None, dt=dt, nsteps=nsteps)
    return 0.5 * sum(float(torch.sum(mass * (a - o) ** 2)) for a, o in zip(u, obs))


def burgers_case(ctx, ne, p, nsteps, dt, nu=2e-3, scheme=A.GF_RK4, seed=2026):
    """Config shape: u_obs is the state after nsteps from a perturbed
    initial state (random Fourier k <= 4, amplitude 0.1)."""
    g, prob = make(ctx, 3, ne, p)
    rng = np.random.default_rng(seed)
    B = GBurgers(prob, BURGERS, nu, scheme=scheme)
    u0 = [dev(fourier_field(g, rng, amp=0.5)) for _ in range(3)]
    obs = [a + dev(fourier_field(g, rng, amp=0.1)) for a in u0]
    B.step(obs, None, dt=dt, nsteps=nsteps)
    mass = prob.zeros()
    GMass(prob).opVec_prod(torch.ones_like(mass), None, mass)
    return g, prob, B, u0, obs, mass, rng


def check_fd(B, prob, mass, u0, obs, grad, dt, nsteps, rng, ndir, eps=1e-6):
    for _ in range(ndir):
        v = [dev(rng.standard_normal(a.numel())) for a in u0]
        s = 1.0 / max(float(torch.max(torch.abs(x))) for x in v)
        v = [x * s for x in v]
        Jp = misfit(B, prob, mass, [a + eps * b for a, b in zip(u0, v)], obs, dt, nsteps)
        Jm = misfit(B, prob, mass, [a - eps * b for a, b in zip(u0, v)], obs, dt, nsteps)
        fd = (Jp - Jm) / (2 * eps)
        gv = vdot(grad, v)
        # tolerance: 1e-6 of max(|g.v|, 1e-3 |g||v|).  For random v in n
        # unknowns g.v ~ |g||v|/sqrt(n), so at the 16^3 p = 6 size (4.2e6
        # unknowns, g.v ~ 5e-4 |g||v|) the floor sets the bound, about 2e-6
        # of |g.v|; at the small sizes the relative term does.
        assert abs(fd - gv) <= 1e-6 * max(abs(gv), 1e-3 * vnorm(grad) * vnorm(v)), (fd, gv)


@pytest.mark.parametrize("scheme", [A.GF_RK4, A.GF_SSP33])
def test_adjoint_gradient_matches_fd_small(ctx, scheme):
    g, prob, B, u0, obs, mass, rng = burgers_case(ctx, [2, 2, 2], 4, 12, 2e-3, scheme=scheme)
    J, grad = B.adjoint_gradient(u0, None, obs, 2e-3, 12, checkpoint_every=5)
    # J itself: same misfit as the forward run (relative 1e-12)
    assert abs(J - misfit(B, prob, mass, u0, obs, 2e-3, 12)) <= 1e-12 * abs(J)
    check_fd(B, prob, mass, u0, obs, grad, 2e-3, 12, rng, ndir=5)


def test_adjoint_gradient_checkpoint_interval_invariant(ctx):
    g, prob, B, u0, obs, mass, rng = burgers_case(ctx, [2, 2, 2], 4, 9, 2e-3)
    ref = None
    for ck in (1, 2, 4, 9, 50):
        J, grad = B.adjoint_gradient(u0, None, obs, 2e-3, 9, checkpoint_every=ck)
        if ref is None:
            ref = (J, [a.clone() for a in grad])
        else:  # recomputation replays the same launches: bit-exact
            assert J == ref[0]
            assert all(torch.equal(a, b) for a, b in zip(grad, ref[1]))


def test_adjoint_gradient_zero_steps(ctx):
    g, prob, B, u0, obs, mass, rng = burgers_case(ctx, [1, 2, 1], 3, 2, 1e-3)
    J, grad = B.adjoint_gradient(u0, None, obs, 1e-3, 0, checkpoint_every=10)
    for a, o, gr in zip(u0, obs, grad):  # dJ/du0 = M (u0 - obs) with no steps
        assert torch.allclose(gr, mass * (a - o), rtol=0, atol=1e-15)


def test_adjoint_gradient_config_16cube_p6(ctx):
    """Adjoint config: 3D Burgers, 16^3 elements, p = 6, 50 RK4 steps,
    FP64, checkpoint every 10 steps; 20 random FD directions at eps = 1e-6
    and the step dot-product test at full size."""
    ne, p, nsteps, dt = [16, 16, 16], 6, 50, 1e-3
    g, prob, B, u0, obs, mass, rng = burgers_case(ctx, ne, p, nsteps, dt, nu=1e-3)
    J, grad = B.adjoint_gradient(u0, None, obs, dt, nsteps, checkpoint_every=10)
    assert np.isfinite(J) and J > 0
    check_fd(B, prob, mass, u0, obs, grad, dt, nsteps, rng, ndir=20)
    v = [dev(rng.standard_normal(a.numel())) for a in u0]
    w = [dev(rng.standard_normal(a.numel())) for a in u0]
    eps = 1e-4
    Gp = rk_step(B, [a + eps * b for a, b in zip(u0, v)], None, dt)
    Gm = rk_step(B, [a - eps * b for a, b in zip(u0, v)], None, dt)
    Jv = [(a - b) / (2 * eps) for a, b in zip(Gp, Gm)]
    lam = [a.clone() for a in w]
    B.step_vjp(u0, None, dt, lam)
    # tolerance: 1e-8 of |Jv||w|
    assert abs(vdot(Jv, w) - vdot(v, lam)) <= 1e-8 * vnorm(Jv) * vnorm(w)


# ---------------------------------------------------------------- autograd harness
class RKStepFn(torch.autograd.Function):
    """One RK step as a differentiable torch op over the C ABI (gradient
    checks only)."""

    @staticmethod
    def forward(ctx, B, dt, *u0):
        ctx.B, ctx.dt = B, dt
        ctx.save_for_backward(*u0)
        return tuple(rk_step(B, [a.detach() for a in u0], None, dt))

    @staticmethod
    def backward(ctx, *gout):
        u0 = ctx.saved_tensors
        lam = [gi.detach().clone().contiguous() for gi in gout]
        ctx.B.step_vjp(list(u0), None, ctx.dt, lam)
        return (None, None, *lam)


class MisfitFn(torch.autograd.Function):
    """J(u0) through nsteps steps; backward = the checkpointed adjoint."""

    @staticmethod
    def forward(ctx, B, obs, dt, nsteps, ck, *u0):
        J, grad = B.adjoint_gradient([a.detach() for a in u0], None, obs, dt, nsteps, ck)
        ctx.save_for_backward(*grad)
        return torch.tensor(J, dtype=torch.float64, device=u0[0].device)

    @staticmethod
    def backward(ctx, gJ):
        return (None, None, None, None, None, *[gJ * gr for gr in ctx.saved_tensors])


@pytest.mark.parametrize("scheme", [A.GF_RK4, A.GF_SSP34])
def test_autograd_gradcheck_rk_step(ctx, scheme):
    g, prob = make(ctx, 2, [2, 2], 2)
    rng = np.random.default_rng(8)
    B = GBurgers(prob, BURGERS, 0.05, scheme=scheme)
    u0 = tuple(dev(0.5 * rng.standard_normal(g.ndof())).requires_grad_() for _ in range(2))
    assert torch.autograd.gradcheck(lambda *u: RKStepFn.apply(B, 1e-2, *u), u0, eps=1e-6,
                                    atol=1e-8, rtol=1e-6)


def test_autograd_gradcheck_misfit(ctx):
    g, prob = make(ctx, 2, [2, 2], 3)
    rng = np.random.default_rng(9)
    B = GBurgers(prob, BURGERS, 0.05, scheme=A.GF_RK4)
    u0 = tuple(dev(0.5 * rng.standard_normal(g.ndof())).requires_grad_() for _ in range(2))
    obs = [dev(0.5 * rng.standard_normal(g.ndof())) for _ in range(2)]
    assert torch.autograd.gradcheck(lambda *u: MisfitFn.apply(B, obs, 5e-3, 7, 3, *u), u0,
                                    eps=1e-6, atol=1e-8, rtol=1e-6)


def test_adjoint_rejects_bad_arguments(ctx):
    g, prob = make(ctx, 2, [2, 2], 3)
    lib = A.load()
    B = GBurgers(prob, BURGERS, 0.05)
    u = prob.zeros(ncomp=2)
    tr = B.traits()
    u32 = [a.float() for a in u]
    assert lib.gf_rk_step_vjp(prob.handle, A.GF_F32, C.byref(tr), A.ptr_array(u32), None, 1e-3,
                              A.ptr_array(u32)) == A.GF_ERR_ARG
    J = C.c_double()
    assert lib.gf_adjoint_gradient(prob.handle, C.byref(tr), A.ptr_array(u), None, A.ptr_array(u),
                                   1e-3, 3, 0, C.byref(J), A.ptr_array(u)) == A.GF_ERR_ARG
