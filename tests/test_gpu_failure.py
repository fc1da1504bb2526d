"""Failure semantics on the GPU, made on the host (no device fault):

* maxit spent before the stop rule holds returns GCGERR_NOCONVERGE
  (solvers/gcg.ipp:339-341) on every CG path: plain FP64 Jacobi-PCG, the
  mixed FP32/FP64 solve, the Chebyshev-preconditioned solve and the
  multigrid-preconditioned solve, whose loop runs inside a device WHILE
  graph node (the exit on maxit is taken on the device);
* a non-finite right-hand side returns GF_ERR_NONFINITE before the first
  iteration on every path;
* the RK stepper returns GF_ERR_NONFINITE for a state that is not finite
  after its steps (GBurgers::step_impl asserts it, pdes/gburgers.ipp:
  325-331), and keeps a usable context afterwards.
"""
import numpy as np
import pytest
import torch

from geoflow_b200 import CGTraits, GBurgers, GCG, GHelmholtz, GridBox, Problem, _abi as A

pytestmark = pytest.mark.gpu

PATHS = {
    "jacobi": dict(precond=A.GF_PRECOND_JACOBI),
    "mixed": dict(precond=A.GF_PRECOND_JACOBI, precision=A.GF_CG_MIXED, check_every=4),
    "chebyshev": dict(precond=A.GF_PRECOND_CHEBYSHEV, poly_degree=2),
    "pmg": dict(precond=A.GF_PRECOND_PMG, poly_degree=1),
    "pmg64": dict(precond=A.GF_PRECOND_PMG64, poly_degree=1),
}


def helmholtz_problem(ctx):
    g = GridBox(3, [4, 4, 4], 5)
    prob = Problem(ctx, g)
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    rng = np.random.default_rng(11)
    f = rng.standard_normal(g.nclass)[g.node_class]
    w3 = np.einsum("k,j,i->kji", g.W, g.W, g.W).ravel()
    eg = g.elem_geom.reshape(g.nelems, 4)
    b = (eg[:, 3][:, None] * w3[None, :]).ravel() * f
    return g, prob, H, b


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.mark.parametrize("path", list(PATHS))
def test_maxit_returns_noconverge(ctx, path):
    g, prob, H, b = helmholtz_problem(ctx)
    maxit = 3
    cg = GCG(CGTraits(maxit=maxit, tol=1e-12, **PATHS[path]), prob)
    x = prob.zeros()
    rc = cg.solve(H, dev(b), prob.zeros(), x)
    assert rc == GCG.GCGERR_NOCONVERGE
    assert 1 <= cg.iter_ <= maxit
    assert torch.isfinite(x).all()
    # the same solver converges with room to iterate
    cg2 = GCG(CGTraits(maxit=3000, tol=1e-12, **PATHS[path]), prob)
    x2 = prob.zeros()
    assert cg2.solve(H, dev(b), prob.zeros(), x2) == GCG.GCGERR_NONE


@pytest.mark.parametrize("path", list(PATHS))
def test_nonfinite_rhs_is_reported(ctx, path):
    g, prob, H, b = helmholtz_problem(ctx)
    bad = b.copy()
    bad[g.ndof() // 3] = np.nan
    cg = GCG(CGTraits(maxit=50, tol=1e-10, **PATHS[path]), prob)
    with pytest.raises(A.GFError) as e:
        cg.solve(H, dev(bad), prob.zeros(), prob.zeros())
    assert e.value.code == A.GF_ERR_NONFINITE
    assert cg.iter_ == 0
    # the context and problem stay usable
    x = prob.zeros()
    assert GCG(CGTraits(maxit=3000, tol=1e-10, **PATHS[path]), prob).solve(
        H, dev(b), prob.zeros(), x) == 0


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_rk_nonfinite_state_is_reported(ctx, dtype):
    g = GridBox(3, [2, 2, 2], 4, periodic=[1, 1, 1])
    prob = Problem(ctx, g, dirichlet_mask=False)
    rng = np.random.default_rng(5)
    u0 = [0.1 * rng.standard_normal(g.nclass)[g.node_class] for _ in range(3)]
    B = GBurgers(prob, GBurgers.BURGERS, 1e-2, scheme=A.GF_SSP33)
    u = [dev(a, dtype) for a in u0]
    B.step(u, None, dt=1e-3, nsteps=2)
    assert all(bool(torch.isfinite(t).all()) for t in u)
    u[1][7] = float("inf")
    with pytest.raises(A.GFError) as e:
        B.step(u, None, dt=1e-3, nsteps=2)
    assert e.value.code == A.GF_ERR_NONFINITE
    u = [dev(a, dtype) for a in u0]
    B.step(u, None, dt=1e-3, nsteps=1)
    assert all(bool(torch.isfinite(t).all()) for t in u)
