"""CG with the FP32 p/h-multigrid preconditioner (GF_PRECOND_PMG) against
plain FP64 Jacobi-PCG: the same 1e-12 relative residual, solutions within
~kappa * 1e-12 of each other (1e-9 relative), in a handful of FP64
iterations independent of the element count; the cached hierarchy gives
bit-identical repeated solves.
"""
import ctypes as C

import numpy as np
import pytest

from geoflow_b200 import CGTraits, GCG, GHelmholtz, GridBox, Problem, _abi as A

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def host(t):
    return t.detach().cpu().numpy()


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rhs(g, seed):
    """b = M f for a continuous f (one value per lattice point)."""
    rng = np.random.default_rng(seed)
    f = rng.standard_normal(g.ndof())
    f = f[g.members[g.class_ptr[:-1]]][g.node_class]
    w3 = np.einsum("k,j,i->kji", *([g.W] * g.dim)).ravel() if g.dim == 3 else \
        np.einsum("j,i->ji", g.W, g.W).ravel()
    eg = g.elem_geom.reshape(g.nelems, g.dim + 1)
    mass = (eg[:, g.dim][:, None] * w3[None, :]).ravel()
    return mass * f


COMMON = dict(maxit=3000, tol=1e-12, normtype=A.GF_NORM_EUC, relative=1)

CASES = [(3, [4, 4, 4], 7, None, 2), (3, [4, 2, 4], 5, [1, 0, 1], 2), (3, [2, 2, 2], 3, None, 3),
         (3, [3, 2, 2], 4, None, 1), (2, [8, 8], 6, None, 2), (2, [6, 4], 4, [1, 1], 2),
         (3, [8, 8, 8], 2, None, 2), (3, [2, 2, 2], 1, [1, 1, 1], 2)]


@pytest.mark.parametrize("dim,ne,p,per,m", CASES)
def test_pmg_reaches_fp64_solution(ctx, dim, ne, p, per, m):
    g = GridBox(dim, ne, p, periodic=per)
    prob = Problem(ctx, g)
    b = rhs(g, 3 + p)
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    xj = prob.zeros()
    cgj = GCG(CGTraits(precond=A.GF_PRECOND_JACOBI, **COMMON), prob)
    assert cgj.solve(H, dev(b), dev(0 * b), xj) == 0
    xm = prob.zeros()
    cgm = GCG(CGTraits(precond=A.GF_PRECOND_PMG, poly_degree=m, **COMMON), prob)
    assert cgm.solve(H, dev(b), dev(0 * b), xm) == 0
    assert relerr(host(xm), host(xj)) < 1e-9
    assert cgm.iter_ <= 40
    if g.nelems * p ** dim >= 512:
        assert cgm.iter_ < cgj.iter_


@pytest.mark.parametrize("per", [[1, 0, 0], [0, 0, 0]])
def test_pmg_long_lattice_rows(ctx, per):
    """Lattice rows longer than a block (40 elements at p = 7 along x) are
    walked in segments; isotropic elements (box 20 x 1 x 1)."""
    g = GridBox(3, [40, 2, 2], 7, length=[20.0, 1.0, 1.0], periodic=per)
    prob = Problem(ctx, g)
    b = rhs(g, 13)
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    xj = prob.zeros()
    assert GCG(CGTraits(precond=A.GF_PRECOND_JACOBI, **COMMON), prob).solve(
        H, dev(b), dev(0 * b), xj) == 0
    xm = prob.zeros()
    cgm = GCG(CGTraits(precond=A.GF_PRECOND_PMG, **COMMON), prob)
    assert cgm.solve(H, dev(b), dev(0 * b), xm) == 0
    assert relerr(host(xm), host(xj)) < 1e-9
    assert cgm.iter_ <= 30


def test_pmg_iterations_independent_of_element_count(ctx):
    its = []
    for ne in (2, 4, 8):
        g = GridBox(3, [ne] * 3, 5)
        prob = Problem(ctx, g)
        b = rhs(g, 11)
        H = GHelmholtz(prob)
        H.set_mass_scalar(1.0)
        x = prob.zeros()
        cg = GCG(CGTraits(precond=A.GF_PRECOND_PMG, **COMMON), prob)
        assert cg.solve(H, dev(b), dev(0 * b), x) == 0
        its.append(cg.iter_)
    assert max(its) <= min(its) + 6, its


def test_pmg_hierarchy_reuse_is_bit_identical_and_rebuilds_on_change(ctx):
    g = GridBox(3, [4, 4, 2], 6)
    prob = Problem(ctx, g)
    b = dev(rhs(g, 5))
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    cg = GCG(CGTraits(precond=A.GF_PRECOND_PMG, **COMMON), prob)
    xs = []
    for _ in range(2):
        x = prob.zeros()
        assert cg.solve(H, b, 0 * b, x) == 0
        xs.append(x)
    assert bool((xs[0] == xs[1]).all())
    # another operator (p = 0.5 Laplacian + mass): the hierarchy is rebuilt
    H2 = GHelmholtz(prob)
    H2.set_Lap_scalar(0.5)
    H2.set_mass_scalar(1.0)
    x2 = prob.zeros()
    assert cg.solve(H2, b, 0 * b, x2) == 0
    xj = prob.zeros()
    cgj = GCG(CGTraits(precond=A.GF_PRECOND_JACOBI, **COMMON), prob)
    assert cgj.solve(H2, b, 0 * b, xj) == 0
    assert relerr(host(x2), host(xj)) < 1e-9


def test_pmg_residual_history_is_recorded(ctx):
    g = GridBox(3, [4, 4, 4], 5)
    prob = Problem(ctx, g)
    b = dev(rhs(g, 7))
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    cg = GCG(CGTraits(precond=A.GF_PRECOND_PMG, **COMMON), prob)
    x = prob.zeros()
    assert cg.solve(H, b, 0 * b, x) == 0
    res = cg.get_residuals()
    assert len(res) == cg.iter_ and res[-1] == cg.rnorm_
    assert res[-1] < 1e-6 * res[0] and np.all(res > 0)


def test_pmg_refuses_unstructured_problem(ctx):
    g = GridBox(3, [2, 2, 2], 3)
    prob = Problem(ctx, g, structured=False)
    lib = A.load()
    tr = CGTraits(precond=A.GF_PRECOND_PMG, **COMMON).to_c()
    b = prob.zeros()
    x = prob.zeros()
    it, rn = C.c_int(), C.c_double()
    assert lib.gf_cg_solve(prob.handle, C.byref(tr), 1.0, 1.0, 1, A.ptr(b), A.ptr(b), A.ptr(x),
                           C.byref(it), C.byref(rn), None) == A.GF_ERR_UNSUPPORTED


@pytest.mark.parametrize("dim,ne,p,per,m", CASES)
def test_pmg64_reaches_fp64_solution(ctx, dim, ne, p, per, m):
    """The FP64 V-cycle (GF_PRECOND_PMG64): the same solution as Jacobi-PCG
    and, on the same hierarchy, no more iterations than the FP32 V-cycle
    (the two preconditioners differ by FP32 rounding only)."""
    g = GridBox(dim, ne, p, periodic=per)
    prob = Problem(ctx, g)
    b = rhs(g, 3 + p)
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    xj = prob.zeros()
    assert GCG(CGTraits(precond=A.GF_PRECOND_JACOBI, **COMMON), prob).solve(
        H, dev(b), dev(0 * b), xj) == 0
    its = {}
    for pc in (A.GF_PRECOND_PMG64, A.GF_PRECOND_PMG):
        x = prob.zeros()
        cg = GCG(CGTraits(precond=pc, poly_degree=m, **COMMON), prob)
        assert cg.solve(H, dev(b), dev(0 * b), x) == 0
        assert relerr(host(x), host(xj)) < 1e-9
        its[pc] = cg.iter_
    assert its[A.GF_PRECOND_PMG64] <= its[A.GF_PRECOND_PMG] + 1, its


def test_pmg64_and_pmg_alternate_on_one_problem(ctx):
    """Switching between the FP64 and FP32 V-cycles on one problem rebuilds
    the hierarchy each time; a repeated solve with either is bit-identical."""
    g = GridBox(3, [4, 4, 2], 5)
    prob = Problem(ctx, g)
    b = dev(rhs(g, 9))
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    out = {}
    for pc in (A.GF_PRECOND_PMG64, A.GF_PRECOND_PMG, A.GF_PRECOND_PMG64, A.GF_PRECOND_PMG):
        x = prob.zeros()
        cg = GCG(CGTraits(precond=pc, **COMMON), prob)
        assert cg.solve(H, b, 0 * b, x) == 0
        if pc in out:
            assert bool((out[pc] == x).all())
        out[pc] = x
    assert relerr(host(out[A.GF_PRECOND_PMG64]), host(out[A.GF_PRECOND_PMG])) < 1e-9


@pytest.mark.parametrize("pc", [A.GF_PRECOND_PMG, A.GF_PRECOND_PMG64])
def test_pmg_launch_single_kernels(ctx, pc):
    """gf_pmg_launch (single finest-level kernels for timing): refused before
    the hierarchy exists and for other preconditioners; after
    GF_PMG_PREPARE every selector launches, and a later solve on the same
    hierarchy is bit-identical to the one before the launches."""
    g = GridBox(3, [4, 4, 4], 5)
    prob = Problem(ctx, g)
    b = dev(rhs(g, 21))
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    lib = A.load()
    tr = CGTraits(precond=pc, **COMMON)
    trc = tr.to_c()
    assert lib.gf_pmg_launch(prob.handle, C.byref(trc), 1.0, 1.0, 1, 1,
                             A.GF_PMG_STEP) == A.GF_ERR_ARG
    bad = CGTraits(precond=A.GF_PRECOND_JACOBI, **COMMON).to_c()
    assert lib.gf_pmg_launch(prob.handle, C.byref(bad), 1.0, 1.0, 1, 1,
                             A.GF_PMG_PREPARE) == A.GF_ERR_ARG
    cg = GCG(tr, prob)
    x1 = prob.zeros()
    assert cg.solve(H, b, 0 * b, x1) == 0
    for which in (A.GF_PMG_PREPARE, A.GF_PMG_APPLY64, A.GF_PMG_APPLY, A.GF_PMG_STEP,
                  A.GF_PMG_RESID, A.GF_PMG_RESTRICT, A.GF_PMG_PROLONG):
        assert lib.gf_pmg_launch(prob.handle, C.byref(trc), 1.0, 1.0, 1, 1, which) == 0
    x2 = prob.zeros()
    assert cg.solve(H, b, 0 * b, x2) == 0
    assert bool((x1 == x2).all())
