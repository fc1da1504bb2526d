"""The FP32 3-d apply at p = 7 with its line contractions as 3xTF32
tensor-core products (GF_FP32_APPLY_TF32, k_helm_tf32.cuh) against the
oracle's FP64 apply (FP32 bound 1e-5 relative, max-norm) and against the
FP32x2-FMA kernel; and the multigrid-preconditioned solve, whose FP32
applies it replaces, reaching the same solution."""
import numpy as np
import pytest
import torch

import oracle as O
from geoflow_b200 import CGTraits, GCG, GHelmholtz, GridBox, Problem, _abi as A

pytestmark = pytest.mark.gpu


@pytest.fixture
def tf32_mode():
    lib = A.load()
    prev = lib.gf_set_fp32_apply(A.GF_FP32_APPLY_TF32)
    yield lib
    lib.gf_set_fp32_apply(prev)


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("ne,per,qv", [([2, 2, 2], None, False), ([3, 2, 2], [1, 0, 1], False),
                                       ([2, 3, 2], None, True), ([5, 3, 2], [1, 1, 1], True)])
def test_tf32_apply_matches_oracle(ctx, tf32_mode, ne, per, qv):
    g = GridBox(3, ne, 7, periodic=per, length=[1.0, 0.7, 1.3])
    o = O.OracleBox(3, ne, 7, periodic=per, length=[1.0, 0.7, 1.3])
    prob = Problem(ctx, g)
    rng = np.random.default_rng(31)
    u = rng.standard_normal(g.ndof())
    q = 0.5 + rng.random(g.ndof()) if qv else np.full(g.ndof(), 0.8)
    ref = o.helmholtz(u, p=1.3, q_vec=q)
    H = GHelmholtz(prob)
    H.set_Lap_scalar(1.3)
    H.set_mass_scalar(torch.from_numpy(q).to("cuda", torch.float32) if qv else 0.8)
    ut = torch.from_numpy(u).to("cuda", torch.float32)
    out = {}
    for mode in (A.GF_FP32_APPLY_TF32, A.GF_FP32_APPLY_FMA):
        tf32_mode.gf_set_fp32_apply(mode)
        uo = prob.zeros(torch.float32)
        H.opVec_prod(ut, None, uo)
        out[mode] = uo.double().cpu().numpy()
        assert relerr(out[mode], ref) < 1e-5, mode
    tf32_mode.gf_set_fp32_apply(A.GF_FP32_APPLY_TF32)
    assert relerr(out[A.GF_FP32_APPLY_TF32], out[A.GF_FP32_APPLY_FMA]) < 2e-6


def test_tf32_pmg_solve_matches_fp64(ctx, tf32_mode):
    g = GridBox(3, [6, 6, 6], 7)
    prob = Problem(ctx, g)
    rng = np.random.default_rng(3)
    f = rng.standard_normal(g.nclass)[g.node_class]
    w3 = np.einsum("k,j,i->kji", g.W, g.W, g.W).ravel()
    eg = g.elem_geom.reshape(g.nelems, 4)
    b = torch.from_numpy((eg[:, 3][:, None] * w3[None, :]).ravel() * f).to("cuda")
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    common = dict(maxit=3000, tol=1e-12, normtype=A.GF_NORM_EUC, relative=1)
    xj = prob.zeros()
    assert GCG(CGTraits(precond=A.GF_PRECOND_JACOBI, **common), prob).solve(
        H, b, prob.zeros(), xj) == 0
    its = {}
    for mode in (A.GF_FP32_APPLY_TF32, A.GF_FP32_APPLY_FMA):
        tf32_mode.gf_set_fp32_apply(mode)
        x = prob.zeros()
        cg = GCG(CGTraits(precond=A.GF_PRECOND_PMG, poly_degree=1, **common), prob)
        assert cg.solve(H, b, prob.zeros(), x) == 0
        its[mode] = cg.iter_
        assert float((x - xj).abs().max() / xj.abs().max()) < 1e-9
    assert abs(its[A.GF_FP32_APPLY_TF32] - its[A.GF_FP32_APPLY_FMA]) <= 1
