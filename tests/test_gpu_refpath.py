"""GPU results against the reference's own code: the committed fixture
tests/golden/ref_path.npz holds what the reference's GGFX, GHelmholtz,
GAdvect, GCG and GBurgers/GExRKStepper computed (compiled from its sources,
tests/golden/make_path_golden.py), and each test runs the same inputs
through the C ABI on the GPU.

Stated error bounds (relative, max-norm over the field):
  gather-scatter                      bit-exact (FP64)
  FP64 operator applies               1e-12
  FP64 CG solution (both to 1e-13)    1e-10;  iterations within 2
  FP64 RK runs                        1e-10
  FP32 operator applies               1e-5
  FP32 RK: 2-d advection, RK4, 200 steps        2e-6
           3-d Burgers, SSP-RK3, 100 steps      2e-5
"""
import numpy as np
import pytest
import torch

from geoflow_b200 import (CGTraits, GBurgers, GCG, GGFX, GHelmholtz, GridBox, Problem,
                          _abi as A)

pytestmark = pytest.mark.gpu

GRIDS = {"2d_dir": (2, [4, 3], 4, [0, 0]), "2d_per": (2, [4, 3], 4, [1, 1]),
         "3d_dir": (3, [2, 3, 2], 3, [0, 0, 0]), "3d_per": (3, [2, 2, 3], 4, [1, 1, 1])}
SCHEME = {(1, 0): A.GF_RK1, (2, 0): A.GF_RK2, (3, 0): A.GF_RK3, (4, 0): A.GF_RK4,
          (2, 1): A.GF_SSP22, (3, 1): A.GF_SSP33}
OPS = [GGFX.Sum, GGFX.Smooth, GGFX.Max, GGFX.Min]

FP32_RK_CFG1 = 2e-6
FP32_RK_CFG3 = 2e-5


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def host(t):
    return t.detach().cpu().numpy().astype(np.float64)


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def problem(ctx, dim, ne, p, per, length=None):
    g = GridBox(dim, ne, p, periodic=per, length=length)
    return g, Problem(ctx, g, dirichlet_mask=not all(per))


@pytest.mark.parametrize("tag", list(GRIDS))
def test_grid_matches_reference(ctx, refpath, tag):
    dim, ne, p, per = GRIDS[tag]
    g, prob = problem(ctx, dim, ne, p, per)
    k = f"grid_{tag}_"
    assert np.array_equal(g.mask, refpath[k + "mask"])
    assert np.array_equal(host(GGFX(prob).get_imult()), refpath[k + "imult"])


@pytest.mark.parametrize("tag", list(GRIDS))
@pytest.mark.parametrize("op", range(4))
def test_dss_bit_exact_vs_reference(ctx, refpath, tag, op):
    dim, ne, p, per = GRIDS[tag]
    g, prob = problem(ctx, dim, ne, p, per)
    k = f"grid_{tag}_"
    u = dev(refpath[k + "u"])
    GGFX(prob).doOp(u, OPS[op])
    assert np.array_equal(host(u).view(np.uint64), refpath[k + f"dss{op}"].view(np.uint64))


@pytest.mark.parametrize("tag", list(GRIDS))
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_helmholtz_vs_reference(ctx, refpath, tag, dtype, tol):
    dim, ne, p, per = GRIDS[tag]
    g, prob = problem(ctx, dim, ne, p, per)
    k = f"grid_{tag}_"
    u, q, pv = (dev(refpath[k + s], dtype) for s in ("u", "q", "pv"))
    for pl, ref in ((0.7, refpath[k + "helm_s"]), (pv, refpath[k + "helm_v"])):
        H = GHelmholtz(prob)
        H.set_Lap_scalar(pl)
        H.set_mass_scalar(q)
        uo = prob.zeros(dtype)
        H.opVec_prod(u, None, uo)
        assert relerr(host(uo), ref) < tol


@pytest.mark.parametrize("tag", list(GRIDS))
def test_advect_vs_reference(ctx, refpath, tag):
    dim, ne, p, per = GRIDS[tag]
    g, prob = problem(ctx, dim, ne, p, per)
    k = f"grid_{tag}_"
    u = dev(refpath[k + "u"])
    c = [dev(a) for a in refpath[k + "c"]]
    po = prob.zeros()
    lib = A.load()
    ctx.check(lib.gf_advect_apply(prob.handle, A.GF_F64, A.ptr(u), dim, A.ptr_array(c),
                                  A.ptr(po)))
    assert relerr(host(po), refpath[k + "adv"]) < 1e-12


@pytest.mark.parametrize("tag,dim,ne,p", [("2d", 2, [5, 4], 5), ("3d", 3, [3, 3, 2], 4)])
def test_cg_solution_vs_reference(ctx, refpath, tag, dim, ne, p):
    """Jacobi-PCG on H = M + K with the reference's right-hand side, both
    solvers to 1e-13: solutions within 1e-10, iteration counts within 2."""
    g, prob = problem(ctx, dim, ne, p, [0] * dim)
    k = f"cgt_{tag}_"
    H = GHelmholtz(prob)
    H.set_mass_scalar(1.0)
    x = prob.zeros()
    cg = GCG(CGTraits(maxit=2000, tol=1e-13, precond=A.GF_PRECOND_JACOBI), prob)
    rc = cg.solve(H, dev(refpath[k + "b"]), prob.zeros(), x)
    rc_r, it_r = (int(v) for v in refpath[k + "info"])
    assert rc == rc_r == 0
    assert abs(cg.iter_ - it_r) <= 2
    assert relerr(host(x), refpath[k + "x"]) < 1e-10


def _rk_tags(refpath):
    return sorted({k[3:-5] for k in refpath.files if k.startswith("rk_") and k.endswith("_info")})


@pytest.mark.parametrize("i", range(22))
def test_rk_vs_reference(ctx, refpath, i):
    tag = _rk_tags(refpath)[i]
    k = f"rk_{tag}_"
    dim, p, order, ssp, kind, nsteps = (int(v) for v in refpath[k + "info"])
    ne = [int(v) for v in refpath[k + "ne"]]
    g, prob = problem(ctx, dim, ne, p, [1] * dim)
    u = [dev(a) for a in refpath[k + "u0"]]
    c = [dev(np.full(g.ndof(), 1.0 - 0.5 * d)) for d in range(dim)] if kind == 0 else None
    B = GBurgers(prob, kind, 0.01, scheme=SCHEME[(order, ssp)])
    B.step(u, c, dt=float(refpath[k + "dt"][0]), nsteps=nsteps)
    for a, b in zip(u, refpath[k + "u"]):
        assert relerr(host(a), b) < 1e-10, tag


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-10), (torch.float32, FP32_RK_CFG1)])
def test_advection_2d_full_200_steps_vs_reference(ctx, refpath, dtype, tol):
    """16^2 elements, p = 4, c = (1, 0.5), nu = 0.01, RK4, dt = 1e-4,
    200 steps, against the reference's own run of the same case."""
    g, prob = problem(ctx, 2, [16, 16], 4, [1, 1])
    u = [dev(refpath["cfg1_u0"], dtype)]
    c = [dev(np.ones(g.ndof()), dtype), dev(np.full(g.ndof(), 0.5), dtype)]
    GBurgers(prob, GBurgers.ADVECT, 0.01, scheme=A.GF_RK4).step(u, c, dt=1e-4, nsteps=200)
    assert relerr(host(u[0]), refpath["cfg1_u200"]) < tol


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-10), (torch.float32, FP32_RK_CFG3)])
def test_burgers_3d_100_steps_vs_reference(ctx, refpath, dtype, tol):
    """The 3-d Burgers case (nu = 1e-3, SSP-RK3, CFL 0.3, 100 steps) on a
    3^3-element p = 5 periodic box, against the reference's own run."""
    g, prob = problem(ctx, 3, [3] * 3, 5, [1] * 3, length=[2 * np.pi] * 3)
    u = [dev(a, dtype) for a in refpath["cfg3s_u0"]]
    B = GBurgers(prob, GBurgers.BURGERS, 1e-3, scheme=A.GF_SSP33)
    B.step(u, None, dt=float(refpath["cfg3s_dt"][0]), nsteps=100)
    for a, b in zip(u, refpath["cfg3s_u100"]):
        assert relerr(host(a), b) < tol
