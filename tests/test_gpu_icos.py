"""Operators and stepping on the icosahedral sphere (GF_GEOM_EMBEDDED
problems from gf_icos_grid) against the reference's own GGridIcos, GGFX,
GHelmholtz::embed_prod, GAdvect and GBurgers (fixture
tests/golden/ref_path.npz).  Bounds: gather-scatter bit-exact; operators
1e-11 relative (the grids' metrics agree to ~1e-14); the cosine bell in the
solid-body wind, RK4 over 20 steps, 1e-10."""
import numpy as np
import pytest
import torch

from geoflow_b200 import GBurgers, GGFX, GHelmholtz, IcosGrid, _abi as A

pytestmark = pytest.mark.gpu

CASES = {"l0p4": (0, 4, A.GF_ICOS_BISECTION), "l1p2lag": (1, 2, A.GF_ICOS_LAGRANGIAN)}
OPS = [GGFX.Sum, GGFX.Smooth, GGFX.Max, GGFX.Min]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("tag", list(CASES))
def test_icos_operators_vs_reference(ctx, refpath, tag):
    level, p, refine = CASES[tag]
    g = IcosGrid(level, p, refine=refine)
    prob = g.problem(ctx)
    k = f"icos_{tag}_"
    for op in range(4):
        u = dev(refpath[k + "u"])
        GGFX(prob).doOp(u, OPS[op])
        assert np.array_equal(u.cpu().numpy().view(np.uint64), refpath[k + f"dss{op}"].view(np.uint64))
    H = GHelmholtz(prob)
    H.set_Lap_scalar(0.7)
    H.set_mass_scalar(dev(refpath[k + "q"]))
    uo = prob.zeros()
    H.opVec_prod(dev(refpath[k + "u"]), None, uo)
    assert rel(uo.cpu().numpy(), refpath[k + "helm"]) < 1e-11
    c = [dev(a) for a in refpath[k + "c"]]
    po = prob.zeros()
    ctx.check(A.load().gf_advect_apply(prob.handle, A.GF_F64, A.ptr(dev(refpath[k + "u"])), 3,
                                       A.ptr_array(c), A.ptr(po)))
    assert rel(po.cpu().numpy(), refpath[k + "adv"]) < 1e-11


def test_cosine_bell_advection_vs_reference(ctx, refpath):
    g = IcosGrid(1, 3)
    prob = g.problem(ctx)
    u = [dev(refpath["icosadv_u0"])]
    c = [dev(a) for a in refpath["icosadv_c"]]
    B = GBurgers(prob, GBurgers.ADVECT, 1e-3, scheme=A.GF_RK4)
    B.step(u, c, dt=float(refpath["icosadv_dt"][0]), nsteps=20)
    assert rel(u[0].cpu().numpy(), refpath["icosadv_u"]) < 1e-10


@pytest.mark.parametrize("dtype,bound,tiny", [(torch.float64, 1e-12, 1e-300),
                                              (torch.float32, 2e-5, 1e-30)])
def test_prescribed_velocity_fast_path_matches_general_kernel(ctx, dtype, bound, tiny):
    """Pure advection with nu = 0 takes the coefficient-plane path
    (k_def.cuh adv_element: b_j = -(imass M) sum_k c_k dXi_j/dX_k formed
    once per advance); it differs from the general kernel (taken for any
    nu != 0; here nu = 1e-300 in FP64, 1e-30 in FP32, whose diffusion term
    is below the rounding)
    only by rounding order: 1e-12 relative (FP64) and 2e-5 (FP32) after
    10 RK4 steps on the level-1 p = 5 sphere."""
    from geoflow_b200 import workloads as W
    g = IcosGrid(1, 5)
    prob = g.problem(ctx)
    u0 = W.icos_cosine_bell(g.xyz, 0.3, 1.2)
    c = W.icos_solid_body_wind(g.xyz, alpha=0.4)
    dt = 0.25 * g.minnodedist
    out = []
    for nu in (0.0, tiny):
        u = [torch.from_numpy(u0).to("cuda", dtype)]
        cc = [torch.from_numpy(a).to("cuda", dtype) for a in c]
        GBurgers(prob, GBurgers.ADVECT, nu, scheme=A.GF_RK4).step(u, cc, dt=dt, nsteps=10)
        out.append(u[0].double().cpu().numpy())
    assert not np.array_equal(out[0], u0)
    assert rel(out[0], out[1]) < bound


def test_cdg_mass_icos_integral_on_gpu(ctx):
    """cdg_mass.cpp with data/mass_input.jsn: on the icosahedral sphere
    (GICOS_BISECTION, ilevel 2, p = 4, radius 1) the device integral of 1 is
    the sphere's area 4 pi r^2 within the test's 1e-10 relative; the FP32
    integral within FP32 rounding."""
    import ctypes as C
    g = IcosGrid(2, 4, radius=1.0)
    prob = g.problem(ctx)
    lib = A.load()
    r = C.c_double()
    ones = torch.ones(g.ndof(), dtype=torch.float64, device="cuda")
    ctx.check(lib.gf_integrate(prob.handle, A.GF_F64, A.ptr(ones), C.byref(r)))
    assert abs(r.value - 4.0 * np.pi) / (4.0 * np.pi) < 1e-10
    ctx.check(lib.gf_integrate(prob.handle, A.GF_F32, A.ptr(ones.float()), C.byref(r)))
    assert abs(r.value - 4.0 * np.pi) / (4.0 * np.pi) < 1e-5
