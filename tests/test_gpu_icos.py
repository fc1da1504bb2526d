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
