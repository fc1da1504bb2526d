"""The icosahedral sphere (GGridIcos, GE_2DEMBEDDED) built by the library's
host-side generator (gf_icos_grid) against the reference's own GGridIcos
compiled from its sources (fixture tests/golden/ref_path.npz): node
coordinates bit-identical, the embedded metric dXi/dX and the Jacobian
within 1e-12 (the reference differentiates its shape functions with
GLLBasis::evalDBasis, the library with the GLL derivative matrix; they
differ in the last bits), and the coordinate-matched gather-scatter
classes folding to the reference's GGFX results bit for bit."""
import numpy as np
import pytest

import oracle as O
from geoflow_b200 import IcosGrid, _abi as A

CASES = {"l0p4": (0, 4, A.GF_ICOS_BISECTION), "l1p2lag": (1, 2, A.GF_ICOS_LAGRANGIAN)}


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("tag", list(CASES))
def test_icos_grid_matches_reference(refpath, tag):
    level, p, refine = CASES[tag]
    g = IcosGrid(level, p, refine=refine)
    k = f"icos_{tag}_"
    ref_xyz = refpath[k + "xyz"]
    for d in range(3):
        assert np.array_equal(g.xyz[d].view(np.uint64), ref_xyz[d].view(np.uint64))
    N = g.ndof()
    ng = g.node_geom.reshape(7, N)
    assert rel(ng[:6], refpath[k + "metric"]) < 1e-12
    assert rel(ng[6], refpath[k + "jac"]) < 1e-12
    w2 = np.einsum("j,i->ji", g.W, g.W).ravel()
    mass = np.tile(w2, g.nelems) * ng[6]
    assert rel(mass, refpath[k + "mass"]) < 1e-12


@pytest.mark.parametrize("tag", list(CASES))
@pytest.mark.parametrize("op", range(4))
def test_icos_classes_fold_like_reference(refpath, tag, op):
    level, p, refine = CASES[tag]
    g = IcosGrid(level, p, refine=refine)
    k = f"icos_{tag}_"
    u = refpath[k + "u"].copy()
    O.load().gfo_ggfx_doop(O.dp(u), O.c_size_t(g.nclass), O.ip(g.class_ptr), O.ip(g.members), op)
    assert np.array_equal(u.view(np.uint64), refpath[k + f"dss{op}"].view(np.uint64))


def test_icos_sizes_and_surface():
    for level in range(0, 4):
        ne = [0]
        g = IcosGrid(level, 3, radius=6.371)
        assert g.nelems == 3 * 20 * 4 ** level
        w2 = np.einsum("j,i->ji", g.W, g.W).ravel()
        area = float(np.sum(np.tile(w2, g.nelems) * g.node_geom.reshape(7, -1)[6]))
        assert abs(area / (4 * np.pi * 6.371 ** 2) - 1.0) < 1e-4 / (1 + 10 * level)
        r = np.sqrt(sum(a * a for a in g.xyz))
        assert np.max(np.abs(r - 6.371)) < 1e-12
