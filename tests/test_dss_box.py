"""Box-lattice gather-scatter (k_dss_box, k_dss_rk_box_n: members computed from
the lattice point's coordinates) against the CSR kernels (k_dss_csr,
k_dss_rk_csr: members read from class_ptr/members) on the same grid built
without its box description (Problem(structured=False)).  Both fold the
members of a class in ascending local id (GGFX::doOp, comm/ggfx.hpp:346-443),
so they agree bit for bit: every op and dtype, with -0.0, NaN and Inf in the
input, and through the RK stages that fuse the Smooth with the stage
updates (GExRKStepper, sem/gexrk_stepper.ipp).  The CSR kernel is itself
bit-exact against the oracle (test_gpu_parity.py::test_dss_bit_exact).
"""
import numpy as np
import pytest

from geoflow_b200 import _abi as A

pytestmark = pytest.mark.gpu

SHAPES = [(3, [3, 2, 4], 4, [1, 0, 1]), (3, [2, 2, 2], 7, None), (2, [5, 3], 6, [0, 1]),
          (3, [4, 3, 2], 1, [1, 1, 0]), (3, [2, 3, 2], 5, [1, 1, 1]),
          (2, [1, 4], 3, [1, 0]),  # a single-element periodic direction (CSR both)
          # lattice rows longer than a block (281 and 601 points), and p = 11
          (3, [40, 2, 2], 7, [0, 1, 0]), (2, [300, 2], 2, None), (3, [2, 2, 3], 11, [1, 0, 1])]


def pair(ctx, dim, ne, p, per):
    from geoflow_b200 import GridBox, Problem
    g = GridBox(dim, ne, p, periodic=per)
    return g, Problem(ctx, g, structured=True), Problem(ctx, g, structured=False)


def bits_equal(a, b):
    import torch
    if a.dtype == torch.float64:
        return torch.equal(a.view(torch.int64), b.view(torch.int64))
    return torch.equal(a.view(torch.int32), b.view(torch.int32))


@pytest.mark.parametrize("dim,ne,p,per", SHAPES)
def test_dss_box_equals_csr(ctx, dim, ne, p, per):
    import torch
    from geoflow_b200 import GGFX
    g, pb, pc = pair(ctx, dim, ne, p, per)
    rng = np.random.default_rng(p + 10 * dim)
    u = rng.standard_normal(g.ndof()) * 10.0 ** rng.integers(-3, 4, g.ndof())
    u[::97] = -0.0
    u[5] = np.nan
    u[13] = np.inf
    u[21] = -np.inf
    for dt in (torch.float64, torch.float32):
        for op in (GGFX.Sum, GGFX.Smooth, GGFX.Max, GGFX.Min):
            ub = torch.from_numpy(u).to(device="cuda", dtype=dt)
            uc = ub.clone()
            GGFX(pb).doOp(ub, op)
            GGFX(pc).doOp(uc, op)
            assert bits_equal(ub, uc), (dt, op)


@pytest.mark.parametrize("scheme", [A.GF_RK1, A.GF_RK2, A.GF_RK3, A.GF_RK4, A.GF_SSP22,
                                    A.GF_SSP33, A.GF_SSP34])
@pytest.mark.parametrize("dim,ne,p,per", [SHAPES[0], SHAPES[2], SHAPES[4]])
def test_rk_stages_box_equal_csr(ctx, scheme, dim, ne, p, per):
    import torch
    from geoflow_b200 import GBurgers
    g, pb, pc = pair(ctx, dim, ne, p, per)
    rng = np.random.default_rng(scheme)
    u0 = [0.3 * rng.standard_normal(g.ndof()) for _ in range(dim)]
    for dt in (torch.float64, torch.float32):
        ub = [torch.from_numpy(a).to(device="cuda", dtype=dt) for a in u0]
        uc = [a.clone() for a in ub]
        GBurgers(pb, GBurgers.BURGERS, 1e-2, scheme=scheme).step(ub, None, dt=1e-3, nsteps=3)
        GBurgers(pc, GBurgers.BURGERS, 1e-2, scheme=scheme).step(uc, None, dt=1e-3, nsteps=3)
        for a, b in zip(ub, uc):
            assert bits_equal(a, b), (dt, scheme)


@pytest.mark.parametrize("scheme", [A.GF_RK4, A.GF_SSP33, A.GF_SSP34])
def test_rk_stages_box_equal_csr_one_component(ctx, scheme):
    import torch
    from geoflow_b200 import GBurgers
    g, pb, pc = pair(ctx, *SHAPES[0])
    u0 = np.random.default_rng(scheme + 7).standard_normal(g.ndof())
    for dt in (torch.float64, torch.float32):
        ub = [torch.from_numpy(u0).to(device="cuda", dtype=dt)]
        uc = [ub[0].clone()]
        GBurgers(pb, GBurgers.HEAT, 5e-2, scheme=scheme).step(ub, None, dt=1e-3, nsteps=3)
        GBurgers(pc, GBurgers.HEAT, 5e-2, scheme=scheme).step(uc, None, dt=1e-3, nsteps=3)
        assert bits_equal(ub[0], uc[0]), (dt, scheme)
