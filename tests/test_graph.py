"""CUDA graphs of RK steps and ensembles of them (no reference counterpart):
a replayed graph must give the same bits as the direct calls it recorded."""
import numpy as np
import pytest
import torch

from geoflow_b200 import GBurgers, Graph, GridBox, Problem, _abi as A

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def continuous(g, a):
    return a[g.members[g.class_ptr[:-1]]][g.node_class]


def member(ctx, dim, ne, p, eqn, scheme, seed, dtype=torch.float64):
    g = GridBox(dim, ne, p, periodic=[1] * dim)
    prob = Problem(ctx, g, dirichlet_mask=False)
    rng = np.random.default_rng(seed)
    B = GBurgers(prob, eqn, 0.01, scheme=scheme)
    u = [dev(continuous(g, 0.3 * rng.standard_normal(g.ndof())), dtype) for _ in range(B.nstate)]
    c = ([dev(continuous(g, rng.standard_normal(g.ndof())), dtype) for _ in range(dim)]
         if eqn == A.GF_EQN_ADVECT else None)
    return g, prob, B, u, c


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_graph_replay_matches_direct(ctx, dtype):
    """Config-1 shape: 2-d periodic advection, 16^2 elements p = 4, RK4."""
    g, prob, B, u, c = member(ctx, 2, [16, 16], 4, A.GF_EQN_ADVECT, A.GF_RK4, 1, dtype)
    ud = [a.clone() for a in u]
    B.step(ud, c, dt=1e-4, nsteps=10)
    G = B.capture(u, c, dt=1e-4, nsteps=5)
    assert G.nodes() > 0
    G.launch()
    G.launch()
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(u, ud))
    G.close()


def test_graph_ensemble_matches_members(ctx):
    specs = [(2, [8, 8], 3, A.GF_EQN_ADVECT, A.GF_RK4), (2, [5, 7], 6, A.GF_EQN_HEAT, A.GF_SSP33),
             (3, [2, 3, 2], 4, A.GF_EQN_BURGERS, A.GF_SSP34), (2, [12, 10], 8, A.GF_EQN_BURGERS,
                                                               A.GF_RK2)]
    members, direct = [], []
    for i, (dim, ne, p, eqn, scheme) in enumerate(specs):
        g, prob, B, u, c = member(ctx, dim, ne, p, eqn, scheme, 10 + i)
        ud = [a.clone() for a in u]
        B.step(ud, c, dt=2e-4, nsteps=6)
        direct.append(ud)
        members.append((B, u, c, prob))
    graphs = [B.capture(u, c, dt=2e-4, nsteps=3) for B, u, c, _ in members]
    E = Graph.ensemble(graphs)
    assert E.nodes() == sum(gr.nodes() for gr in graphs)
    E.launch()
    E.launch()
    torch.cuda.synchronize()
    for (B, u, c, _), ud in zip(members, direct):
        assert all(torch.equal(a, b) for a, b in zip(u, ud))
    E.close()
    for gr in graphs:
        gr.close()
