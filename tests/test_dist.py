"""Element-partitioned gather-scatter (geoflow_b200.dist) on 2 and 3 ranks.

CPU: gloo process groups on 127.0.0.1; the rank-local fold is the oracle's
GGFX fold on each rank's classes (the device gf_dss on a GPU), so these
tests check the partition, the exchange plan and the shared-point fold.
Acceptance: bit-identical to the single-process gather-scatter of the
whole grid for Sum, Smooth, Max and Min; the all-reduced multiplicity
weighted dot equals the single-process one to rounding.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from geoflow_b200 import dist as D

CASES = [(2, [5, 3], 3, [1, 0]), (2, [4, 4], 4, [1, 1]), (3, [3, 2, 3], 2, [0, 1, 1]),
         (3, [2, 3, 2], 3, [1, 1, 1]), (3, [1, 2, 3], 2, [0, 0, 0]), (2, [1, 6], 3, [1, 0])]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_fold(shard):
    def fold(u, op):
        a = u.numpy()
        O.load().gfo_ggfx_doop(O.dp(a), O.c_size_t(len(shard.class_ptr) - 1), O.ip(shard.class_ptr),
                               O.ip(shard.members), op)
    return fold


def _worker(rank, world, port, case, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dim, ne, p, per = case
        sh = D.BoxShard(dim, ne, p, per, world, rank)
        box = O.OracleBox(dim, ne, p, periodic=per)
        rng = np.random.default_rng(7)
        ug = rng.standard_normal(box.N) * 10.0 ** rng.integers(-3, 4, box.N)
        sl = slice(sh.e0 * sh.nn, sh.e1 * sh.nn)
        res = {}
        for op in (D.SUM, D.SMOOTH, D.MAX, D.MIN):
            u = torch.from_numpy(ug[sl].copy())
            sh.dss(u, op, _oracle_fold(sh))
            ref = box.dss(ug.copy(), op)[sl]
            res[op] = bool(np.array_equal(u.numpy(), ref))
        a = torch.from_numpy(ug[sl].copy())
        b = torch.from_numpy(np.cos(ug[sl]))
        res["dot"] = sh.dot(a, b)
        res["mult"] = bool(np.array_equal(sh.multiplicity(), box.mult()[sl]))
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", CASES)
def test_partitioned_dss_matches_single_process(case, world):
    dim, ne, p, per = case
    if int(np.prod(ne)) < world:
        pytest.skip("fewer elements than ranks")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    out = dict(q.get(timeout=120) for _ in range(world))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    box = O.OracleBox(dim, ne, p, periodic=per)
    rng = np.random.default_rng(7)
    ug = rng.standard_normal(box.N) * 10.0 ** rng.integers(-3, 4, box.N)
    ref_dot = float(np.sum(ug * np.cos(ug) / box.mult()))
    for r in range(world):
        for op in (D.SUM, D.SMOOTH, D.MAX, D.MIN):
            assert out[r][op], (r, op)
        assert out[r]["mult"]
        assert abs(out[r]["dot"] - ref_dot) <= 1e-12 * abs(ref_dot) + 1e-12


def test_partition_matches_find_rank_subdomain():
    """nper = ne // nranks elements per rank, the last rank the rest."""
    assert [D.rank_range(10, 3, r) for r in range(3)] == [(0, 3), (3, 6), (6, 10)]
    assert [D.rank_range(8, 4, r) for r in range(4)] == [(0, 2), (2, 4), (4, 6), (6, 8)]


@pytest.mark.gpu
def test_shard_problem_uses_the_device_fold(ctx):
    """One rank's problem built from ShardGrid, folded by gf_dss on the GPU,
    with the exchange path run over a 1-rank process group: equals the
    whole-grid gather-scatter for every operation."""
    from geoflow_b200 import GGFX, Problem
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        sh = D.BoxShard(3, [3, 2, 2], 4, [1, 0, 1], 1, 0)
        prob = Problem(ctx, D.ShardGrid(sh), structured=False)
        box = O.OracleBox(3, [3, 2, 2], 4, periodic=[1, 0, 1])
        ug = np.random.default_rng(3).standard_normal(box.N)
        for op in (D.SUM, D.SMOOTH, D.MAX, D.MIN):
            u = torch.from_numpy(ug.copy()).to("cuda")
            sh.dss(u, op, lambda t, o: GGFX(prob).doOp(t, o))
            assert np.array_equal(u.cpu().numpy(), box.dss(ug.copy(), op))
        assert np.array_equal(prob.grid.mask, box.mask)
    finally:
        dist.destroy_process_group()
