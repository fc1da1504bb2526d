"""The partitioned RK stepper and CG (geoflow_b200.dist.DistStepper,
DistCG) on 2 and 3 ranks against the single-process run of the whole grid.

CPU: gloo process groups on 127.0.0.1, rank-local operators from the
oracle (OracleOps).  Acceptance:
  * RK steps (step_b RK2/RK4, SSP22/33/34; advection, Burgers, heat):
    bit-identical to the whole-grid oracle run (every operation is the
    same, only the gather-scatter is split at the exchange);
  * CG: the same GCGERR code, iteration counts within 1, solutions within
    1e-12 relative (both to 1e-13): the inner products sum rank by rank
    and are all-reduced, so they round differently.
GPU (one device): two processes on cuda:0 exchanging through gloo, the
rank-local operators and the shared-point fold as library kernels
(DeviceOps, gf_dss_fold_copies): bit-identical to gf_rk_advance on the
whole grid.  (The two ranks' kernels never wait on each other; the
exchange goes through the host.)
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

RK_CASES = [  # dim, ne, p, eqn, scheme
    (2, [4, 3], 4, 0, 4), (2, [4, 3], 4, 1, 33), (2, [3, 4], 3, 2, 22),
    (3, [3, 2, 2], 3, 1, 4), (3, [2, 2, 3], 3, 0, 33), (3, [3, 2, 2], 3, 1, 34),
    (3, [2, 3, 2], 2, 2, 2)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _state(box, eqn, seed):
    rng = np.random.default_rng(seed)
    cont = lambda: rng.standard_normal(box.nclass)[box.node_class]
    nst = box.dim if eqn == 1 else 1
    u = [0.3 * cont() for _ in range(nst)]
    c = [np.full(box.N, 1.0 - 0.4 * d) for d in range(box.dim)] if eqn == 0 else None
    return u, c


def _rk_worker(rank, world, port, case, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dim, ne, p, eqn, scheme = case
        per = [1] * dim
        sh = D.BoxShard(dim, ne, p, per, world, rank)
        box = O.OracleBox(dim, ne, p, periodic=per)
        u, c = _state(box, eqn, 11)
        sl = slice(sh.e0 * sh.nn, sh.e1 * sh.nn)
        ops = D.OracleOps(sh, box)
        ut = [torch.from_numpy(a[sl].copy()) for a in u]
        ct = [torch.from_numpy(a[sl].copy()) for a in c] if c else None
        D.DistStepper(sh, ops, eqn, 0.02, scheme).step(ut, ct, dt=2e-3, nsteps=3)
        q.put((rank, [t.numpy() for t in ut]))
    finally:
        dist.destroy_process_group()


def _run(world, target, case):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, case, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    out = dict(q.get(timeout=300) for _ in range(world))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    return out


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("dim,ne,p", [(3, [3, 2, 2], 4), (2, [4, 3], 5), (3, [5, 7, 3], 2)])
def test_shard_geometry_bit_identical_to_whole_grid(dim, ne, p, world):
    """Each rank's element geometry carries the single-GPU grid's bits (the
    element lengths are formed per element, as gf_box_grid does)."""
    from geoflow_b200.sem import GridBox
    g = GridBox(dim, ne, p, periodic=[1] * dim)
    for r in range(world):
        sh = D.BoxShard(dim, ne, p, [1] * dim, world, r)
        ref = g.elem_geom.reshape(-1, dim + 1)[sh.e0:sh.e1].ravel()
        assert np.array_equal(D.ShardGrid(sh).elem_geom, ref)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", RK_CASES)
def test_partitioned_rk_bit_identical(case, world):
    dim, ne, p, eqn, scheme = case
    out = _run(world, _rk_worker, case)
    box = O.OracleBox(dim, ne, p, periodic=[1] * dim)
    u, c = _state(box, eqn, 11)
    box.rk_advance(eqn, 0.02, scheme, u, c=c, dt=2e-3, nsteps=3)
    got = [np.concatenate([out[r][k] for r in range(world)]) for k in range(len(u))]
    for a, b in zip(got, u):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


CG_CASES = [(2, [5, 4], 4, O.NORM_INF), (3, [3, 3, 2], 3, O.NORM_EUC)]


def _cg_worker(rank, world, port, case, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dim, ne, p, norm = case
        sh = D.BoxShard(dim, ne, p, [0] * dim, world, rank)
        box = O.OracleBox(dim, ne, p, periodic=[0] * dim)
        rng = np.random.default_rng(5)
        b = box.mass * rng.standard_normal(box.nclass)[box.node_class]
        dinv = 1.0 / box.helmholtz_diag(1.0, np.ones(box.N))
        sl = slice(sh.e0 * sh.nn, sh.e1 * sh.nn)
        ops = D.OracleOps(sh, box)
        x = torch.zeros(sh.nlocal, dtype=torch.float64)
        cg = D.DistCG(sh, ops, p=1.0, q=1.0, maxit=2000, tol=1e-13, normtype=norm)
        rc, it = cg.solve(torch.from_numpy(b[sl].copy()), x, torch.from_numpy(dinv[sl].copy()),
                          xb=torch.zeros(sh.nlocal, dtype=torch.float64))
        q.put((rank, (rc, it, x.numpy())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", CG_CASES)
def test_partitioned_cg_matches_single_process(case, world):
    dim, ne, p, norm = case
    out = _run(world, _cg_worker, case)
    box = O.OracleBox(dim, ne, p, periodic=[0] * dim)
    rng = np.random.default_rng(5)
    b = box.mass * rng.standard_normal(box.nclass)[box.node_class]
    dinv = 1.0 / box.helmholtz_diag(1.0, np.ones(box.N))
    x = np.zeros(box.N)
    rc, it, _ = box.cg_solve(b, x, p=1.0, q_vec=np.ones(box.N), xb=np.zeros(box.N), maxit=2000,
                             normtype=norm, tol=1e-13, dinv=dinv)
    xd = np.concatenate([out[r][2] for r in range(world)])
    for r in range(world):
        assert out[r][0] == rc == 0
        assert abs(out[r][1] - it) <= 1
    assert np.max(np.abs(xd - x)) <= 1e-12 * np.max(np.abs(x))


def _gpu_worker(rank, world, port, case, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from geoflow_b200 import Context
        dim, ne, p, eqn, scheme, dtype = case
        dt_ = torch.float64 if dtype == "f64" else torch.float32
        ctx = Context(0)
        sh = D.BoxShard(dim, ne, p, [1] * dim, world, rank)
        box = O.OracleBox(dim, ne, p, periodic=[1] * dim)
        u, c = _state(box, eqn, 13)
        sl = slice(sh.e0 * sh.nn, sh.e1 * sh.nn)
        ops = D.DeviceOps(sh, ctx, dirichlet_mask=False)
        ut = [torch.from_numpy(a[sl].copy()).to("cuda", dt_) for a in u]
        ct = [torch.from_numpy(a[sl].copy()).to("cuda", dt_) for a in c] if c else None
        D.DistStepper(sh, ops, eqn, 0.02, scheme).step(ut, ct, dt=2e-3, nsteps=3)
        q.put((rank, [t.cpu().numpy() for t in ut]))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("case", [(3, [3, 2, 2], 4, 1, 33, "f64"), (3, [3, 2, 2], 4, 1, 33, "f32"),
                                  (2, [4, 3], 5, 0, 4, "f64"), (3, [2, 3, 2], 3, 2, 4, "f32")])
def test_partitioned_rk_on_gpu_bit_identical_to_single(ctx, case):
    from geoflow_b200 import GBurgers, GridBox, Problem
    dim, ne, p, eqn, scheme, dtype = case
    world = 2
    out = _run(world, _gpu_worker, case)
    dt_ = torch.float64 if dtype == "f64" else torch.float32
    g = GridBox(dim, ne, p, periodic=[1] * dim)
    prob = Problem(ctx, g, dirichlet_mask=False)
    box = O.OracleBox(dim, ne, p, periodic=[1] * dim)
    u, c = _state(box, eqn, 13)
    ut = [torch.from_numpy(a).to("cuda", dt_) for a in u]
    ct = [torch.from_numpy(a).to("cuda", dt_) for a in c] if c else None
    GBurgers(prob, eqn, 0.02, scheme=scheme).step(ut, ct, dt=2e-3, nsteps=3)
    for k in range(len(u)):
        got = np.concatenate([out[r][k] for r in range(world)])
        ref = ut[k].cpu().numpy()
        assert np.array_equal(got, ref), k
