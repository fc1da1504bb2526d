"""Element-partitioned gather-scatter over ranks (one process per GPU).

Partition: GGridBox::find_rank_subdomain (grid/ggrid_box.ipp:855-980):
rank r owns the contiguous global elements [r*nper, r*nper + nthis) in
lexicographic order, nper = ne // nranks, the last rank the remainder.

Interface exchange: a unique node (a GLL lattice point of the box) whose
element copies live on several ranks is "shared".  GGFX folds a class in
ascending local id; with a contiguous partition, global local ids order
the copies across ranks.  To stay bit-identical to the single-GPU
gather-scatter, ranks exchange the copies' *values* (not partial sums):
each rank sends the values of its copies of every node it shares with a
peer and folds each shared node over all copies in global order, with the
reduction functors of comm/ggfx.hpp:36-76 (Sum and Smooth from 0, Max and
Min from the extreme values).  Interior nodes are folded by the local
gather-scatter (libgfgpu's gf_dss on the rank's GPU); the shared nodes are
then overwritten with the exchanged fold.

The exchange uses torch.distributed point-to-point calls, so the same code
runs over NCCL (CUDA tensors) or gloo (CPU tensors).  Sizes and indices are
computed on the host from the box description alone; no rank needs the
global arrays.
"""
from __future__ import annotations

import numpy as np

SUM, SMOOTH, MAX, MIN = 0, 1, 2, 3


def rank_range(nglobal: int, nranks: int, rank: int):
    """[first, last) global elements of `rank` (find_rank_subdomain)."""
    nper = nglobal // nranks
    n = nper if rank != nranks - 1 else nglobal - (nranks - 1) * nper
    return nper * rank, nper * rank + n


class BoxShard:
    """One rank's part of a GGridBox of ne elements per direction, order p:
    its elements, the lattice point of every local node, the rank-local
    gather-scatter classes and the exchange plan for the shared points."""

    def __init__(self, dim, ne, p, periodic, nranks, rank):
        self.dim, self.p, self.n = dim, p, p + 1
        self.ne = [int(v) for v in ne][:dim]
        self.per = [int(bool(v)) for v in periodic][:dim]
        self.nranks, self.rank = nranks, rank
        self.nn = self.n ** dim
        self.nglobal = int(np.prod(self.ne))
        self.nper = self.nglobal // nranks
        self.e0, self.e1 = rank_range(self.nglobal, nranks, rank)
        self.M = [self.ne[d] * p + (0 if self.per[d] else 1) for d in range(dim)]
        self.nlocal = (self.e1 - self.e0) * self.nn
        # lattice id of every local node
        e = np.repeat(np.arange(self.e0, self.e1, dtype=np.int64), self.nn)
        a = np.tile(np.arange(self.nn, dtype=np.int64), self.e1 - self.e0)
        self.lid = self._lattice(e, a)
        # rank-local classes (ascending local id inside a class)
        order = np.argsort(self.lid, kind="stable")
        uids, starts = np.unique(self.lid[order], return_index=True)
        self.class_ptr = np.append(starts, self.nlocal).astype(np.int32)
        self.members = order.astype(np.int32)
        self.node_class = np.empty(self.nlocal, dtype=np.int32)
        self.node_class[order] = np.repeat(np.arange(len(uids), dtype=np.int32),
                                           np.diff(self.class_ptr))
        self._plan(uids)

    # ---- lattice helpers ----
    def _coords(self, e):
        c0 = e % self.ne[0]
        r = e // self.ne[0]
        c1 = r % self.ne[1]
        c2 = r // self.ne[1] if self.dim > 2 else np.zeros_like(e)
        return c0, c1, c2

    def _lattice(self, e, a):
        n, p = self.n, self.p
        loc = [a % n, (a // n) % n, a // (n * n)]
        ec = self._coords(e)
        lid = np.zeros_like(e)
        stride = 1
        for d in range(self.dim):
            g = ec[d] * p + loc[d]
            if self.per[d]:
                g = np.where(g == self.ne[d] * p, 0, g)
            lid = lid + g * stride
            stride *= self.M[d]
        return lid

    def _cands(self, g, d):
        """Up to two (element coordinate, local index) pairs per lattice
        coordinate, in ascending element coordinate; valid flags."""
        p, ne = self.p, self.ne[d]
        r, q = g % p, g // p
        ec = np.stack([q, np.zeros_like(q)], 1)
        li = np.stack([r, np.zeros_like(r)], 1)
        ok = np.stack([np.ones_like(q, bool), np.zeros_like(q, bool)], 1)
        face = r == 0
        if self.per[d]:
            wrap = face & (q == 0)
            inner = face & (q > 0)
            ec[wrap] = [0, ne - 1]
            li[wrap] = [0, p]
            ok[wrap] = [True, True]
            ec[inner, 0], ec[inner, 1] = q[inner] - 1, q[inner]
            li[inner] = [p, 0]
            ok[inner] = [True, True]
        else:
            lo = face & (q >= 1)
            hi = face & (q < ne)
            both = lo & hi
            ec[both, 0], ec[both, 1] = q[both] - 1, q[both]
            li[both] = [p, 0]
            ok[both] = [True, True]
            only_lo = lo & ~hi
            ec[only_lo, 0], li[only_lo, 0] = q[only_lo] - 1, p
        return ec, li, ok

    def rank_of(self, e):
        return np.minimum(e // self.nper, self.nranks - 1) if self.nper > 0 else \
            np.full_like(e, self.nranks - 1)

    # ---- exchange plan ----
    def _plan(self, uids):
        import itertools
        dim, n, nn, me = self.dim, self.n, self.nn, self.rank
        g, rem = [], uids.copy()
        for d in range(dim):
            g.append(rem % self.M[d])
            rem = rem // self.M[d]
        cand = [self._cands(g[d], d) for d in range(dim)]
        combos = 2 ** dim
        estr = [1, self.ne[0], self.ne[0] * (self.ne[1] if dim > 1 else 1)]
        mem_e = np.zeros((len(uids), combos), np.int64)
        mem_a = np.zeros((len(uids), combos), np.int64)
        valid = np.ones((len(uids), combos), bool)
        for col, bits in enumerate(itertools.product([0, 1], repeat=dim)):
            for d, b in enumerate(bits):
                ec, li, ok = cand[d]
                mem_e[:, col] += ec[:, b] * estr[d]
                mem_a[:, col] += li[:, b] * n ** d
                valid[:, col] &= ok[:, b]
        gidx = np.where(valid, mem_e * nn + mem_a, np.iinfo(np.int64).max)
        order = np.argsort(gidx, axis=1, kind="stable")
        gidx = np.take_along_axis(gidx, order, 1)
        mem_e = np.take_along_axis(mem_e, order, 1)
        valid = np.take_along_axis(valid, order, 1)
        ranks = np.where(valid, self.rank_of(mem_e), -1)
        shared = ((ranks != me) & valid).any(1)
        self.sh_uids = uids[shared]
        gidx, ranks, valid = gidx[shared], ranks[shared], valid[shared]
        self.mult = valid.sum(1)  # global copies of each shared point
        own = (ranks == me)
        rows, cols = np.nonzero(own)  # row-major: ascending point, ascending copy
        self.own_local = (gidx[rows, cols] - self.e0 * nn).astype(np.int64)
        self.own_row = rows.astype(np.int64)
        pos = np.full(gidx.shape, -1, np.int64)
        pos[rows, cols] = np.arange(len(rows))
        self.peers = sorted(int(s) for s in np.unique(ranks[valid & ~own]))
        self.send_idx, self.recv_cnt = {}, {}
        off = len(rows)
        for s in self.peers:
            with_s = (ranks == s).any(1)
            r_own = own & with_s[:, None]
            rr, cc = np.nonzero(r_own)
            self.send_idx[s] = (gidx[rr, cc] - self.e0 * nn).astype(np.int64)
            rs, cs = np.nonzero(ranks == s)
            self.recv_cnt[s] = len(rs)
            pos[rs, cs] = off + np.arange(len(rs))
            off += len(rs)
        self.pool_size = off
        self.gather = np.where(valid, pos, off)  # the extra slot pads invalid copies
        self.valid = valid

    # ---- multiplicity of every local node (global copies) ----
    def multiplicity(self):
        m = np.diff(self.class_ptr)[self.node_class].astype(np.float64)
        m[self.own_local] = self.mult[self.own_row]
        return m

    # ---- device-resident plan (indices uploaded once per device) ----
    def device_plan(self, device):
        """int32 index tensors of the exchange on `device`: own copies, the
        copies sent to each peer, the fold table (pool index of every copy
        of every shared point, -1 where a point has fewer copies) and the
        output map (own copy -> point)."""
        import torch
        key = str(device)
        plans = self.__dict__.setdefault("_plans", {})
        if key not in plans:
            i32 = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int32), device=device)
            table = np.where(self.valid, self.gather, -1)
            plans[key] = {"own": i32(self.own_local), "row": i32(self.own_row),
                          "send": {s: i32(self.send_idx[s]) for s in self.peers},
                          "table": i32(table), "maxc": int(table.shape[1]) if table.size else 1}
        return plans[key]

    def dss(self, u, op, local_fold, transport=None, prob=None):
        """GGFX::doOp over all ranks, in place on this rank's element-local
        torch tensor u.  local_fold(u, op) folds the rank-local classes (the
        library's gf_dss on the rank's GPU); the shared points are then
        overwritten with the fold over every copy, in global order.  With
        `prob` (the rank's Problem) and a CUDA u the packing and the fold
        run as library kernels (gf_gather, gf_dss_fold_copies) on indices
        kept on the device; otherwise as torch operations.  `transport`
        moves the send buffers (default: torch.distributed point-to-point)."""
        transport = transport or TorchTransport()
        if prob is not None and u.is_cuda:
            return self._dss_device(u, op, local_fold, transport, prob)
        import torch
        dev = u.device
        t = lambda a: torch.as_tensor(a, device=dev)
        own = u[t(self.own_local)]
        sends = {s: u[t(self.send_idx[s])].contiguous() for s in self.peers}
        local_fold(u, op)
        recvs = transport.exchange(self, sends, u.dtype, dev)
        pad = torch.zeros(1, dtype=u.dtype, device=dev)
        pool = torch.cat([own] + [recvs[s] for s in self.peers] + [pad])
        V = pool[t(self.gather)]
        ok = t(self.valid)
        big = torch.finfo(u.dtype).max
        if op in (SUM, SMOOTH):
            acc = torch.zeros(V.shape[0], dtype=u.dtype, device=dev)
            for j in range(V.shape[1]):
                acc = torch.where(ok[:, j], acc + V[:, j], acc)
            if op == SMOOTH:
                acc = acc / t(self.mult).to(u.dtype)
        elif op == MAX:
            acc = torch.full((V.shape[0],), -big, dtype=u.dtype, device=dev)
            for j in range(V.shape[1]):
                acc = torch.where(ok[:, j] & (acc < V[:, j]), V[:, j], acc)
        else:
            acc = torch.full((V.shape[0],), big, dtype=u.dtype, device=dev)
            for j in range(V.shape[1]):
                acc = torch.where(ok[:, j] & (V[:, j] < acc), V[:, j], acc)
        u[t(self.own_local)] = acc[t(self.own_row)]
        return u

    def _dss_device(self, u, op, local_fold, transport, prob):
        import torch
        from . import _abi as A
        lib = A.load()
        P = self.device_plan(u.device)
        code = A.GF_F64 if u.dtype == torch.float64 else A.GF_F32
        nown = len(self.own_local)
        npool = self.pool_size
        pool = torch.empty(npool + 1, dtype=u.dtype, device=u.device)
        chk = lambda rc, what: prob.ctx.check(rc, what)
        if nown:
            chk(lib.gf_gather(prob.handle, code, nown, A.ptr(P["own"]), A.ptr(u), A.ptr(pool)),
                "gf_gather")
        sends = {}
        for s in self.peers:
            idx = P["send"][s]
            buf = torch.empty(len(self.send_idx[s]), dtype=u.dtype, device=u.device)
            if len(buf):
                chk(lib.gf_gather(prob.handle, code, len(buf), A.ptr(idx), A.ptr(u), A.ptr(buf)),
                    "gf_gather")
            sends[s] = buf
        local_fold(u, op)
        recvs = transport.exchange(self, sends, u.dtype, u.device)
        off = nown
        for s in self.peers:
            n = self.recv_cnt[s]
            if n:
                pool[off:off + n].copy_(recvs[s])
            off += n
        if nown:
            chk(lib.gf_dss_fold_copies(prob.handle, code, int(op), P["maxc"], A.ptr(P["table"]),
                                       A.ptr(pool), nown, A.ptr(P["own"]), A.ptr(P["row"]),
                                       A.ptr(u)), "gf_dss_fold_copies")
        return u

    def dot(self, a, b, transport=None):
        """Multiplicity-weighted inner product over all ranks (the weights
        of GCG's gdot, gtvector.ipp:1136-1153): sum a b / mult, all-reduced."""
        import torch
        key = ("imult", str(a.device), a.dtype)
        cache = self.__dict__.setdefault("_cache", {})
        if key not in cache:
            cache[key] = torch.as_tensor(1.0 / self.multiplicity(), dtype=a.dtype, device=a.device)
        s = float(torch.sum(a * b * cache[key]).item())
        return (transport or TorchTransport()).allreduce(s, "sum")


class ShardGrid:
    """The grid description of one rank's elements of a uniform box (the
    attributes geoflow_b200.Problem reads from a GridBox): GLL basis,
    per-element affine geometry, Dirichlet mask on the non-periodic box
    faces, and the rank-local classes of the BoxShard."""

    def __init__(self, shard: BoxShard, length=None):
        from .sem import gll_basis
        dim = shard.dim
        self.dim, self.p, self.n = dim, shard.p, shard.n
        self.ne = list(shard.ne)
        self.periodic = list(shard.per)
        self.nelems = shard.e1 - shard.e0
        self.nn = shard.nn
        self.xi, self.W, self.D = gll_basis(shard.p)
        L = np.array(length if length is not None else [1.0] * dim, dtype=np.float64)
        h = L / np.array(self.ne, dtype=np.float64)
        # per-element lengths as gf_box_grid forms them, (lo + h) - lo with
        # lo = x0 + i h, so the geometry carries the same bits as the
        # single-GPU grid's
        e = np.arange(shard.e0, shard.e1, dtype=np.int64)
        Le = []
        for d in range(dim):
            lo = 0.0 + (e % self.ne[d]).astype(np.float64) * h[d]
            Le.append((lo + h[d]) - lo)
            e = e // self.ne[d]
        geo = np.empty((self.nelems, dim + 1))
        for d in range(dim):
            geo[:, d] = 2.0 / Le[d]
        geo[:, dim] = 0.25 * Le[0] * Le[1] if dim == 2 else 0.125 * Le[0] * Le[1] * Le[2]
        self.elem_geom = geo.ravel()
        # Dirichlet mask: lattice points on a non-periodic box face
        lid = shard.lid.copy()
        self.mask = np.ones(shard.nlocal)
        for d in range(dim):
            g = lid % shard.M[d]
            lid //= shard.M[d]
            if not shard.per[d]:
                self.mask[(g == 0) | (g == shard.M[d] - 1)] = 0.0
        self.class_ptr, self.members = shard.class_ptr, shard.members
        self.node_class = shard.node_class
        self.nclass = len(shard.class_ptr) - 1

    def ndof(self) -> int:
        return self.nelems * self.nn


# ---------------------------------------------------------------------------
# transports
class TorchTransport:
    """The exchange and the scalar all-reduce over torch.distributed:
    NCCL with CUDA tensors, gloo with CPU tensors (CUDA buffers stage
    through host memory under gloo)."""

    def exchange(self, shard, sends, dtype, device):
        import torch
        import torch.distributed as dist
        stage = device.type == "cuda" and dist.get_backend() == "gloo"
        bdev = "cpu" if stage else device
        recvs = {s: torch.empty(shard.recv_cnt[s], dtype=dtype, device=bdev) for s in shard.peers}
        sb = {s: (b.cpu() if stage else b) for s, b in sends.items()}
        reqs = [dist.irecv(recvs[s], src=s) for s in shard.peers if shard.recv_cnt[s]]
        reqs += [dist.isend(sb[s], dst=s) for s in shard.peers if len(sb[s])]
        for r in reqs:
            r.wait()
        return {s: r.to(device) for s, r in recvs.items()} if stage else recvs

    def allreduce(self, v, op):
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX)
        return float(t.item())


# ---------------------------------------------------------------------------
# rank-local operations: the oracle on the CPU (tests) or the library on
# the rank's GPU
def _butcher(order):
    """GButcherRK::computeCoeffs (pdes/gbutcherrk.ipp:69-125) as the
    stepper uses it: alpha, beta[m][j], c."""
    beta = [[0.0] * 4 for _ in range(4)]
    if order == 1:
        c = [1.0, 0, 0, 0]
    elif order == 2:
        c = [0.5, 0.5, 0, 0]
        beta[1][0] = 1.0
    elif order == 3:
        c = [0.25, 0.0, 0.75, 0]
        beta[1][0] = 1.0 / 3.0
        beta[2][1] = 2.0 / 3.0
    else:
        c = [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]
        beta[1][0] = 0.5
        beta[2][1] = 0.5
        beta[3][2] = 1.0
    return beta, c


class OracleOps:
    """The oracle's element-local operators on one rank's elements (slices
    of a whole-grid OracleBox) and IEEE double stage arithmetic in numpy,
    for the multi-process tests on the CPU (test infrastructure)."""

    def __init__(self, shard, box):
        import ctypes as C
        import oracle as O
        self.O, self.shard, self.box = O, shard, box
        e0, e1, nn = shard.e0, shard.e1, shard.nn
        sl = slice(e0 * nn, e1 * nn)
        self.sl = sl
        g = O.GfoGrid()
        g.dim, g.Ne = box.dim, e1 - e0
        self._keep = [np.ascontiguousarray(a[sl]) for a in box.dXidX]
        self._jac = np.ascontiguousarray(box.Jac[sl])
        self._mass = np.ascontiguousarray(box.mass[sl])
        self.imass = np.ascontiguousarray(box.imass[sl])
        for d in range(3):
            g.n[d] = box.n
            g.D[d] = O.dp(box.D)
            g.W[d] = O.dp(box.W)
            g.dXidX[d] = O.dp(self._keep[d])
        g.Jac = O.dp(self._jac)
        g.mass = O.dp(self._mass)
        self.g = g
        self.C = C
        self.prob = None
        self.mask = np.ascontiguousarray(box.mask[sl])

    def new(self, like):
        import torch
        return torch.zeros_like(like)

    def fold(self, u, op):
        a = u.numpy()
        O = self.O
        O.load().gfo_ggfx_doop(O.dp(a), O.c_size_t(len(self.shard.class_ptr) - 1),
                               O.ip(self.shard.class_ptr), O.ip(self.shard.members), op)

    def rhs(self, eqn, nu, u, c, K):
        O, C = self.O, self.C
        nst = len(u)
        arrs = [t.numpy() for t in u]
        ua = (O.P_double * 3)(*[O.dp(a) for a in arrs] + [None] * (3 - nst))
        ca = (O.P_double * 3)(*([O.dp(t.numpy()) for t in c] if c else []) +
                              [None] * (3 - (len(c) if c else 0)))
        outs = [t.numpy() for t in K]
        oa = (O.P_double * 3)(*[O.dp(a) for a in outs] + [None] * (3 - nst))
        O.load().gfo_dudt(C.byref(self.g), eqn, C.c_double(nu), O.dp(self.imass), nst, ua, ca, oa)

    def helm(self, p, q, u, out):
        O, C = self.O, self.C
        qv = np.full(len(self.imass), q)
        O.load().gfo_helmholtz(C.byref(self.g), O.dp(u.numpy()), C.c_double(p), None, O.dp(qv),
                               O.dp(out.numpy()))

    @staticmethod
    def stage_sum(uin, Ks, bs, y):
        s = np.zeros_like(uin.numpy())
        for K, b in zip(Ks, bs):
            s = 1.0 * s + b * K.numpy()
        v = uin.numpy().copy()
        v += s
        y.numpy()[:] = v

    @staticmethod
    def update(x, dt, uin, a, y, b, a2, y2, b2):
        v = dt * x.numpy() + 1.0 * uin.numpy()
        if y is not None:
            v = a * v + b * y.numpy()
        if y2 is not None:
            v = a2 * v + b2 * y2.numpy()
        x.numpy()[:] = v

    @staticmethod
    def accum(uout, K, ch):
        uout.numpy()[:] = uout.numpy() + K.numpy() * ch

    def coef(self, v, dtype):
        return float(v)


class DeviceOps:
    """The library's element-local kernels on the rank's GPU: the rank's
    Problem (built from ShardGrid, inverse mass replaced by the assembled
    one), gf_dudt, gf_helmholtz_apply, gf_dss for the local fold and the
    stage arithmetic entry points."""

    def __init__(self, shard, ctx, transport=None, length=None, dirichlet_mask=True):
        import torch
        from . import _abi as A
        from .sem import Problem
        self.A, self.shard, self.ctx = A, shard, ctx
        self.grid = ShardGrid(shard, length=length)
        self.prob = Problem(ctx, self.grid, dirichlet_mask=dirichlet_mask, structured=False)
        self.mask = torch.as_tensor(self.grid.mask, device=ctx.torch_device)
        # assembled mass over all ranks -> inverse mass of GMass (1/Smooth(M))
        w = np.einsum("k,j,i->kji", self.grid.W, self.grid.W, self.grid.W).ravel() \
            if self.grid.dim == 3 else np.einsum("j,i->ji", self.grid.W, self.grid.W).ravel()
        eg = self.grid.elem_geom.reshape(self.grid.nelems, self.grid.dim + 1)
        mass = torch.as_tensor((eg[:, self.grid.dim][:, None] * w[None, :]).ravel(),
                               device=ctx.torch_device)
        mult = torch.as_tensor(shard.multiplicity(), device=ctx.torch_device)
        sm = mass.clone()
        shard.dss(sm, SUM, self.fold, transport, self.prob)
        imass = (1.0 / (sm / mult)).cpu().numpy()
        ctx.check(A.load().gf_problem_set_imass(self.prob.handle, A.ptr(imass)), "set_imass")

    def new(self, like):
        import torch
        return torch.zeros_like(like)

    def _code(self, t):
        import torch
        return self.A.GF_F64 if t.dtype == torch.float64 else self.A.GF_F32

    def fold(self, u, op):
        A = self.A
        self.ctx.check(A.load().gf_dss(self.prob.handle, self._code(u), int(op), A.ptr(u)), "gf_dss")

    def rhs(self, eqn, nu, u, c, K):
        A = self.A
        self.ctx.check(A.load().gf_dudt(self.prob.handle, self._code(u[0]), eqn, nu, len(u),
                                        A.ptr_array(u), A.ptr_array(c or []), A.ptr_array(K)),
                       "gf_dudt")

    def helm(self, p, q, u, out):
        A = self.A
        self.ctx.check(A.load().gf_helmholtz_apply(self.prob.handle, self._code(u), p, None, q,
                                                   None, 1, A.ptr(u), A.ptr(out)), "helm")

    def stage_sum(self, uin, Ks, bs, y):
        A = self.A
        k = [A.ptr(t) for t in Ks] + [None] * (3 - len(Ks))
        b = list(bs) + [0.0] * (3 - len(bs))
        self.ctx.check(A.load().gf_rk_stage_sum(self.prob.handle, self._code(uin), A.ptr(uin),
                                                len(Ks), k[0], k[1], k[2], b[0], b[1], b[2],
                                                A.ptr(y)), "gf_rk_stage_sum")

    def update(self, x, dt, uin, a, y, b, a2, y2, b2):
        A = self.A
        self.ctx.check(A.load().gf_rk_update(self.prob.handle, self._code(x), A.ptr(x), dt,
                                             A.ptr(uin), a, A.ptr(y) if y is not None else None,
                                             b, a2, A.ptr(y2) if y2 is not None else None, b2),
                       "gf_rk_update")

    def accum(self, uout, K, ch):
        A = self.A
        self.ctx.check(A.load().gf_rk_accum(self.prob.handle, self._code(uout), A.ptr(uout),
                                            A.ptr(K), ch), "gf_rk_accum")

    def coef(self, v, dtype):
        import torch
        return float(np.float32(v)) if dtype == torch.float32 else float(v)


# ---------------------------------------------------------------------------
class DistStepper:
    """GExRKStepper over an element-partitioned box: step_b (RK1-4) and
    step_ssp22/33/34 (pdes/gexrk_stepper.ipp:252-341, 533-819) on every
    rank's elements with each Smooth a partitioned gather-scatter.  The
    operations and their order are those of gf_rk_advance (api_rk.cu) on
    the whole grid, so with the library's kernels the partitioned step is
    bit-identical to the single-GPU one (and with the oracle's, to the
    oracle's).  eqn: 0 advection (c given), 1 Burgers, 2 heat."""

    def __init__(self, shard, ops, eqn, nu, scheme, transport=None):
        self.shard, self.ops, self.eqn, self.nu, self.scheme = shard, ops, eqn, nu, scheme
        self.tr = transport or TorchTransport()

    def smooth(self, v):
        self.shard.dss(v, SMOOTH, self.ops.fold, self.tr, self.ops.prob)

    def _h(self, v, dt, dtype):
        """a coefficient times dt, rounded as the device stepper rounds it"""
        import torch
        if dtype == torch.float32:
            return float(np.float32(np.float32(v) * np.float32(dt)))
        return float(v) * float(dt)

    def step(self, u, c=None, dt=1e-4, nsteps=1):
        for _ in range(nsteps):
            uold = [t.clone() for t in u]
            if self.scheme <= 4:
                self._step_b(uold, u, dt, c)
            else:
                self._step_ssp(uold, u, dt, c)
        return u

    def _step_b(self, uin, uout, dt, c):
        ops, ns = self.ops, self.scheme
        beta, cc = _butcher(ns)
        dtype = uin[0].dtype
        K = [[ops.new(t) for t in uin] for _ in range(max(ns - 1, 1))]
        um = [ops.new(t) for t in uin]
        for k in range(len(uin)):
            uout[k].copy_(uin[k])
        for m in range(ns - 1):
            for k in range(len(uin)):
                ops.stage_sum(uin[k], [K[j][k] for j in range(m)],
                              [self._h(beta[m][j], dt, dtype) for j in range(m)], um[k])
            ops.rhs(self.eqn, self.nu, um, c, K[m])
            ch = self._h(cc[m], dt, dtype)
            for k in range(len(uin)):
                self.smooth(K[m][k])
                ops.accum(uout[k], K[m][k], ch)
        for k in range(len(uin)):
            ops.stage_sum(uin[k], [K[j][k] for j in range(ns - 1)],
                          [self._h(beta[ns - 1][j], dt, dtype) for j in range(ns - 1)], um[k])
            self.smooth(um[k])
        Kf = [ops.new(t) for t in uin]
        ops.rhs(self.eqn, self.nu, um, c, Kf)
        ch = self._h(cc[ns - 1], dt, dtype)
        for k in range(len(uin)):
            self.smooth(Kf[k])
            ops.accum(uout[k], Kf[k], ch)
            self.smooth(uout[k])

    def _substep(self, u, x, dt, uin, a, y, b, a2=1.0, y2=None, b2=0.0):
        ops = self.ops
        dtype = u[0].dtype
        cf = lambda v: ops.coef(v, dtype)
        ops.rhs(self.eqn, self.nu, u, self._c, x)
        for k in range(len(x)):
            ops.update(x[k], cf(dt), uin[k], cf(a), y[k] if y is not None else None, cf(b),
                       cf(a2), y2[k] if y2 is not None else None, cf(b2))
            self.smooth(x[k])

    def _step_ssp(self, uin, uout, dt, c):
        self._c = c
        ops = self.ops
        K = [[ops.new(t) for t in uin] for _ in range(3)]
        s = self.scheme
        if s == 22:
            self._substep(uin, K[0], dt, uin, 1.0, None, 0.0)
            self._substep(K[0], uout, dt, K[0], 0.5, uin, 0.5)
        elif s == 33:
            self._substep(uin, K[0], dt, uin, 1.0, None, 0.0)
            self._substep(K[0], K[1], dt, K[0], 0.25, uin, 0.75)
            self._substep(K[1], uout, dt, K[1], 2.0 / 3.0, uin, 1.0 / 3.0)
        else:
            self._substep(uin, K[0], dt, uin, 0.5, uin, 0.5)
            self._substep(K[0], K[1], dt, K[0], 0.5, K[0], 0.5)
            self._substep(K[1], K[2], dt, K[1], 1.0 / 6.0, K[1], 1.0 / 6.0, 1.0, uin, 2.0 / 3.0)
            self._substep(K[2], uout, dt, K[2], 0.5, K[2], 0.5)


class DistCG:
    """GCG::solve_impl (solvers/gcg.ipp:239-345, the Deville-Fischer-Mund
    form, with a diagonal preconditioner) over an element-partitioned box:
    the operator applies on every rank's elements, the assembly (DSS Sum)
    as a partitioned gather-scatter, the multiplicity-weighted inner
    products of GTVector::gdot (blas/gtvector.ipp:1136-1153) and the norms
    all-reduced.  dinv is the rank's part of the assembled inverse
    diagonal.  Returns (GCGERR code, iterations)."""

    def __init__(self, shard, ops, p=1.0, q=1.0, maxit=512, tol=1e-6, normtype=0,
                 transport=None):
        self.shard, self.ops, self.p, self.q = shard, ops, p, q
        self.maxit, self.tol, self.normtype = maxit, tol, normtype
        self.tr = transport or TorchTransport()
        self.residuals = []

    def _norm(self, x):
        import torch
        if self.normtype == 0:
            return self.tr.allreduce(float(x.abs().max()) if x.numel() else 0.0, "max")
        s = self.tr.allreduce(float(torch.sum(x * x)), "sum")
        n = self.tr.allreduce(float(x.numel()), "sum")
        return float(np.sqrt(s / n))

    def _assemble(self, v):
        self.shard.dss(v, SUM, self.ops.fold, self.tr, self.ops.prob)

    def solve(self, b, x, dinv, xb=None):
        import torch
        ops = self.ops
        mask = torch.as_tensor(ops.mask, dtype=b.dtype, device=b.device)
        dot = lambda a, c: self.shard.dot(a, c, self.tr)
        if xb is not None:
            x.mul_(mask)
            x.add_(xb)
        w = ops.new(b)
        ops.helm(self.p, self.q, x, w)
        r = b - w
        self._assemble(r)
        r.mul_(mask)
        z = dinv * r
        w = z.clone()
        rho = dot(r, z)
        rnorm = self._norm(b)
        rtol = self.tol if rnorm < 1.0 else self.tol * rnorm
        rnorm, it, rc = 10.0 * rtol, 0, 0
        q = ops.new(b)
        self.residuals = []
        while it < self.maxit and rnorm > rtol:
            ops.helm(self.p, self.q, w, q)
            self._assemble(q)
            q.mul_(mask)
            alpha = rho / dot(w, q)
            x.add_(alpha * w)
            r.add_(-alpha * q)
            z = dinv * r
            rhom, rho = rho, dot(r, z)
            w = z + (rho / rhom) * w
            rnorm = self._norm(r)
            self.residuals.append(rnorm)
            it += 1
        x.mul_(mask)
        if it >= self.maxit and rnorm > self.tol:
            rc = 1
        if xb is not None:
            x.add_(xb)
        return rc, it
