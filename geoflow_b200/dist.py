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

    def dss(self, u, op, local_fold):
        """GGFX::doOp over all ranks, in place on this rank's element-local
        torch tensor u.  local_fold(u, op) folds the rank-local classes (the
        library's gf_dss on the rank's GPU); the shared points are then
        overwritten with the fold over every copy, in global order."""
        import torch
        import torch.distributed as dist
        dev = u.device
        t = lambda a: torch.as_tensor(a, device=dev)
        own = u[t(self.own_local)]
        sends = {s: u[t(self.send_idx[s])].contiguous() for s in self.peers}
        local_fold(u, op)
        recvs = {s: torch.empty(self.recv_cnt[s], dtype=u.dtype, device=dev) for s in self.peers}
        reqs = [dist.irecv(recvs[s], src=s) for s in self.peers if self.recv_cnt[s]]
        reqs += [dist.isend(sends[s], dst=s) for s in self.peers if len(self.send_idx[s])]
        for r in reqs:
            r.wait()
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

    def dot(self, a, b):
        """Multiplicity-weighted inner product over all ranks (the weights
        of GCG's gdot, gtvector.ipp:1136-1153): sum a b / mult, all-reduced."""
        import torch
        import torch.distributed as dist
        w = torch.as_tensor(1.0 / self.multiplicity(), dtype=a.dtype, device=a.device)
        s = torch.sum(a * b * w).reshape(1)
        dist.all_reduce(s)
        return float(s.item())


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
        geo = [2.0 / h[d] for d in range(dim)] + [float(np.prod(h / 2.0))]
        self.elem_geom = np.tile(np.array(geo), self.nelems)
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
