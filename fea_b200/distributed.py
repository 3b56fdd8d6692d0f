"""One reduced system over several ranks: node partition, halo exchange,
and Jacobi-PCG with two scalar all-reduces per iteration.

Partition.  Rank r owns a contiguous range of the plan's nodes, hence a
contiguous range of the reduced rows (the plan numbers DOFs node by node).
With every element incident to an owned node kept on the rank (a one-element
halo), the rank's gather assembly produces its owned rows completely, with
the same columns as the single-device CSR: no exchange is needed to
assemble.  ``ShardedSystem.from_plan_rows`` cuts the single-device CSR the
same way, which is what the tests use.

PCG.  Per iteration one halo exchange of the search direction p (the owned
values each neighbour's rows read, sent once per neighbour pair) before the
row-local SpMV, and two scalar all-reduces (p.q and r.z).  The recurrence is
the library's (fea_pcg_solve): Jacobi preconditioner, stop test
(r.D^-1 r) / (b.D^-1 b) < tol, breakdown on p.q <= 0.

The exchange uses ``torch.distributed`` point-to-point calls (NCCL between
GPUs, gloo between CPU ranks), copying into the local vector: every SpMV
reads only local memory.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def partition_rows(node_dofs, world):
    """Contiguous node ranges with about the same number of reduced rows:
    (row_start [world + 1], node_start [world + 1]); node_dofs [N] = free
    DOFs per node."""
    node_dofs = np.asarray(node_dofs, dtype=np.int64)
    cum = np.concatenate([[0], np.cumsum(node_dofs)])
    n = int(cum[-1])
    nodes = [0]
    for r in range(1, world):
        nodes.append(int(np.searchsorted(cum, r * n / world, side="left")))
    nodes.append(node_dofs.shape[0])
    nodes = np.maximum.accumulate(np.asarray(nodes, dtype=np.int64))
    return cum[nodes], nodes


class ShardedSystem:
    """Rank ``rank``'s rows [row0, row1) of an n x n CSR matrix, its halo
    (the columns outside the range that its rows read) and the exchange
    lists: for each other rank, which of this rank's owned entries it reads
    (``send``) and where the entries read from it land in the halo
    (``recv``)."""

    def __init__(self, rank, world, row_start, indptr_local, cols_global, n, send, recv, halo_cols):
        self.rank, self.world = rank, world
        self.row_start = row_start
        self.row0, self.row1 = int(row_start[rank]), int(row_start[rank + 1])
        self.nloc = self.row1 - self.row0
        self.n = n
        self.indptr = indptr_local
        self.halo_cols = halo_cols
        # local column index: owned columns first, then the halo in halo_cols order
        loc = torch.empty_like(cols_global)
        own = (cols_global >= self.row0) & (cols_global < self.row1)
        loc[own] = cols_global[own] - self.row0
        if halo_cols.numel():
            pos = torch.searchsorted(halo_cols, cols_global[~own])
            loc[~own] = self.nloc + pos
        self.cols = loc
        self.send, self.recv = send, recv

    @classmethod
    def from_plan_rows(cls, rank, world, row_start, indptr, indices):
        """Cut the single-device CSR (indptr, indices over all n rows) into
        rank ``rank``'s shard; every rank computes every rank's halo from the
        shared pattern, so the exchange lists agree without communication."""
        row_start = np.asarray(row_start, dtype=np.int64)
        indptr = torch.as_tensor(indptr, dtype=torch.int64)
        indices = torch.as_tensor(indices, dtype=torch.int64)
        n = int(indptr.shape[0] - 1)
        halos = []
        for r in range(world):
            a, b = int(row_start[r]), int(row_start[r + 1])
            c = indices[int(indptr[a]):int(indptr[b])]
            halos.append(torch.unique(c[(c < a) | (c >= b)]))
        a, b = int(row_start[rank]), int(row_start[rank + 1])
        indptr_local = indptr[a:b + 1] - indptr[a]
        cols = indices[int(indptr[a]):int(indptr[b])].clone()
        send, recv = {}, {}
        for r in range(world):
            if r == rank:
                continue
            h = halos[r]                                        # what rank r reads ...
            mine = h[(h >= a) & (h < b)]                          # ... from me
            if mine.numel():
                send[r] = mine - a
            ra, rb = int(row_start[r]), int(row_start[r + 1])
            hm = halos[rank]
            theirs = (hm >= ra) & (hm < rb)                       # my halo entries owned by r
            if bool(theirs.any()):
                recv[r] = torch.nonzero(theirs).flatten()
        return cls(rank, world, row_start, indptr_local, cols, n, send, recv, halos[rank])

    def to(self, device):
        self.indptr = self.indptr.to(device)
        self.cols = self.cols.to(device)
        self.send = {r: v.to(device) for r, v in self.send.items()}
        self.recv = {r: v.to(device) for r, v in self.recv.items()}
        return self

    # -- communication ---------------------------------------------------------
    def exchange(self, x_ext):
        """Fill the halo part of x_ext [nloc + nhalo] from the owners: one
        message each way per neighbour pair, posted in rank order."""
        nl = self.nloc
        reqs, bufs = [], {}
        for r in sorted(set(self.send) | set(self.recv)):
            if r in self.send:
                reqs.append(dist.isend(x_ext[:nl][self.send[r]].contiguous(), r))
            if r in self.recv:
                bufs[r] = torch.empty(self.recv[r].numel(), dtype=x_ext.dtype, device=x_ext.device)
                reqs.append(dist.irecv(bufs[r], r))
        for q in reqs:
            q.wait()
        for r, buf in bufs.items():
            x_ext[nl + self.recv[r]] = buf

    @staticmethod
    def allreduce(vals):
        t = torch.stack(vals) if isinstance(vals, (list, tuple)) else vals
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t

    # -- local algebra ---------------------------------------------------------
    def spmv(self, values, x_ext):
        """Owned rows times the extended vector (torch CSR)."""
        A = torch.sparse_csr_tensor(self.indptr, self.cols, values, (self.nloc, self.nloc + self.halo_cols.numel()))
        return A @ x_ext

    def diagonal(self, values):
        rows = torch.repeat_interleave(torch.arange(self.nloc, device=values.device), self.indptr[1:] - self.indptr[:-1])
        d = torch.zeros(self.nloc, dtype=values.dtype, device=values.device)
        on = self.cols == rows
        d[rows[on]] = values[on]
        return d


def sharded_pcg(S: ShardedSystem, values, b, x, tol, max_iter):
    """Jacobi-PCG on the sharded system, in place on the owned x; returns
    (iterations, (r.D^-1 r)/(b.D^-1 b), status) with status 0 converged,
    -6 iteration cap, -7 breakdown (the library's codes).  Every rank takes
    the same steps: the decisions depend only on all-reduced scalars."""
    nl = S.nloc
    nh = S.halo_cols.numel()
    dinv = 1.0 / S.diagonal(values)
    ext = torch.zeros(nl + nh, dtype=values.dtype, device=values.device)
    ext[:nl] = x
    S.exchange(ext)
    r = b - S.spmv(values, ext)
    z = dinv * r
    p = z.clone()
    sc = S.allreduce([torch.dot(r, z), torch.dot(b, dinv * b)])
    rz, bb = float(sc[0]), float(sc[1])
    if bb == 0.0 or rz / bb < tol:
        return 0, (rz / bb if bb else 0.0), 0
    for it in range(1, max_iter + 1):
        ext[:nl] = p
        S.exchange(ext)
        q = S.spmv(values, ext)
        pq = float(S.allreduce(torch.dot(p, q).reshape(1))[0])
        if not pq > 0.0:
            return it, rz / bb, -7
        a = rz / pq
        x.add_(p, alpha=a)
        r.add_(q, alpha=-a)
        z = dinv * r
        rz_new = float(S.allreduce(torch.dot(r, z).reshape(1))[0])
        if rz_new / bb < tol:
            return it, rz_new / bb, 0
        p = z + (rz_new / rz) * p
        rz = rz_new
    return max_iter, rz / bb, -6


def rank_elements(elems, node_lo, node_hi):
    """Positions of the elements with a node in [node_lo, node_hi): the
    elements a rank owning those nodes evaluates (owned ones and the
    one-element halo), in their original order."""
    el = np.asarray(elems)
    return np.nonzero(((el >= node_lo) & (el < node_hi)).any(axis=1))[0]
