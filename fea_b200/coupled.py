"""The reduced system of an assembly whose nodes are tied to reference points.

With ``constraints.Couple`` the tied nodes' DOFs are not unknowns: they follow
the six DOFs (v, z) of a reference point, u_t = v + R(z) y_t - y_t.  The
element and pressure kernels still run on a plan whose rows are the free AND
the tied DOFs (the plan system); this class maps the reduced unknowns
(instance DOFs that are neither fixed nor tied, then the reference points'
free DOFs: the reference's GC order, assembly.py:90-105) to the plan's
displacement, and condenses the plan's R and K onto the reduced unknowns with
P = d u_plan / d gc:

    R_red = P^T R_plan - f_points,
    K_red = P^T K_plan P + sum_t R_plan[t] d2u_t/dz2   (the point's z-z block),

which is the matrix and residual that Couple.modify_R_K (couple.py:68-166)
appends to the reference's COO.  The pattern is the reference's structural
one: every plan entry that touches a tied DOF reaches all six DOFs of its
point, and each point's 6 x 6 block is full.  The pattern and the index maps
are built once; each assembly gathers and scatters on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .constraints import rigid_motion
from .plan import stream, vptr


class CoupledSystem:
    def __init__(self, asm, plan_mask, tied):
        """plan_mask: uint8 [N] plan DOF bits (free or tied); tied: list of
        (couple, node ids, reference point); asm: the initialized Assembly."""
        P = asm.plan
        self.asm = asm
        self.device = P.device
        dev = self.device
        N = plan_mask.shape[0]
        rem_inst = np.concatenate([asm.RGC_remain_index[ins._RGC_index].astype(np.uint8) @ np.array([1, 2, 4], np.uint8)
                                   for ins in asm._instances.values()]) if asm._instances else np.zeros(0, np.uint8)
        # plan DOF p <-> (node, component)
        pn, pk = [], []
        for k in range(3):
            nk = np.nonzero(plan_mask >> k & 1)[0]
            pn.append(nk)
            pk.append(np.full(nk.shape, k))
        pn, pk = np.concatenate(pn), np.concatenate(pk)
        order = np.lexsort((pk, pn))
        pn, pk = pn[order], pk[order]
        self.nplan = pn.shape[0]
        free_p = (rem_inst[pn] >> pk & 1).astype(bool)
        self.nfree = int(free_p.sum())
        # reference points: reduced DOFs after the instance DOFs
        self.points = []
        base = self.nfree
        rp_slot = {}
        for name, rp in asm._reference_points.items():
            keep = np.nonzero(asm.RGC_remain_index[rp._RGC_index])[0]
            self.points.append((name, rp, keep, base))
            rp_slot[name] = (keep, base)
            base += keep.shape[0]
        self.ndof = base
        # tied plan DOFs: (plan index, couple id, local node, component)
        node_to = {}
        self.couples = []
        for ci, (cpl, nodes, rp_name) in enumerate(tied):
            for i, n in enumerate(nodes):
                node_to[int(n)] = (ci, i)
            keep, b0 = rp_slot[rp_name]
            self.couples.append((cpl, torch.as_tensor(np.asarray(nodes), dtype=torch.int64), keep, b0))
        tied_p = np.nonzero(~free_p)[0]
        t_ci = np.array([node_to[int(pn[p])][0] for p in tied_p], dtype=np.int64)
        t_i = np.array([node_to[int(pn[p])][1] for p in tied_p], dtype=np.int64)
        t_q = pk[tied_p]
        red = np.full(self.nplan, -1, np.int64)
        red[free_p] = np.arange(self.nfree)
        tidx = np.full(self.nplan, -1, np.int64)
        tidx[tied_p] = np.arange(tied_p.shape[0])
        keep_of = [np.asarray(c[2], np.int64) for c in self.couples]
        base_of = np.array([c[3] for c in self.couples], np.int64)
        # plan CSR entries
        ip = P.indptr.cpu().numpy()
        ix = P.indices.cpu().numpy().astype(np.int64)
        prow = np.repeat(np.arange(self.nplan), np.diff(ip))
        ff = free_p[prow] & free_p[ix]
        fc = free_p[prow] & ~free_p[ix]
        cc = ~free_p[prow] & ~free_p[ix]
        keys = [red[prow[ff]] * self.ndof + red[ix[ff]]]
        # (free row, point DOF) pairs: each plan entry from a free row into a
        # tied column reaches every free DOF j of that column's point
        e_fc = np.nonzero(fc)[0]
        c_fc = t_ci[tidx[ix[e_fc]]] if e_fc.size else np.zeros(0, np.int64)
        pr_e, pr_j, pr_rows, pr_cols = [], [], [], []
        for c, keep in enumerate(keep_of):
            ec = e_fc[c_fc == c]
            for jj, j in enumerate(keep):
                pr_e.append(ec); pr_j.append(np.full(ec.shape, j)); pr_rows.append(red[prow[ec]])
                pr_cols.append(np.full(ec.shape, base_of[c] + jj))
        cat = lambda a: np.concatenate(a) if a else np.zeros(0, np.int64)
        pr_e, pr_j, pr_rows, pr_cols = cat(pr_e), cat(pr_j), cat(pr_rows), cat(pr_cols)
        pair_key = pr_rows * self.ndof + pr_cols
        upair, pslot = np.unique(pair_key, return_inverse=True)
        keys += [upair, (upair % self.ndof) * self.ndof + upair // self.ndof]
        # point x point entries: plan entries between tied DOFs, and each point's own full block
        e_cc = np.nonzero(cc)[0]
        c1 = t_ci[tidx[prow[e_cc]]] if e_cc.size else np.zeros(0, np.int64)
        c2 = t_ci[tidx[ix[e_cc]]] if e_cc.size else np.zeros(0, np.int64)
        q_rows, q_cols, q_e, q_a, q_b = [], [], [], [], []
        for ca, ka in enumerate(keep_of):
            for cb, kb in enumerate(keep_of):
                ec = e_cc[(c1 == ca) & (c2 == cb)]
                for ja, a in enumerate(ka):
                    for jb, b in enumerate(kb):
                        q_rows.append(np.full(ec.shape, base_of[ca] + ja)); q_cols.append(np.full(ec.shape, base_of[cb] + jb))
                        q_e.append(ec); q_a.append(np.full(ec.shape, a)); q_b.append(np.full(ec.shape, b))
        for c, keep in enumerate(keep_of):
            m = keep.shape[0]
            q_rows.append(np.repeat(base_of[c] + np.arange(m), m)); q_cols.append(np.tile(base_of[c] + np.arange(m), m))
            q_e.append(np.full(m * m, -1)); q_a.append(np.full(m * m, -1)); q_b.append(np.full(m * m, -1))
        q_rows, q_cols, q_e, q_a, q_b = cat(q_rows), cat(q_cols), cat(q_e), cat(q_a), cat(q_b)
        qkey = q_rows * self.ndof + q_cols
        uq, qslot = np.unique(qkey, return_inverse=True)
        keys.append(uq)
        allk = np.unique(np.concatenate(keys))
        self.nnz = allk.shape[0]
        rows = allk // self.ndof
        cols = allk % self.ndof
        self.indptr = torch.from_numpy(np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=self.ndof))])
                                       .astype(np.int64)).to(dev)
        self.indices = torch.from_numpy(cols.astype(np.int32)).to(dev)
        self._rows = torch.from_numpy(rows).to(dev)
        pos = lambda k: torch.from_numpy(np.searchsorted(allk, k)).to(dev)
        t = lambda a: torch.from_numpy(np.asarray(a, np.int64)).to(dev)
        # value maps
        self.ff_src = t(np.nonzero(ff)[0])
        self.ff_dst = pos(keys[0])
        self.fc_e, self.fc_slot = t(pr_e), t(pslot)
        self.fc_t = t(tidx[ix[pr_e]])
        self.fc_j = t(pr_j)
        self.npair = upair.shape[0]
        self.pair_dst, self.pair_dst_T = pos(upair), pos((upair % self.ndof) * self.ndof + upair // self.ndof)
        real = q_e >= 0
        self.cc_e, self.cc_slot = t(q_e[real]), t(qslot[real])
        self.cc_t1, self.cc_t2 = t(tidx[prow[q_e[real]]]), t(tidx[ix[q_e[real]]])
        self.cc_a, self.cc_b = t(q_a[real]), t(q_b[real])
        self.nq = uq.shape[0]
        self.q_dst = pos(uq)
        self.q_key = t(uq)
        # residual maps and tied-DOF tables
        self.free_pos = t(np.nonzero(free_p)[0])
        self.t_pos = t(tied_p)
        self.t_ci, self.t_i, self.t_q = t(t_ci), t(t_i), t(t_q)
        self._diag_pos = None

    # -- displacement -----------------------------------------------------------
    def motions(self, gc, order=2):
        """Per couple: (v, z, Y, dY, d2Y) at the reduced gc."""
        out = []
        for cpl, nodes, keep, b0 in self.couples:
            q = torch.zeros(6, dtype=torch.float64, device=self.device)
            q[torch.as_tensor(keep, device=self.device)] = gc[b0:b0 + keep.shape[0]]
            y = cpl._ref_location.to(self.device)
            Y, dY, d2Y = rigid_motion(q[3:], y, order=order)
            out.append((q[:3], q[3:], Y, dY, d2Y))
        return out

    def plan_gc(self, gc, mot=None):
        """The plan's displacement: free DOFs copied, tied DOFs v + R(z) y - y."""
        mot = self.motions(gc, order=0) if mot is None else mot
        g = torch.empty(self.nplan, dtype=torch.float64, device=self.device)
        g[self.free_pos] = gc[:self.nfree]
        if self.t_pos.numel():
            g[self.t_pos] = self._tied_values(mot)
        return g

    def _tied_values(self, mot):
        vals = torch.empty(self.t_pos.numel(), dtype=torch.float64, device=self.device)
        for ci, m in enumerate(mot):
            sel = self.t_ci == ci
            vals[sel] = m[0][self.t_q[sel]] + m[2][self.t_i[sel], self.t_q[sel]]
        return vals

    def _ptied(self, mot):
        """P rows of the tied DOFs over their point's six local DOFs [nt, 6]."""
        Pt = torch.zeros(self.t_pos.numel(), 6, dtype=torch.float64, device=self.device)
        for ci, m in enumerate(mot):
            sel = torch.nonzero(self.t_ci == ci).flatten()
            Pt[sel, self.t_q[sel]] = 1.0
            Pt[sel, 3:] = m[3][self.t_i[sel], self.t_q[sel]]
        return Pt

    def point_loads(self):
        """Per couple's point: the generalized force f [6] of its loads."""
        f = {}
        for ld in self.asm._loads.values():
            rp = getattr(ld, "rp_name", None)
            if rp is not None:
                v = f.setdefault(rp, torch.zeros(6, dtype=torch.float64, device=self.device))
                v[ld._offset:ld._offset + 3] += ld._value.to(self.device)
        return f

    # -- condensation -----------------------------------------------------------
    def condense(self, gc, R_plan, K_plan, mot):
        dev = self.device
        Pt = self._ptied(mot)
        R = torch.empty(self.ndof, dtype=torch.float64, device=dev)
        R[:self.nfree] = R_plan[self.free_pos]
        Rt = R_plan[self.t_pos]
        loads = self.point_loads()
        for name, rp, keep, b0 in self.points:
            R[b0:b0 + keep.shape[0]] = 0.0
        for ci, (cpl, nodes, keep, b0) in enumerate(self.couples):
            sel = self.t_ci == ci
            r6 = (Rt[sel, None] * Pt[sel]).sum(0)
            kk = torch.as_tensor(keep, device=dev)
            R[b0:b0 + keep.shape[0]] += r6[kk]
        for name, rp, keep, b0 in self.points:
            if name in loads:
                R[b0:b0 + keep.shape[0]] -= loads[name][torch.as_tensor(keep, device=dev)]
        if K_plan is None:
            return R, None
        K = torch.zeros(self.nnz, dtype=torch.float64, device=dev)
        K[self.ff_dst] = K_plan[self.ff_src]
        if self.npair:
            pv = torch.zeros(self.npair, dtype=torch.float64, device=dev)
            pv.index_add_(0, self.fc_slot, K_plan[self.fc_e] * Pt[self.fc_t, self.fc_j])
            K[self.pair_dst] = pv
            K[self.pair_dst_T] = pv
        qv = torch.zeros(self.nq, dtype=torch.float64, device=dev)
        if self.cc_e.numel():
            qv.index_add_(0, self.cc_slot, Pt[self.cc_t1, self.cc_a] * K_plan[self.cc_e] * Pt[self.cc_t2, self.cc_b])
        # the point's z-z block gains sum_t R_t d2u_t/dz2
        for ci, (cpl, nodes, keep, b0) in enumerate(self.couples):
            sel = torch.nonzero(self.t_ci == ci).flatten()
            G = torch.einsum("t,tpq->pq", Rt[sel], mot[ci][4][self.t_i[sel], self.t_q[sel]])
            full = torch.zeros(6, 6, dtype=torch.float64, device=dev)
            full[3:, 3:] = G
            kk = torch.as_tensor(keep, device=dev)
            blk = full[kk][:, kk]
            rr = (b0 + torch.arange(keep.shape[0], device=dev))[:, None].expand(-1, keep.shape[0])
            cc_ = (b0 + torch.arange(keep.shape[0], device=dev))[None, :].expand(keep.shape[0], -1)
            slot = torch.searchsorted(self.q_key, (rr * self.ndof + cc_).reshape(-1))
            qv.index_add_(0, slot, blk.reshape(-1))
        K[self.q_dst] += qv
        return R, K

    # -- the linear-system interface the solvers use -----------------------------
    def coo_indices(self):
        return torch.stack([self._rows, self.indices.to(torch.int64)])

    def zeros(self, n):
        return torch.zeros(n, dtype=torch.float64, device=self.device)

    def pcg(self, values, b, x, tol, max_iter, check_every=20, jacobi=True, raise_on_cap=False,
            raise_on_breakdown=True, generic=True):
        """Jacobi-PCG on this CSR (the library's plain-CSR solver)."""
        w = torch.empty(L.fea_pcg_work_len(self.ndof), dtype=torch.float64, device=self.device)
        it, rr = C.c_int32(0), C.c_double(0.0)
        st = L.fea_pcg_solve(self.ndof, vptr(self.indptr), vptr(self.indices), vptr(values), vptr(b), vptr(x),
                             float(tol), int(max_iter), int(check_every), int(bool(jacobi)), vptr(w), w.numel(),
                             C.byref(it), C.byref(rr), stream())
        ok = [L.FEA_OK, L.FEA_ENOTCONV] + ([] if raise_on_breakdown else [L.FEA_EBREAKDOWN])
        if st not in ok or (raise_on_cap and st == L.FEA_ENOTCONV):
            L.check(st, "fea_pcg_solve")
        return int(it.value), float(rr.value), st

    def to_f32(self, values):
        raise NotImplementedError("the FP32 inner solve covers systems without reference points")

    def pcg_mixed(self, *a, **k):
        raise NotImplementedError("the FP32 inner solve covers systems without reference points")
