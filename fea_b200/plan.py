"""Device-resident assembly plan: the mesh, the reduced CSR pattern and the
per-node gather lists, plus typed wrappers of every library entry point.

One ``DevicePlan`` serves one reduced system (all element groups and pressure
face groups of an assembly, Dirichlet DOFs removed).  The plan is built once
per mesh on the host (C++ ``fea_plan_build``) and uploaded; every later call
only launches kernels on the current torch stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L

KIND = {"C3D4": L.FEA_C3D4, "C3D8": L.FEA_C3D8, "T3": L.FEA_T3, "Q4": L.FEA_Q4}
NODES_PER = {L.FEA_C3D4: 4, L.FEA_C3D8: 8, L.FEA_T3: 3, L.FEA_Q4: 4}


def vptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def need(t, n, device, what):
    """A caller's buffer handed to a kernel as a raw pointer: float64,
    contiguous, on the plan's device, at least n entries (else ValueError,
    before any launch)."""
    if t is None:
        return
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if (not isinstance(t, torch.Tensor) or t.dtype != torch.float64 or t.device.type != device.type
            or t.device.index != idx or not t.is_contiguous() or t.numel() < n):
        raise ValueError("%s: expected a contiguous float64 tensor of at least %d entries on %s, got %s" %
                         (what, n, device, "%s %s %s%s" % (tuple(t.shape), t.dtype, t.device,
                                                          "" if t.is_contiguous() else " (strided)")
                          if isinstance(t, torch.Tensor) else type(t).__name__))


class HostPlan:
    """Result of ``fea_plan_build`` (host memory)."""

    _DT = {L.FEA_A_RDOF: np.int32, L.FEA_A_MASK: np.uint8, L.FEA_A_DBASE: np.int32, L.FEA_A_VBASE: np.int64,
           L.FEA_A_ROWLEN: np.int32, L.FEA_A_INDPTR: np.int64, L.FEA_A_INDICES: np.int32,
           L.FEA_A_ADJPTR: np.int64, L.FEA_A_ADJCOL: np.int32, L.FEA_A_ADJOFF: np.int32,
           L.FEA_A_MOFF: np.int32}
    _GDT = {L.A_INC: np.int32, L.A_BOFF: np.uint16, L.A_NODEINC: np.int32, L.A_CHUNKPTR: np.int32,
            L.A_CHUNKINC: np.int32, L.A_CHUNKLIST: np.int32, L.A_CHUNKDIM: np.int32, L.A_SOFF: np.int32,
            L.A_ROFF: np.int32, L.A_UPTR: np.int64, L.A_UBLK: np.int64, L.A_ALLPTR: np.int32,
            L.A_ALLINC: np.int32, L.A_INCPOS: np.int32, L.A_STAGEPOS: np.int32, L.A_REGION: np.int64}

    def __init__(self, n_nodes, free_mask, groups, faces, vol_threads=0, smem_doubles=0):
        self._h = None
        mask = np.ascontiguousarray(free_mask, dtype=np.uint8)
        for _, c in list(groups) + list(faces):
            # node ids are checked before the int32 cast, which would wrap
            # an id of 2^32 + k onto node k
            c = np.asarray(c)
            if c.size and (c.min() < 0 or c.max() >= n_nodes):
                L.check(L.FEA_ERANGE, "fea_plan_build")
        gconn = [np.ascontiguousarray(c, dtype=np.int32) for _, c in groups]
        fconn = [np.ascontiguousarray(c, dtype=np.int32) for _, c in faces]
        self._keep = (mask, gconn, fconn)
        gk = (C.c_int32 * max(1, len(groups)))(*[k for k, _ in groups])
        gn = (C.c_int64 * max(1, len(groups)))(*[c.shape[0] for c in gconn])
        gp = (C.c_void_p * max(1, len(groups)))(*[c.ctypes.data for c in gconn])
        fk = (C.c_int32 * max(1, len(faces)))(*[k for k, _ in faces])
        fn = (C.c_int64 * max(1, len(faces)))(*[c.shape[0] for c in fconn])
        fp = (C.c_void_p * max(1, len(faces)))(*[c.ctypes.data for c in fconn])
        h = C.c_void_p()
        L.check(L.fea_plan_build(int(n_nodes), mask.ctypes.data, len(groups), gk, gn, gp, len(faces), fk, fn, fp,
                                 int(vol_threads), int(smem_doubles), C.byref(h)), "fea_plan_build")
        self._h = h
        self.n_groups, self.n_faces = len(groups), len(faces)

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and L is not None and getattr(L, "fea_plan_free", None) is not None:
            L.fea_plan_free(h)

    def scalar(self, sid, group=0):
        v = C.c_int64(0)
        L.check(L.fea_plan_get(self._h, sid, group, None, C.byref(v)), "fea_plan_get")
        return int(v.value)

    def array(self, aid, group=0):
        if aid >= L.F_BASE:
            dt = self._GDT[aid - L.F_BASE]
        elif aid >= L.G_BASE:
            dt = self._GDT[aid - L.G_BASE]
        else:
            dt = self._DT[aid]
        n = C.c_int64(0)
        L.check(L.fea_plan_get(self._h, aid, group, None, C.byref(n)), "fea_plan_get")
        out = np.empty(n.value, dtype=dt)
        L.check(L.fea_plan_get(self._h, aid, group, out.ctypes.data if n.value else None, C.byref(n)),
                "fea_plan_get")
        return out


class GatherGroup:
    """Device arrays of one element or face group and its ctypes descriptor."""

    def __init__(self, hp: HostPlan, base, index, kind, conn, device):
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.kind = kind
        self.nn = NODES_PER[kind]
        self.conn = dev(np.asarray(conn, dtype=np.int32))
        self.inc = dev(hp.array(base + L.A_INC, index))
        self.boff = dev(hp.array(base + L.A_BOFF, index).view(np.int16))
        nodeinc = hp.array(base + L.A_NODEINC, index)
        self.nodeinc = dev(nodeinc)
        self.chunkptr = dev(hp.array(base + L.A_CHUNKPTR, index))
        self.chunkinc = dev(hp.array(base + L.A_CHUNKINC, index))
        self.chunklist = dev(hp.array(base + L.A_CHUNKLIST, index))
        self.chunkdim = dev(hp.array(base + L.A_CHUNKDIM, index))
        self.soff = dev(hp.array(base + L.A_SOFF, index))
        self.roff = dev(hp.array(base + L.A_ROFF, index))
        uptr = hp.array(base + L.A_UPTR, index) if base == L.G_BASE else np.zeros(0, np.int64)
        self.uptr = dev(uptr) if uptr.size else None
        self.ublk = dev(hp.array(base + L.A_UBLK, index)) if uptr.size else None
        self.incpos = dev(hp.array(base + L.A_INCPOS, index)) if uptr.size else None
        self.stagepos = dev(hp.array(base + L.A_STAGEPOS, index)) if uptr.size else None
        region = hp.array(base + L.A_REGION, index) if uptr.size else np.zeros(1, np.int64)
        self.region = dev(region) if uptr.size else None
        nblk = int(region[-1])
        maxblk = int(np.diff(region).max()) if region.size > 1 else 0
        self.allptr = dev(hp.array(base + L.A_ALLPTR, index))
        self.allinc = dev(hp.array(base + L.A_ALLINC, index))
        self.ne = int(self.conn.shape[0])
        # True when every node with free DOFs has an incidence in this group
        self.covers_active = bool(np.all((np.diff(nodeinc) > 0) | (hp.array(L.FEA_A_MASK) == 0)))
        self.desc = L.Group(kind, self.nn, self.ne, self.conn.data_ptr(), self.inc.data_ptr(), self.boff.data_ptr(),
                            self.nodeinc.data_ptr(), self.chunkptr.data_ptr(), self.chunkinc.data_ptr(),
                            self.chunklist.data_ptr(), self.chunkdim.data_ptr(), self.soff.data_ptr(),
                            self.roff.data_ptr(), self.uptr.data_ptr() if self.uptr is not None else None,
                            self.ublk.data_ptr() if self.ublk is not None else None,
                            self.allptr.data_ptr(), self.allinc.data_ptr(),
                            hp.scalar(base + L.S_NCHUNK, index),
                            hp.scalar(base + L.S_MAXVAL, index), hp.scalar(base + L.S_THREADS, index),
                            hp.scalar(base + L.S_SMEM, index),
                            self.incpos.data_ptr() if self.incpos is not None else None,
                            self.stagepos.data_ptr() if self.stagepos is not None else None,
                            self.region.data_ptr() if self.region is not None else None, nblk, maxblk,
                            hp.scalar(L.FEA_S_G_HXSTRIDE, index) if uptr.size else 0)
        self.nchunk = int(self.desc.nchunk)


class DevicePlan:
    """Reduced system of one assembly on one CUDA device.

    X: [N,3] float64 reference coordinates (elements); free_mask: uint8 [N]
    (bit k = DOF k free); groups: [(kind name, conn [E,nn])]; faces:
    [(kind name, conn [F,nf])].
    """

    def __init__(self, X, free_mask, groups, faces=(), device=None, vol_threads=0, smem_doubles=0):
        if not torch.cuda.is_available():
            raise RuntimeError("fea_b200 needs a CUDA device (sm_100a); none is available")
        self.device = torch.device(device if device is not None else "cuda")
        Xn = np.ascontiguousarray(torch.as_tensor(X).detach().cpu().numpy(), dtype=np.float64)
        self.n_nodes = Xn.shape[0]
        gl = [(KIND[k], np.asarray(c)) for k, c in groups]
        fl = [(KIND[k], np.asarray(c)) for k, c in faces]
        with torch.cuda.device(self.device):
            self.host = hp = HostPlan(self.n_nodes, free_mask, gl, fl, vol_threads, smem_doubles)
            dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
            self.ndof = hp.scalar(L.FEA_S_NDOF)
            self.nnz = hp.scalar(L.FEA_S_NNZ)
            self.X = dev(Xn)
            self.rdof = dev(hp.array(L.FEA_A_RDOF))
            self.mask = dev(hp.array(L.FEA_A_MASK))
            self.dbase = dev(hp.array(L.FEA_A_DBASE))
            self.vbase = dev(hp.array(L.FEA_A_VBASE))
            self.rowlen = dev(hp.array(L.FEA_A_ROWLEN))
            self.indptr = dev(hp.array(L.FEA_A_INDPTR))
            self.indices = dev(hp.array(L.FEA_A_INDICES))
            self.adjptr = dev(hp.array(L.FEA_A_ADJPTR))
            self.adjcol = dev(hp.array(L.FEA_A_ADJCOL))
            self.adjoff = dev(hp.array(L.FEA_A_ADJOFF))
            self.moff = dev(hp.array(L.FEA_A_MOFF))
            self.nodes = L.Nodes(self.n_nodes, self.ndof, self.nnz, self.X.data_ptr(), self.rdof.data_ptr(),
                                 self.mask.data_ptr(), self.vbase.data_ptr(), self.rowlen.data_ptr(),
                                 self.dbase.data_ptr(), self.adjptr.data_ptr(), self.adjcol.data_ptr(),
                                 self.adjoff.data_ptr(), self.moff.data_ptr())
            self.groups = [GatherGroup(hp, L.G_BASE, i, k, c, self.device) for i, (k, c) in enumerate(gl)]
            self.faces = [GatherGroup(hp, L.F_BASE, i, k, c, self.device) for i, (k, c) in enumerate(fl)]
        self._scratch = None
        self._coo = None

    # -- buffers ------------------------------------------------------------
    def zeros(self, n, dtype=torch.float64):
        return torch.zeros(n, dtype=dtype, device=self.device)

    def scratch(self, n):
        if self._scratch is None or self._scratch.numel() < n:
            self._scratch = torch.empty(max(n, 1024), dtype=torch.float64, device=self.device)
        return self._scratch

    def coo_indices(self):
        """int64 [2, nnz] (row, col) of the reduced CSR pattern (cached)."""
        if self._coo is None:
            counts = self.indptr[1:] - self.indptr[:-1]
            rows = torch.repeat_interleave(torch.arange(self.ndof, device=self.device), counts)
            self._coo = torch.stack([rows, self.indices.to(torch.int64)])
        return self._coo

    # -- element / load kernels ---------------------------------------------
    def stage(self, gi):
        """Scratch of the element kernels of group gi (C3D8: staged upper block rows and residual slots)."""
        g = self.groups[gi]
        n = int(L.fea_assemble_work_len(C.byref(g.desc)))
        if n == 0:
            return None, 0
        if getattr(g, "_stage", None) is None or g._stage.numel() < n:
            g._stage = torch.empty(n, dtype=torch.float64, device=self.device)
        return g._stage, n

    def assemble_volume(self, gi, mu, kappa, gc, K=None, R=None, elemR=None, accumulate=False):
        g = self.groups[gi]
        need(gc, self.ndof, self.device, "gc")
        need(K, self.nnz, self.device, "K")
        need(R, self.ndof, self.device, "R")
        need(elemR, g.nn * 3 * g.ne, self.device, "elemR")
        w, wn = self.stage(gi) if K is not None else (None, 0)
        L.check(L.fea_assemble_volume(C.byref(self.nodes), C.byref(g.desc), float(mu), float(kappa), vptr(gc),
                                      vptr(K), vptr(R), vptr(elemR), int(bool(accumulate)), vptr(w), int(wn),
                                      stream()), "fea_assemble_volume")

    def assemble_pressure(self, fi, p, Xinst, gc, K=None, R=None):
        f = self.faces[fi]
        need(Xinst, 3 * self.n_nodes, self.device, "Xinst")
        need(gc, self.ndof, self.device, "gc")
        need(K, self.nnz, self.device, "K")
        need(R, self.ndof, self.device, "R")
        L.check(L.fea_assemble_pressure(C.byref(self.nodes), C.byref(f.desc), float(p), vptr(Xinst), vptr(gc),
                                        vptr(K), vptr(R), stream()), "fea_assemble_pressure")

    def energy_volume(self, gi, mu, kappa, gc, out):
        g = self.groups[gi]
        n = L.fea_reduce_scratch_len(g.ne)
        s = self.scratch(n)
        L.check(L.fea_energy_volume(C.byref(self.nodes), C.byref(g.desc), float(mu), float(kappa), vptr(gc),
                                    vptr(out), vptr(s), s.numel(), stream()), "fea_energy_volume")

    def pressure_volume(self, fi, Xinst, gc, out):
        f = self.faces[fi]
        n = L.fea_reduce_scratch_len(f.ne)
        s = self.scratch(n)
        L.check(L.fea_energy_pressure(C.byref(self.nodes), C.byref(f.desc), vptr(Xinst), vptr(gc), vptr(out),
                                      vptr(s), s.numel(), stream()), "fea_energy_pressure")

    # -- device line search (fea_ls_*) --------------------------------------------
    def ls_prepare(self, dgc, R, e0, state):
        nb = min((self.ndof + 255) // 256, 1024) if self.ndof else 1
        s = self.scratch(2 * nb)
        L.check(L.fea_ls_prepare(self.ndof, vptr(dgc), vptr(R), vptr(e0), vptr(state), vptr(s), s.numel(),
                                 stream()), "fea_ls_prepare")

    def ls_energy_volume(self, gi, mu, kappa, gc, dgc, state, k0, out, accumulate):
        g = self.groups[gi]
        s = self.scratch(L.fea_ls_scratch_len(g.ne))
        L.check(L.fea_ls_energy_volume(C.byref(self.nodes), C.byref(g.desc), float(mu), float(kappa), vptr(gc),
                                       vptr(dgc), vptr(state), int(k0), int(bool(accumulate)), vptr(out), vptr(s),
                                       s.numel(), stream()), "fea_ls_energy_volume")

    def ls_energy_pressure(self, fi, p, Xinst, gc, dgc, state, k0, out, accumulate):
        f = self.faces[fi]
        s = self.scratch(L.fea_ls_scratch_len(f.ne))
        L.check(L.fea_ls_energy_pressure(C.byref(self.nodes), C.byref(f.desc), float(p), vptr(Xinst), vptr(gc),
                                         vptr(dgc), vptr(state), int(k0), int(bool(accumulate)), vptr(out), vptr(s),
                                         s.numel(), stream()), "fea_ls_energy_pressure")

    def ls_select(self, E, k0, c1, max_step, state, dgc, gc):
        L.check(L.fea_ls_select(self.ndof, vptr(E), int(k0), float(c1), float(max_step), vptr(state), vptr(dgc),
                                vptr(gc), stream()), "fea_ls_select")

    def adjoint_vjp_volume(self, gi, mu, kappa, gc, lam_full, dX, dmu):
        """dX += d(lam . R_e)/dX (all nodes); dmu[0] = d(lam . R_e)/dmu."""
        g = self.groups[gi]
        s = self.scratch(L.fea_reduce_scratch_len(g.ne))
        L.check(L.fea_adjoint_vjp_volume(C.byref(self.nodes), C.byref(g.desc), float(mu), float(kappa), vptr(gc),
                                         vptr(lam_full), vptr(dX), vptr(dmu), vptr(s), s.numel(), stream()),
                "fea_adjoint_vjp_volume")

    def adjoint_hvp_pressure(self, fi, p, Xinst, gc, v_full, out):
        """out += p d2V/dx2 v (all nodes) for face group fi."""
        L.check(L.fea_adjoint_hvp_pressure(C.byref(self.nodes), C.byref(self.faces[fi].desc), float(p), vptr(Xinst),
                                           vptr(gc), vptr(v_full), vptr(out), stream()), "fea_adjoint_hvp_pressure")

    def lumped_mass_inv(self, rhos):
        m = self.zeros(self.ndof)
        for gi, rho in enumerate(rhos):
            L.check(L.fea_lumped_mass(C.byref(self.nodes), C.byref(self.groups[gi].desc), float(rho), vptr(m),
                                      stream()), "fea_lumped_mass")
        L.check(L.fea_invert_mass(self.ndof, vptr(m), stream()), "fea_invert_mass")
        return m

    def mass_csr(self, rhos):
        """Consistent mass in the values of the reduced CSR pattern [nnz]."""
        Mv = self.zeros(self.nnz)
        for gi, rho in enumerate(rhos):
            L.check(L.fea_mass_csr(C.byref(self.nodes), C.byref(self.groups[gi].desc), float(rho), vptr(Mv),
                                   stream()), "fea_mass_csr")
        return Mv

    def axpy(self, alpha, x, y):
        """y += alpha x (float64 device vectors of one length), in place."""
        if x.numel() != y.numel() or x.dtype != torch.float64 or y.dtype != torch.float64:
            raise ValueError("axpy: float64 vectors of one length")
        L.check(L.fea_axpy(int(y.numel()), float(alpha), vptr(x), vptr(y), stream()), "fea_axpy")
        return y

    # -- linear algebra --------------------------------------------------------
    def spmv(self, values, x, y=None, generic=False):
        """y = K x on the plan's reduced matrix (node-row kernel; generic=True
        runs the plain CSR kernel on the same arrays)."""
        y = self.zeros(self.ndof) if y is None else y
        if generic:
            L.check(L.fea_spmv(self.ndof, vptr(self.indptr), vptr(self.indices), vptr(values), vptr(x), vptr(y),
                               stream()), "fea_spmv")
        else:
            L.check(L.fea_spmv_nodes(C.byref(self.nodes), vptr(self.indices), vptr(values), vptr(x), vptr(y),
                                     stream()), "fea_spmv_nodes")
        return y

    def pcg(self, values, b, x, tol, max_iter, check_every=20, jacobi=True, raise_on_cap=False,
            raise_on_breakdown=True, generic=False):
        """Jacobi-PCG, in place on x. Returns (iterations, relres, status).
        The node-row solver runs unless jacobi is False or generic is True."""
        n = self.ndof
        wl = L.fea_pcg_work_len(n)
        w = self.scratch(wl)
        it, rr = C.c_int32(0), C.c_double(0.0)
        if generic or not jacobi:
            st = L.fea_pcg_solve(n, vptr(self.indptr), vptr(self.indices), vptr(values), vptr(b), vptr(x),
                                 float(tol), int(max_iter), int(check_every), int(bool(jacobi)), vptr(w), w.numel(),
                                 C.byref(it), C.byref(rr), stream())
        else:
            st = L.fea_pcg_solve_nodes(C.byref(self.nodes), vptr(self.indices), vptr(values), vptr(b), vptr(x),
                                       float(tol), int(max_iter), int(check_every), vptr(w), w.numel(), C.byref(it),
                                       C.byref(rr), stream())
        ok = [L.FEA_OK, L.FEA_ENOTCONV] + ([] if raise_on_breakdown else [L.FEA_EBREAKDOWN])
        if st not in ok or (raise_on_cap and st == L.FEA_ENOTCONV):
            L.check(st, "fea_pcg_solve")
        return int(it.value), float(rr.value), st

    def f32_layout(self):
        """The padded FP32 copy of this plan's matrix (fea_f32_layout_t):
        per node, its column list and rows on 16-byte boundaries, padded to
        multiples of 4.  Built once; fill_f32 writes the values."""
        if getattr(self, "_f32q", None) is None:
            mask = self.mask.cpu().numpy()
            f = np.array([bin(int(m) & 7).count("1") for m in range(8)], np.int64)[mask]
            L4 = np.where(mask != 0, (self.rowlen.cpu().numpy().astype(np.int64) + 3) & ~3, 0)
            cbase = torch.from_numpy(np.concatenate([[0], np.cumsum(L4)])).to(self.device)
            qbase = torch.from_numpy(np.concatenate([[0], np.cumsum(f * L4)])).to(self.device)
            cols = torch.zeros(max(int(cbase[-1]), 4), dtype=torch.int32, device=self.device)
            vals = torch.zeros(max(int(qbase[-1]), 4), dtype=torch.float32, device=self.device)
            desc = L.F32Layout(cbase.data_ptr(), qbase.data_ptr(), cols.data_ptr(), vals.data_ptr())
            self._f32q = (desc, cbase, qbase, cols, vals)
            self._f32q_cols = False
        return self._f32q

    def fill_f32(self, values):
        """FP32 values (and, the first time, the column lists) of the padded layout."""
        desc = self.f32_layout()[0]
        L.check(L.fea_f32_layout_fill(C.byref(self.nodes), vptr(self.indices), vptr(values), C.byref(desc),
                                      int(not self._f32q_cols), stream()), "fea_f32_layout_fill")
        self._f32q_cols = True
        return desc

    def pcg_mixed(self, values, values32, b, x, tol, inner_tol, max_iter, check_every=20, raise_on_breakdown=True,
                  generic=False):
        """FP32 inner CG with FP64 residual replacement, in place on x.
        values32 None: the padded FP32 node layout, filled from values here
        (128-bit loads); a float tensor: the plan's own layout (or CSR with
        generic).  Returns (iterations, replacements, relres, status)."""
        n = self.ndof
        wl = L.fea_pcg_mixed_work_len(n)
        w = self.scratch(wl)
        it, outer, rr = C.c_int32(0), C.c_int32(0), C.c_double(0.0)
        if values32 is None and not generic:
            desc = self.fill_f32(values)
            st = L.fea_pcg_solve_mixed_nodes32(C.byref(self.nodes), vptr(self.indices), vptr(values), C.byref(desc),
                                               vptr(b), vptr(x), float(tol), float(inner_tol), int(max_iter),
                                               int(check_every), vptr(w), w.numel(), C.byref(it), C.byref(outer),
                                               C.byref(rr), stream())
        elif generic:
            st = L.fea_pcg_solve_mixed(n, vptr(self.indptr), vptr(self.indices), vptr(values), vptr(values32),
                                       vptr(b), vptr(x), float(tol), float(inner_tol), int(max_iter),
                                       int(check_every), vptr(w), w.numel(), C.byref(it), C.byref(outer),
                                       C.byref(rr), stream())
        else:
            st = L.fea_pcg_solve_mixed_nodes(C.byref(self.nodes), vptr(self.indices), vptr(values), vptr(values32),
                                             vptr(b), vptr(x), float(tol), float(inner_tol), int(max_iter),
                                             int(check_every), vptr(w), w.numel(), C.byref(it), C.byref(outer),
                                             C.byref(rr), stream())
        ok = [L.FEA_OK, L.FEA_ENOTCONV] + ([] if raise_on_breakdown else [L.FEA_EBREAKDOWN])
        if st not in ok:
            L.check(st, "fea_pcg_solve_mixed")
        return int(it.value), int(outer.value), float(rr.value), st

    def to_f32(self, values, out=None):
        out = torch.empty(values.numel(), dtype=torch.float32, device=self.device) if out is None else out
        L.check(L.fea_convert_f32(values.numel(), vptr(values), vptr(out), stream()), "fea_convert_f32")
        return out

    def explicit_stage(self, stage, dt, minv, R, u, vh, vhp, a, v):
        """One stage of the central-difference step around an assembled
        residual R (fea_explicit_stage); unused arguments may be None."""
        L.check(L.fea_explicit_stage(self.ndof, int(stage), float(dt), vptr(minv), vptr(R), vptr(u), vptr(vh),
                                     vptr(vhp), vptr(a), vptr(v), stream()), "fea_explicit_stage")

    def explicit_run(self, gi, mu, kappa, minv, dt, steps, u, vh, a, v, fp32=False, init=False):
        w = self.scratch(L.fea_explicit_work_len(C.byref(self.nodes)))
        L.check(L.fea_explicit_run(C.byref(self.nodes), C.byref(self.groups[gi].desc), float(mu), float(kappa),
                                   vptr(minv), float(dt), int(steps), int(bool(fp32)), int(bool(init)), vptr(u),
                                   vptr(vh), vptr(a), vptr(v), vptr(w), w.numel(), stream()), "fea_explicit_run")
