"""Out-of-bounds writes, checked without a sanitizer: every output and scratch
buffer a kernel receives through the C ABI is the head of a larger device
buffer whose tail holds a sentinel, and after repeated calls the tails must
be untouched (inputs must be unchanged).  The meshes' element and node
counts are not multiples of the kernels' CTA sizes (hex5: 125 C3D8, tet3:
162 C3D4, cfg1: 6,000 C3D4 with a partly fixed boundary).
"""
import ctypes as C

import pytest
import torch

from tests.helpers import fea_model

pytestmark = pytest.mark.gpu

SENT = -7.25
TAIL = 4096
CASES = [("hex5", "C3D8"), ("tet3", "C3D4"), ("cfg1", "C3D4")]


def guarded(n, dtype=torch.float64):
    buf = torch.full((int(n) + TAIL,), SENT, dtype=dtype, device="cuda")
    return buf, buf[:int(n)]


def intact(buf, n):
    return bool((buf[int(n):] == SENT).all())


def ptr(t):
    return C.c_void_p(t.data_ptr())


def _model(golden, name, kind):
    g = golden(name)
    c, e, load = fea_model(g, kind)
    c.initialize()
    asm = c.assembly
    gc = (1e-3 * torch.randn(asm.plan.ndof, generator=torch.Generator().manual_seed(7),
                             dtype=torch.float64)).cuda()
    return asm, e, load, gc


@pytest.mark.parametrize("name,kind", CASES)
def test_assembly_energy_and_mass_stay_in_bounds(golden, name, kind):
    from fea_b200 import _lib as L
    asm, e, load, gc = _model(golden, name, kind)
    P = asm.plan
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    gc0 = gc.clone()
    mu, kappa = e.materials.parameters()
    g = P.groups[0]
    wl = int(L.fea_assemble_work_len(C.byref(g.desc)))
    for _ in range(3):
        Kb, K = guarded(P.nnz)
        Rb, R = guarded(P.ndof)
        Wb, W = guarded(wl)
        L.check(L.fea_assemble_volume(C.byref(P.nodes), C.byref(g.desc), float(mu), float(kappa), ptr(gc), ptr(K),
                                      ptr(R), None, 0, ptr(W) if wl else None, wl, st), "assemble")
        f = P.faces[0]
        L.check(L.fea_assemble_pressure(C.byref(P.nodes), C.byref(f.desc), float(load.pressure), ptr(asm._Xinst),
                                        ptr(gc), ptr(K), ptr(R), st), "pressure")
        ns = int(L.fea_reduce_scratch_len(g.ne))
        Ob, O_ = guarded(1)
        Sb, S = guarded(ns)
        L.check(L.fea_energy_volume(C.byref(P.nodes), C.byref(g.desc), float(mu), float(kappa), ptr(gc), ptr(O_),
                                    ptr(S), ns, st), "energy")
        nsf = int(L.fea_reduce_scratch_len(f.ne))
        Pb, Po = guarded(1)
        Fb, Fs = guarded(nsf)
        L.check(L.fea_energy_pressure(C.byref(P.nodes), C.byref(f.desc), ptr(asm._Xinst), ptr(gc), ptr(Po),
                                      ptr(Fs), nsf, st), "energy_pressure")
        mb, m = guarded(P.ndof)
        m.zero_()
        L.check(L.fea_lumped_mass(C.byref(P.nodes), C.byref(g.desc), 1.0, ptr(m), st), "lumped")
        Mb, Mv = guarded(P.nnz)
        Mv.zero_()
        L.check(L.fea_mass_csr(C.byref(P.nodes), C.byref(g.desc), 1.0, ptr(Mv), st), "mass_csr")
        torch.cuda.synchronize()
        for buf, n in ((Kb, P.nnz), (Rb, P.ndof), (Wb, wl), (Ob, 1), (Sb, ns), (Pb, 1), (Fb, nsf), (mb, P.ndof),
                       (Mb, P.nnz)):
            assert intact(buf, n)
        assert torch.equal(gc, gc0)
        assert bool(torch.isfinite(K).all()) and bool(torch.isfinite(R).all())


@pytest.mark.parametrize("name,kind", CASES)
def test_spmv_and_pcg_stay_in_bounds(golden, name, kind):
    from fea_b200 import _lib as L
    asm, e, load, gc = _model(golden, name, kind)
    P = asm.plan
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    R, K = asm.assemble_csr(gc)
    K0, b = K.clone(), (-R).contiguous()
    b0 = b.clone()
    yb, y = guarded(P.ndof)
    L.check(L.fea_spmv_nodes(C.byref(P.nodes), ptr(P.indices), ptr(K), ptr(b), ptr(y), st), "spmv")
    wl = int(L.fea_pcg_work_len(P.ndof))
    for _ in range(2):
        xb, x = guarded(P.ndof)
        x.zero_()
        wb, w = guarded(wl)
        it, rr = C.c_int32(0), C.c_double(0.0)
        s = L.fea_pcg_solve_nodes(C.byref(P.nodes), ptr(P.indices), ptr(K), ptr(b), ptr(x), 1e-20, 2000, 20,
                                  ptr(w), wl, C.byref(it), C.byref(rr), st)
        assert s in (L.FEA_OK, L.FEA_ENOTCONV)
        torch.cuda.synchronize()
        assert intact(xb, P.ndof) and intact(wb, wl)
    torch.cuda.synchronize()
    assert intact(yb, P.ndof)
    assert torch.equal(K, K0) and torch.equal(b, b0)


@pytest.mark.parametrize("name,kind", CASES)
def test_explicit_and_adjoint_stay_in_bounds(golden, name, kind):
    from fea_b200 import _lib as L
    asm, e, load, gc = _model(golden, name, kind)
    P = asm.plan
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    mu, kappa = e.materials.parameters()
    g = P.groups[0]
    minv = asm.lumped_mass_inv()
    n = P.ndof
    ub, u = guarded(n)
    u.copy_(gc)
    vhb, vh = guarded(n)
    vh.zero_()
    ab, a = guarded(n)
    a.zero_()
    vb, v = guarded(n)
    v.zero_()
    wl = int(L.fea_explicit_work_len(C.byref(P.nodes)))
    wb, w = guarded(wl)
    L.check(L.fea_explicit_run(C.byref(P.nodes), C.byref(g.desc), float(mu), float(kappa), ptr(minv), 1e-4, 7, 0, 1,
                               ptr(u), ptr(vh), ptr(a), ptr(v), ptr(w), wl, st), "explicit")
    N = P.n_nodes
    lam = (1e-2 * torch.randn(3 * N, generator=torch.Generator().manual_seed(8), dtype=torch.float64)).cuda()
    dXb, dX = guarded(3 * N)
    dX.zero_()
    dmb, dm = guarded(1)
    dm.zero_()
    ns = int(L.fea_reduce_scratch_len(g.ne))
    sb, s = guarded(ns)
    L.check(L.fea_adjoint_vjp_volume(C.byref(P.nodes), C.byref(g.desc), float(mu), float(kappa), ptr(gc), ptr(lam),
                                     ptr(dX), ptr(dm), ptr(s), ns, st), "vjp")
    torch.cuda.synchronize()
    for buf, m in ((ub, n), (vhb, n), (ab, n), (vb, n), (wb, wl), (dXb, 3 * N), (dmb, 1), (sb, ns)):
        assert intact(buf, m)
    assert bool(torch.isfinite(u).all()) and bool(torch.isfinite(dX).all())


def test_batched_pcg_stays_in_bounds():
    """Three cantilever systems in the batched PCG with their work buffers and
    iterates as guarded views; the right-hand sides and matrices unchanged."""
    from fea_b200 import serving, solver as S
    reqs = serving.make_requests(3, float("inf"), seed=5, min_elems=2000, max_elems=6000)
    eng = serving.BatchedPCG(4, 4 * max((serving.request_rows(r) // 3 + 15) // 16 + 1 for r in reqs), 8, True)
    keep = []
    for k, r in enumerate(reqs):
        asm = serving.build_assembly(r)
        R, K = asm.assemble_csr(asm.GC)
        b = (-R).contiguous()
        xb, x = guarded(b.numel())
        x.zero_()
        wl = serving.BatchedPCG.work_len(asm.plan)
        wb, w = guarded(wl)
        lin = S.LinearSolve(K, b, x, 1e-20, 100000, False)
        lin.x = x
        eng.assign(k, asm.plan, lin, w)
        keep.append((asm, K.clone(), b.clone(), K, b, xb, x, wb, wl))
    eng.sync()
    for k in range(len(reqs)):
        eng.start(k)
    for _ in range(5):
        eng.run_round()
    torch.cuda.synchronize()
    for asm, K0, b0, K, b, xb, x, wb, wl in keep:
        assert intact(xb, x.numel()) and intact(wb, wl)
        assert torch.equal(K, K0) and torch.equal(b, b0)
        assert bool(torch.isfinite(x).all())
