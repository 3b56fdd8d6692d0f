"""Argument checks of the C ABI, on the host only: every device entry point
rejects a bad call with its documented status before its first CUDA call,
and launches nothing (the library's launch counter does not move).  The
calls pass fake device addresses that no check may dereference, so the
module runs only where no GPU is visible: there, a call that got past its
checks would return a CUDA error code instead of the expected status.
"""
import ctypes as C

import pytest
import torch

pytestmark = pytest.mark.skipif(torch.cuda.is_available(),
                                reason="fake device addresses: host-side checks only")

FAKE = 0x10000            # 16-byte aligned, never dereferenced
EINVAL, ERANGE, ECHUNK, EWORK, ETOOBIG = -1, -2, -3, -5, -8


def _p(k=0):
    return C.c_void_p(FAKE + 16 * k)


def _nodes(ndof=30):
    from fea_b200 import _lib as L
    N = L.Nodes()
    N.n_nodes, N.ndof, N.nnz = 10, ndof, 900
    for i, f in enumerate(("X_dev", "rdof_dev", "mask_dev", "vbase_dev", "rowlen_dev", "dbase_dev",
                           "adjptr_dev", "adjcol_dev", "adjoff_dev", "moff_dev")):
        setattr(N, f, FAKE + 16 * (i + 1))
    return N


def _group(kind, nn, threads, ne=5):
    from fea_b200 import _lib as L
    G = L.Group()
    G.kind, G.nn, G.ne, G.threads = kind, nn, ne, threads
    for i, (f, _) in enumerate(L.Group._fields_):
        if f.endswith("_dev"):
            setattr(G, f, FAKE + 16 * (i + 20))
    G.nchunk, G.maxval, G.smem_doubles, G.nblk, G.maxblk = 1, 8, 64, 36 * ne, 40
    return G


def _slot(n=100, nnz=900, work_len=None, active=1):
    from fea_b200 import _lib as L
    s = L.PcgbSlot()
    s.n, s.nnz = n, nnz
    for i, f in enumerate(("indptr_dev", "indices_dev", "values_dev", "b_dev", "x_dev", "work_dev")):
        setattr(s, f, FAKE + 16 * (i + 40))
    s.work_len = int(L.fea_pcgb_work_len(n, 0)) if work_len is None else work_len
    s.tol, s.max_iter, s.active = 1e-20, 100, active
    return s


def test_volume_entry_points_check_arguments_first():
    from fea_b200 import _lib as L
    n0 = L.fea_launch_count()
    N = _nodes()
    hexg = _group(L.FEA_C3D8, 8, 32)
    tetg = _group(L.FEA_C3D4, 4, 256)
    wl = int(L.fea_assemble_work_len(C.byref(hexg)))
    assert wl == ((36 * 5 * 9 + 1) & ~1) + 5 * 8 * 4
    assert L.fea_assemble_work_len(C.byref(tetg)) == 0 and L.fea_assemble_work_len(None) == 0

    def vol(G, K=_p(1), R=_p(2), elemR=None, work=_p(3), work_len=wl, nodes=N):
        return L.fea_assemble_volume(C.byref(nodes) if nodes is not None else None, C.byref(G), 1.0, 10.0,
                                     _p(4), K, R, elemR, 0, work, work_len, None)

    assert vol(hexg, nodes=None) == EINVAL
    assert vol(_group(L.FEA_T3, 3, 128)) == EINVAL                  # a face kind
    assert vol(_group(L.FEA_C3D8, 4, 32)) == EINVAL                 # node count of the kind
    assert vol(_group(L.FEA_C3D8, 8, 128)) == ECHUNK                # threads of another plan layout
    assert vol(_group(L.FEA_C3D4, 4, 32)) == ECHUNK
    assert vol(hexg, work=None) == EWORK
    assert vol(hexg, work_len=wl - 1) == EWORK
    assert vol(hexg, work=C.c_void_p(FAKE + 8)) == EINVAL           # not 16-byte aligned
    for f in ("incpos_dev", "stagepos_dev", "region_dev", "uptr_dev", "ublk_dev"):
        g = _group(L.FEA_C3D8, 8, 32)
        setattr(g, f, None)
        assert vol(g) == EINVAL, f
    g = _group(L.FEA_C3D8, 8, 32)
    g.maxblk = -1
    assert vol(g) == EINVAL
    assert vol(hexg, K=None, R=None) == 0                           # nothing to compute
    assert vol(tetg, K=None, R=None) == 0
    assert vol(hexg, K=None, R=None, elemR=_p(5)) == EINVAL         # the R-only path writes R
    # gc may be NULL only when no DOF is free
    assert L.fea_assemble_volume(C.byref(N), C.byref(hexg), 1.0, 10.0, None, _p(1), _p(2), None, 0, _p(3), wl,
                                 None) == EINVAL
    N0 = _nodes(ndof=0)
    assert L.fea_assemble_volume(C.byref(N0), C.byref(hexg), 1.0, 10.0, None, None, None, None, 0, None, 0,
                                 None) == 0
    # an element group without elements needs no staging scratch, but the
    # node-side arrays its gather reads
    e0 = _group(L.FEA_C3D8, 8, 32, ne=0)
    e0.nblk, e0.maxval = 0, 0
    assert L.fea_assemble_work_len(C.byref(e0)) == 0
    e0.region_dev = None
    assert L.fea_assemble_volume(C.byref(N), C.byref(e0), 1.0, 10.0, _p(4), _p(1), _p(2), None, 0, None, 0,
                                 None) == EINVAL

    face = _group(L.FEA_Q4, 4, 128)
    assert L.fea_assemble_pressure(C.byref(N), C.byref(face), 1.0, _p(1), _p(2), None, None, None) == 0
    assert L.fea_assemble_pressure(C.byref(N), C.byref(tetg), 1.0, _p(1), _p(2), _p(3), _p(4), None) == EINVAL
    assert L.fea_assemble_pressure(C.byref(N), C.byref(_group(L.FEA_T3, 3, 64)), 1.0, _p(1), _p(2), _p(3),
                                   _p(4), None) == EINVAL
    assert L.fea_assemble_pressure(C.byref(N), C.byref(face), 1.0, None, _p(2), _p(3), _p(4), None) == EINVAL

    ns = int(L.fea_reduce_scratch_len(tetg.ne))
    assert ns == 2
    assert L.fea_energy_volume(C.byref(N), C.byref(tetg), 1.0, 10.0, _p(1), _p(2), _p(3), ns - 1, None) == EWORK
    assert L.fea_energy_volume(C.byref(N), C.byref(face), 1.0, 10.0, _p(1), _p(2), _p(3), ns, None) == EINVAL
    assert L.fea_energy_pressure(C.byref(N), C.byref(face), _p(1), _p(2), _p(3), _p(4), ns - 1, None) == EWORK
    assert L.fea_energy_pressure(C.byref(N), C.byref(tetg), _p(1), _p(2), _p(3), _p(4), ns, None) == EINVAL
    big = _group(L.FEA_C3D4, 4, 128, ne=L.FEA_NOALLOC_MAX_ELEMS + 1)
    assert L.fea_energy_volume_noalloc(C.byref(N), C.byref(big), 1.0, 10.0, _p(1), _p(2), None) == ETOOBIG
    neg = _group(L.FEA_C3D4, 4, 128, ne=-1)
    assert L.fea_energy_volume_noalloc(C.byref(N), C.byref(neg), 1.0, 10.0, _p(1), _p(2), None) == EINVAL
    assert L.fea_energy_volume_noalloc(C.byref(N), C.byref(tetg), 1.0, 10.0, _p(1), None, None) == EINVAL

    assert L.fea_lumped_mass(C.byref(N), C.byref(tetg), 1.0, None, None) == EINVAL
    assert L.fea_lumped_mass(C.byref(N), C.byref(face), 1.0, _p(1), None) == EINVAL
    nob = _group(L.FEA_C3D8, 8, 32)
    nob.boff_dev = None
    assert L.fea_mass_csr(C.byref(N), C.byref(nob), 1.0, _p(1), None) == EINVAL
    assert L.fea_axpy(-1, 1.0, _p(1), _p(2), None) == EINVAL
    assert L.fea_axpy(5, 1.0, None, _p(2), None) == EINVAL
    assert L.fea_axpy(0, 1.0, None, None, None) == 0
    assert L.fea_invert_mass(-1, _p(1), None) == EINVAL
    assert L.fea_invert_mass(0, _p(1), None) == 0

    ewl = int(L.fea_explicit_work_len(C.byref(N)))
    assert ewl == 30 + 12 * 10                                      # u buffer + two node-major copies
    assert L.fea_explicit_work_len(None) == 0
    ex = lambda G, steps=3, wlen=ewl, w=_p(6): L.fea_explicit_run(C.byref(N), C.byref(G), 1.0, 10.0, _p(1), 1e-4,
                                                                  steps, 0, 0, _p(2), _p(3), _p(4), _p(5), w, wlen,
                                                                  None)
    assert ex(tetg, steps=-1) == EINVAL
    assert ex(face) == EINVAL
    assert ex(tetg, wlen=ewl - 1) == EWORK
    assert ex(tetg, w=C.c_void_p(FAKE + 8)) == EINVAL               # not 16-byte aligned
    assert L.fea_adjoint_vjp_volume(C.byref(N), C.byref(tetg), 1.0, 10.0, _p(1), _p(2), _p(3), _p(4), _p(5),
                                    ns - 1, None) == EWORK
    noall = _group(L.FEA_C3D4, 4, 128)
    noall.allptr_dev = None
    assert L.fea_adjoint_vjp_volume(C.byref(N), C.byref(noall), 1.0, 10.0, _p(1), _p(2), _p(3), _p(4), _p(5),
                                    ns, None) == EINVAL
    assert L.fea_adjoint_hvp_pressure(C.byref(N), C.byref(tetg), 1.0, _p(1), _p(2), _p(3), _p(4), None) == EINVAL
    assert L.fea_launch_count() == n0


def test_solver_entry_points_check_arguments_first():
    from fea_b200 import _lib as L
    n0 = L.fea_launch_count()
    N = _nodes(ndof=30)
    it, rr, outer = C.c_int32(-5), C.c_double(-5.0), C.c_int32(-5)
    wl = int(L.fea_pcg_work_len(30))
    wm = int(L.fea_pcg_mixed_work_len(30))
    assert wm > wl > 5 * 30
    cg = lambda n, work_len, work=_p(6): L.fea_pcg_solve(n, _p(1), _p(2), _p(3), _p(4), _p(5), 1e-20, 100, 10, 1,
                                                          work, work_len, C.byref(it), C.byref(rr), None)
    assert cg(-1, wl) == EINVAL
    assert cg(30, wl, work=None) == EINVAL
    assert cg(30, wl - 1) == EWORK
    assert cg(0, int(L.fea_pcg_work_len(0))) == 0 and it.value == 0 and rr.value == 0.0
    assert L.fea_pcg_solve(30, _p(1), _p(2), _p(3), _p(4), _p(5), 1e-20, -1, 10, 1, _p(6), wl, None, None,
                           None) == EINVAL
    cgn = lambda nodes, work_len: L.fea_pcg_solve_nodes(C.byref(nodes), _p(2), _p(3), _p(4), _p(5), 1e-20, 100,
                                                         10, _p(6), work_len, None, None, None)
    assert cgn(N, wl - 1) == EWORK
    nv = _nodes()
    nv.vbase_dev = None
    assert cgn(nv, wl) == EINVAL
    it.value, rr.value = -5, -5.0
    assert L.fea_pcg_solve_nodes(C.byref(_nodes(ndof=0)), _p(2), _p(3), _p(4), _p(5), 1e-20, 100, 10, _p(6),
                                 int(L.fea_pcg_work_len(0)), C.byref(it), C.byref(rr), None) == 0
    assert it.value == 0 and rr.value == 0.0
    mixed = lambda work_len, v32=_p(7): L.fea_pcg_solve_mixed(30, _p(1), _p(2), _p(3), v32, _p(4), _p(5), 1e-20,
                                                              0.0, 100, 10, _p(6), work_len, C.byref(it),
                                                              C.byref(outer), C.byref(rr), None)
    assert mixed(wm, v32=None) == EINVAL
    assert mixed(wl) == EWORK                                       # the FP64 length is not enough
    assert L.fea_pcg_solve_mixed_nodes(C.byref(N), _p(2), _p(3), _p(7), _p(4), _p(5), 1e-20, 0.0, 100, 10, _p(6),
                                       wm - 1, None, None, None, None) == EWORK
    assert L.fea_spmv(-1, _p(1), _p(2), _p(3), _p(4), _p(5), None) == EINVAL
    assert L.fea_spmv(0, _p(1), _p(2), _p(3), _p(4), _p(5), None) == 0
    assert L.fea_spmv_nodes(C.byref(nv), _p(2), _p(3), _p(4), _p(5), None) == EINVAL
    assert L.fea_spmv_nodes(C.byref(_nodes(ndof=0)), _p(2), _p(3), _p(4), _p(5), None) == 0
    assert L.fea_convert_f32(-1, _p(1), _p(2), None) == EINVAL
    assert L.fea_convert_f32(0, _p(1), _p(2), None) == 0
    assert L.fea_launch_count() == n0


def test_batched_pcg_rejects_a_bad_table_before_touching_the_device():
    """fea_pcgb_set checks every descriptor before its first device call: a
    valid slot 0 followed by a bad slot 1 returns the bad slot's status, not
    a CUDA error from clearing slot 0's counters."""
    from fea_b200 import _lib as L
    n0 = L.fea_launch_count()
    assert L.fea_pcgb_table_bytes(0, 10) == 0 and L.fea_pcgb_table_bytes(4, 0) == 0
    assert L.fea_pcgb_table_bytes(4, 10) > 4 * 16
    T = _p(60)

    def put(*slots, max_slots=4, max_items=1000):
        arr = (L.PcgbSlot * max(len(slots), 1))(*slots)
        return L.fea_pcgb_set(T, max_slots, max_items, len(slots), arr, None)

    assert put(_slot(), _slot(work_len=10)) == EWORK
    bad = _slot()
    bad.n = -1
    assert put(_slot(), bad) == EINVAL
    nob = _slot()
    nob.b_dev = None
    assert put(_slot(), nob) == EINVAL
    lay = _slot()
    lay.vbase_dev = FAKE                                            # node layout without its other arrays
    assert put(_slot(), lay) == EINVAL
    assert put(_slot(), _slot(), max_slots=1) == EINVAL
    assert L.fea_pcgb_set(None, 4, 1000, 0, None, None) == EINVAL
    assert L.fea_pcgb_set(T, 4, 1000, 1, None, None) == EINVAL
    # more active items than the table holds; an inactive slot adds none
    big = _slot(n=100000)
    assert put(big, max_items=10) == ERANGE
    assert L.fea_pcgb_start(T, 4, 1000, 4, 100, 900, None) == EINVAL
    assert L.fea_pcgb_start(T, 4, 1000, -1, 100, 900, None) == EINVAL
    assert L.fea_pcgb_start(T, 4, 1000, 0, 0, 0, None) == 0         # no rows: nothing to start
    assert L.fea_pcgb_iterate(T, 4, 1000, -1, None) == EINVAL
    assert L.fea_pcgb_iterate(None, 4, 1000, 1, None) == EINVAL
    assert L.fea_pcgb_state(T, 4, 1000, 5, _p(1), None) == EINVAL
    assert L.fea_pcgb_state(T, 4, 1000, 2, None, None) == EINVAL
    assert L.fea_pcgb_state(T, 4, 1000, 0, None, None) == 0
    assert L.fea_launch_count() == n0
