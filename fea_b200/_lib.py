"""ctypes binding of libfea_b200.so (the C ABI declared in include/fea_b200.h).

The library is built in-tree (``python fea_b200/_build.py``).  Importing this
module loads it; a missing library raises ImportError — there is no fallback
implementation of any kernel.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfea_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("fea_b200: native library %s is missing; build it with "
                      "`python %s` (nvcc, sm_100a)" % (LIB_PATH, os.path.join(HERE, "_build.py")))
lib = C.CDLL(LIB_PATH)

FEA_OK = 0
ERRORS = {-1: "invalid argument", -2: "index out of range", -3: "a node does not fit one gather chunk",
          -4: "shared memory request exceeds the device limit", -5: "work buffer too small",
          -6: "iteration cap reached", -7: "PCG breakdown (p.Ap <= 0 or non-finite)",
          -8: "size beyond a fixed limit (an allocation-free entry point, or FEA_PLAN_MAX_ELEMS per group)"}
FEA_EINVAL, FEA_ERANGE, FEA_ECHUNK, FEA_ESMEM, FEA_EWORK = -1, -2, -3, -4, -5
FEA_ENOTCONV = -6
FEA_EBREAKDOWN = -7
FEA_ETOOBIG = -8
FEA_NOALLOC_MAX_ELEMS = 4194304
FEA_PLAN_MAX_ELEMS = 134217727      # elements (faces) per group: incidences e * 16 + a in 32 bits

FEA_C3D4, FEA_C3D8, FEA_T3, FEA_Q4 = 4, 8, 3, 40

(FEA_S_NDOF, FEA_S_NNZ, FEA_S_NNZB) = (0, 1, 2)
(FEA_A_RDOF, FEA_A_MASK, FEA_A_DBASE, FEA_A_VBASE, FEA_A_ROWLEN, FEA_A_INDPTR, FEA_A_INDICES,
 FEA_A_ADJPTR, FEA_A_ADJCOL, FEA_A_ADJOFF, FEA_A_MOFF) = range(10, 21)
G_BASE, F_BASE = 30, 50
FEA_S_G_HXSTRIDE = 70     # element-group scalar past the face id range
(A_INC, A_BOFF, A_NODEINC, A_CHUNKPTR, A_CHUNKINC, S_NCHUNK, S_MAXVAL, S_THREADS, S_SMEM, A_CHUNKLIST,
 A_CHUNKDIM, A_SOFF, A_ROFF, A_UPTR, A_UBLK, A_ALLPTR, A_ALLINC, A_INCPOS, A_STAGEPOS, A_REGION) = range(20)


class FeaError(RuntimeError):
    def __init__(self, what, status):
        self.status = status
        msg = ERRORS.get(status, "CUDA error %d" % status if status > 0 else "status %d" % status)
        super().__init__("%s failed: %s" % (what, msg))


def check(status, what):
    if status != FEA_OK:
        raise FeaError(what, status)
    return status


class Nodes(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("ndof", C.c_int64), ("nnz", C.c_int64),
                ("X_dev", C.c_void_p), ("rdof_dev", C.c_void_p), ("mask_dev", C.c_void_p),
                ("vbase_dev", C.c_void_p), ("rowlen_dev", C.c_void_p), ("dbase_dev", C.c_void_p),
                ("adjptr_dev", C.c_void_p), ("adjcol_dev", C.c_void_p), ("adjoff_dev", C.c_void_p),
                ("moff_dev", C.c_void_p)]


class Group(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nn", C.c_int32), ("ne", C.c_int64),
                ("conn_dev", C.c_void_p), ("inc_dev", C.c_void_p), ("boff_dev", C.c_void_p),
                ("nodeinc_dev", C.c_void_p), ("chunkptr_dev", C.c_void_p), ("chunkinc_dev", C.c_void_p),
                ("chunklist_dev", C.c_void_p), ("chunkdim_dev", C.c_void_p), ("soff_dev", C.c_void_p),
                ("roff_dev", C.c_void_p), ("uptr_dev", C.c_void_p), ("ublk_dev", C.c_void_p),
                ("allptr_dev", C.c_void_p), ("allinc_dev", C.c_void_p),
                ("nchunk", C.c_int64), ("maxval", C.c_int32), ("threads", C.c_int32),
                ("smem_doubles", C.c_int64), ("incpos_dev", C.c_void_p), ("stagepos_dev", C.c_void_p),
                ("region_dev", C.c_void_p), ("nblk", C.c_int64), ("maxblk", C.c_int32), ("hx_stride", C.c_int32)]


class PcgbSlot(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz", C.c_int64), ("indptr_dev", C.c_void_p), ("indices_dev", C.c_void_p),
                ("values_dev", C.c_void_p), ("b_dev", C.c_void_p), ("x_dev", C.c_void_p), ("work_dev", C.c_void_p),
                ("work_len", C.c_int64), ("tol", C.c_double), ("max_iter", C.c_int32), ("active", C.c_int32),
                ("n_nodes", C.c_int64), ("vbase_dev", C.c_void_p), ("rowlen_dev", C.c_void_p),
                ("dbase_dev", C.c_void_p), ("mask_dev", C.c_void_p)]


P = C.c_void_p
I32, I64, D = C.c_int32, C.c_int64, C.c_double
NP, GP = C.POINTER(Nodes), C.POINTER(Group)


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


fea_plan_build = _sig("fea_plan_build", I32, I64, P, I32, P, P, P, I32, P, P, P, I32, I64, C.POINTER(P))
fea_plan_free = _sig("fea_plan_free", None, P)
fea_plan_get = _sig("fea_plan_get", I32, P, I32, I32, P, C.POINTER(I64))
fea_assemble_work_len = _sig("fea_assemble_work_len", I64, GP)
fea_assemble_volume = _sig("fea_assemble_volume", I32, NP, GP, D, D, P, P, P, P, I32, P, I64, P)
fea_assemble_pressure = _sig("fea_assemble_pressure", I32, NP, GP, D, P, P, P, P, P)
fea_reduce_scratch_len = _sig("fea_reduce_scratch_len", I64, I64)
fea_energy_volume = _sig("fea_energy_volume", I32, NP, GP, D, D, P, P, P, I64, P)
fea_energy_pressure = _sig("fea_energy_pressure", I32, NP, GP, P, P, P, P, I64, P)
fea_energy_volume_noalloc = _sig("fea_energy_volume_noalloc", I32, NP, GP, D, D, P, P, P)
fea_lumped_mass = _sig("fea_lumped_mass", I32, NP, GP, D, P, P)
fea_invert_mass = _sig("fea_invert_mass", I32, I64, P, P)
fea_mass_csr = _sig("fea_mass_csr", I32, NP, GP, D, P, P)
fea_axpy = _sig("fea_axpy", I32, I64, D, P, P, P)
fea_pcg_work_len = _sig("fea_pcg_work_len", I64, I64)
fea_pcg_solve = _sig("fea_pcg_solve", I32, I64, P, P, P, P, P, D, I32, I32, I32, P, I64,
                     C.POINTER(I32), C.POINTER(D), P)
fea_pcg_mixed_work_len = _sig("fea_pcg_mixed_work_len", I64, I64)
fea_pcg_solve_mixed = _sig("fea_pcg_solve_mixed", I32, I64, P, P, P, P, P, P, D, D, I32, I32, P, I64,
                           C.POINTER(I32), C.POINTER(I32), C.POINTER(D), P)
fea_spmv = _sig("fea_spmv", I32, I64, P, P, P, P, P, P)
fea_spmv_nodes = _sig("fea_spmv_nodes", I32, NP, P, P, P, P, P)
fea_pcg_solve_nodes = _sig("fea_pcg_solve_nodes", I32, NP, P, P, P, P, D, I32, I32, P, I64, C.POINTER(I32),
                           C.POINTER(D), P)
fea_pcg_solve_mixed_nodes = _sig("fea_pcg_solve_mixed_nodes", I32, NP, P, P, P, P, P, D, D, I32, I32, P, I64,
                                 C.POINTER(I32), C.POINTER(I32), C.POINTER(D), P)
fea_convert_f32 = _sig("fea_convert_f32", I32, I64, P, P, P)


class F32Layout(C.Structure):
    _fields_ = [("cbase_dev", C.c_void_p), ("qbase_dev", C.c_void_p), ("cols_dev", C.c_void_p),
                ("vals_dev", C.c_void_p)]


fea_f32_layout_fill = _sig("fea_f32_layout_fill", I32, NP, P, P, C.POINTER(F32Layout), I32, P)
fea_pcg_solve_mixed_nodes32 = _sig("fea_pcg_solve_mixed_nodes32", I32, NP, P, P, C.POINTER(F32Layout), P, P, D, D,
                                   I32, I32, P, I64, C.POINTER(I32), C.POINTER(I32), C.POINTER(D), P)
fea_pcgb_work_len = _sig("fea_pcgb_work_len", I64, I64, I64)
fea_pcgb_table_bytes = _sig("fea_pcgb_table_bytes", I64, I32, I64)
fea_pcgb_set = _sig("fea_pcgb_set", I32, P, I32, I64, I32, C.POINTER(PcgbSlot), P)
fea_pcgb_start = _sig("fea_pcgb_start", I32, P, I32, I64, I32, I64, I64, P)
fea_pcgb_iterate = _sig("fea_pcgb_iterate", I32, P, I32, I64, I32, P)
fea_pcgb_state = _sig("fea_pcgb_state", I32, P, I32, I64, I32, P, P)
fea_explicit_work_len = _sig("fea_explicit_work_len", I64, NP)
fea_explicit_run = _sig("fea_explicit_run", I32, NP, GP, D, D, P, D, I64, I32, I32, P, P, P, P, P, I64, P)
fea_explicit_stage = _sig("fea_explicit_stage", I32, I64, I32, D, P, P, P, P, P, P, P, P)
fea_ls_ladder_len = _sig("fea_ls_ladder_len", I32)
fea_ls_scratch_len = _sig("fea_ls_scratch_len", I64, I64)
fea_ls_prepare = _sig("fea_ls_prepare", I32, I64, P, P, P, P, P, I64, P)
fea_ls_energy_volume = _sig("fea_ls_energy_volume", I32, NP, GP, D, D, P, P, P, I32, I32, P, P, I64, P)
fea_ls_energy_pressure = _sig("fea_ls_energy_pressure", I32, NP, GP, D, P, P, P, P, I32, I32, P, P, I64, P)
fea_ls_select = _sig("fea_ls_select", I32, I64, P, I32, D, D, P, P, P, P)
FEA_LS_M, FEA_LS_NSTATE = 8, 8
(FEA_LS_DE, FEA_LS_E0, FEA_LS_SMAX, FEA_LS_SIGN, FEA_LS_ALPHA, FEA_LS_ENEW, FEA_LS_FOUND, FEA_LS_ROUND) = range(8)
fea_adjoint_vjp_volume = _sig("fea_adjoint_vjp_volume", I32, NP, GP, D, D, P, P, P, P, P, I64, P)
fea_adjoint_hvp_pressure = _sig("fea_adjoint_hvp_pressure", I32, NP, GP, D, P, P, P, P, P)
fea_version = _sig("fea_version", I32)
fea_launch_count = _sig("fea_launch_count", I64)

# every symbol the header declares (checked by the CPU test suite)
EXPORTED = ["fea_plan_build", "fea_plan_free", "fea_plan_get", "fea_assemble_work_len", "fea_assemble_volume", "fea_assemble_pressure",
            "fea_reduce_scratch_len", "fea_energy_volume", "fea_energy_volume_noalloc", "fea_energy_pressure", "fea_lumped_mass",
            "fea_invert_mass", "fea_mass_csr", "fea_axpy", "fea_pcg_work_len", "fea_pcg_solve", "fea_pcg_mixed_work_len",
            "fea_pcg_solve_mixed", "fea_spmv", "fea_spmv_nodes", "fea_pcg_solve_nodes", "fea_pcg_solve_mixed_nodes", "fea_convert_f32", "fea_f32_layout_fill", "fea_pcg_solve_mixed_nodes32", "fea_pcgb_work_len", "fea_pcgb_table_bytes", "fea_pcgb_set", "fea_pcgb_start",
            "fea_pcgb_iterate", "fea_pcgb_state", "fea_explicit_work_len", "fea_explicit_run", "fea_explicit_stage",
            "fea_adjoint_vjp_volume", "fea_adjoint_hvp_pressure", "fea_version", "fea_launch_count",
            "fea_ls_ladder_len", "fea_ls_scratch_len", "fea_ls_prepare", "fea_ls_energy_volume",
            "fea_ls_energy_pressure", "fea_ls_select"]
