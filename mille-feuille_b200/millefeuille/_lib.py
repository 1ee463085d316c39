"""ctypes binding of libmillefeuille.so (the C ABI in include/millefeuille.h).

The library is built in-tree (mille-feuille_b200/build.py).  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# MILLEFEUILLE_LIB selects another build of the same ABI, e.g. the
# bounds-checked libmillefeuille_check.so (build.py --check)
LIB_PATH = os.environ.get("MILLEFEUILLE_LIB") or os.path.join(HERE, "libmillefeuille.so")
LIB_CHECK_PATH = os.path.join(HERE, "libmillefeuille_check.so")
# the same library with cg_solve_inc in FP64 (main-cg.cu's entry point)
LIB_FP64_PATH = os.path.join(HERE, "libmillefeuille_fp64.so")

MF_SUCCESS, MF_ERR_INVALID, MF_ERR_CUDA, MF_ERR_NOMEM, MF_ERR_TIMEOUT = 0, 1, 2, 3, 4
MF_ERR_UNSUPPORTED, MF_ERR_BREAKDOWN, MF_ERR_IO, MF_ERR_NOT_BUILT, MF_ERR_CHECK = 5, 6, 7, 8, 9
MF_METHOD_CG, MF_METHOD_BICGSTAB = 0, 1
MF_PREC_FP64, MF_PREC_MIXED, MF_PREC_PARITY = 0, 1, 2


class MFError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: [{status}] {status_string(status)}" if what else status_string(status))


class Options(C.Structure):
    _fields_ = [("method", C.c_int), ("precision", C.c_int), ("tol", C.c_double), ("max_iter", C.c_int),
                ("fixed_iters", C.c_int), ("replace_every", C.c_int), ("demote_fp16", C.c_double),
                ("demote_int8", C.c_double), ("use_lossless", C.c_int), ("wait_timeout_s", C.c_double),
                ("blocks_per_sm", C.c_int), ("threads_per_block", C.c_int), ("x0_given", C.c_int),
                ("l2_window", C.c_int), ("test_stall_barrier", C.c_int), ("demote_min_fraction", C.c_double),
                ("relax_eta", C.c_double), ("relax_int8", C.c_int), ("test_check_limit", C.c_int)]


class Report(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("converged", C.c_int),
                ("relres_true", C.c_double), ("relres_rec", C.c_double), ("residual", C.c_double),
                ("time_ms", C.c_double), ("replacements", C.c_int), ("grid_blocks", C.c_int),
                ("threads_per_block", C.c_int), ("tile_uses", C.c_longlong * 4), ("tiles_skipped", C.c_longlong),
                ("nnz_uses", C.c_longlong * 4), ("phase_ms", C.c_double * 6), ("host_ms", C.c_double * 4)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_
             if k not in ("tile_uses", "nnz_uses", "phase_ms", "host_ms")}
        d["host_ms"] = dict(zip(("stage_h2d", "prepare", "launch_to_readback", "d2h_sync"),
                                [round(v, 4) for v in self.host_ms]))
        d["tile_uses"] = list(self.tile_uses)
        d["nnz_uses"] = list(self.nnz_uses)
        d["phase_ms"] = dict(zip(("spmv", "vec_update", "dir_update", "barrier", "replacement", "barrier_spin"),
                                 [round(v, 4) for v in self.phase_ms]))
        return d


class MatrixInfo(C.Structure):
    _fields_ = [("n_rows", C.c_int), ("n_cols", C.c_int), ("nnz", C.c_longlong), ("tilem", C.c_int),
                ("tilen", C.c_int), ("tilenum", C.c_int), ("csrsize", C.c_int), ("csrptrlen", C.c_int),
                ("cnt_non_new", C.c_int), ("rowblkblock", C.c_int), ("nseg", C.c_int),
                ("slice_entries", C.c_longlong), ("build_ms", C.c_double), ("device", C.c_int)]


class CgBenchResult(C.Structure):
    _fields_ = [("time_ms", C.c_double), ("iterations", C.c_int), ("l2_norm", C.c_double),
                ("residual", C.c_double)]


# Every symbol the header declares (the CPU test checks they are all exported).
EXPORTED = [
    "mf_status_string", "cg_solve_inc", "cg_solve_sync", "cg_solve_reduce", "bicgstab", "bicgstab_sync",
    "bicgstab_inc", "mf_read_matrix", "mf_write_cbd", "mf_free_host", "mf_options_default", "mf_matrix_create",
    "mf_matrix_destroy", "mf_matrix_get_info", "mf_tile_array_bytes", "mf_tile_export", "mf_solve", "mf_spmv",
    "mf_debug_ref_labels", "mf_build_arch", "mf_spmv_noalloc", "mf_value_grad", "mf_matrix_create_transposed",
    "mf_solve_multi", "mf_batch_create", "mf_batch_tune", "mf_batch_configure", "mf_batch_config",
    "mf_batch_solve", "mf_batch_destroy",
    "mf_batch_partition", "mf_batch_schedule", "mf_debug_spmv_tiles", "mf_debug_solver_labels",
    "mf_dropin_last_report", "mf_debug_spmm",
]

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libmillefeuille.so not built at {LIB_PATH}; run mille-feuille_b200/build.py")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp, fp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_float)
    L.mf_status_string.argtypes = [C.c_int]
    L.mf_status_string.restype = C.c_char_p
    L.mf_build_arch.restype = C.c_char_p
    L.mf_options_default.argtypes = [C.POINTER(Options)]
    L.mf_matrix_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.c_longlong, vp, vp, vp, vp, C.c_int, vp]
    L.mf_matrix_destroy.argtypes = [vp]
    L.mf_matrix_get_info.argtypes = [vp, C.POINTER(MatrixInfo)]
    L.mf_tile_array_bytes.argtypes = [vp, C.c_char_p, C.POINTER(C.c_size_t)]
    L.mf_tile_export.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
    L.mf_solve.argtypes = [vp, vp, vp, C.POINTER(Options), C.POINTER(Report), C.c_int, vp]
    L.mf_spmv.argtypes = [vp, vp, vp, C.c_int, C.c_int, vp, dp]
    L.mf_spmv_noalloc.argtypes = [vp, vp, vp, C.c_int, vp]
    L.mf_value_grad.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, vp]
    L.mf_solve_multi.argtypes = [vp, C.c_int, vp, vp, C.POINTER(Options), C.POINTER(Report), C.c_int, vp]
    L.mf_batch_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp), C.POINTER(C.c_int), vp]
    L.mf_batch_tune.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int), vp]
    L.mf_batch_configure.argtypes = [vp, C.c_int, C.c_int, vp]
    L.mf_batch_config.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.mf_batch_solve.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(Options), C.POINTER(Report), C.c_int,
                                 vp]
    L.mf_batch_destroy.argtypes = [vp]
    L.mf_batch_partition.argtypes = [C.c_int, ip, C.POINTER(C.c_longlong), ip, C.c_int, C.c_int, ip, dp]
    L.mf_batch_schedule.argtypes = [C.c_int, dp, ip, C.c_int, ip, ip, ip, ip, ip]
    L.mf_matrix_create_transposed.argtypes = [C.POINTER(vp), vp, vp]
    L.mf_debug_ref_labels.argtypes = [vp, vp, C.c_int, vp, C.c_int]
    L.mf_debug_spmv_tiles.argtypes = [vp, vp, vp, C.c_int, C.c_int]
    L.mf_debug_solver_labels.argtypes = [vp, vp, C.c_int]
    L.mf_dropin_last_report.argtypes = [C.POINTER(Report)]
    L.mf_debug_spmm.argtypes = [vp, vp, vp, C.c_int, C.c_int, dp]
    L.mf_read_matrix.argtypes = [C.c_char_p, ip, ip, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(dp), ip]
    L.mf_write_cbd.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, vp, vp, vp]
    L.mf_free_host.argtypes = [vp]
    cg_args = [ip, ip, dp, fp, dp, dp, C.c_int, ip, C.c_int, C.c_double, C.c_char_p, C.c_int, C.c_int, C.c_int,
               C.POINTER(CgBenchResult), C.c_int]
    for name in ("cg_solve_inc", "cg_solve_sync", "cg_solve_reduce"):
        getattr(L, name).argtypes = cg_args
        getattr(L, name).restype = None
    for name in ("bicgstab", "bicgstab_sync", "bicgstab_inc"):
        getattr(L, name).argtypes = [ip, ip, dp, dp, dp, C.c_int, C.c_char_p, C.c_int]
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def status_string(status: int) -> str:
    try:
        return load().mf_status_string(int(status)).decode()
    except Exception:
        return f"status {status}"


def check(status: int, what: str = "") -> None:
    if status != MF_SUCCESS:
        raise MFError(status, what)
