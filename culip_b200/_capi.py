"""ctypes bindings of libculipx (include/culipx.h).

The library is loaded from culip_b200/lib/libculipx.so (built in-tree by
culip_b200/build.py).  There is no fallback: if the library is missing or
fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libculipx.so")

OK, INVALID_ARG, OOM, BREAKDOWN, MAXIT, TIMEOUT, CUDA_ERROR, NOT_SUPPORTED, PENDING, STALLED = range(10)
F64, F32 = 0, 1
PIV_STATIC, PIV_BK, PIV_ROOK = 0, 1, 2
LEFT, MIDDLE, RIGHT = 0, 1, 2
SOLVE_STRIPE, SOLVE_BLOCK, SOLVE_SCALAR, SOLVE_JACOBI = 0, 1, 2, 3
FMT_CSR, FMT_SELL = 0, 1

STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "BREAKDOWN", 4: "MAXIT", 5: "TIMEOUT", 6: "CUDA_ERROR",
                7: "NOT_SUPPORTED", 8: "PENDING", 9: "STALLED"}


class CulipxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class KktSpec(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("m", ctypes.c_int), ("nnz_per_col", ctypes.c_int), ("band_half", ctypes.c_int),
                ("hmin", ctypes.c_double), ("hmax", ctypes.c_double), ("delta", ctypes.c_double),
                ("gamma", ctypes.c_double), ("seed", ctypes.c_ulonglong)]


vp = ctypes.c_void_p
i32 = ctypes.c_int
i64 = ctypes.c_longlong
f64 = ctypes.c_double

# name -> argtypes (restype int unless listed)
_SIGS = {
    "culipx_version": [],
    "culipx_kkt_nnz": [ctypes.POINTER(KktSpec), ctypes.POINTER(i64)],
    "culipx_kkt_generate": [ctypes.POINTER(KktSpec), vp, vp, vp],
    "culipx_kkt_blocking": [i32, i32, i32, vp, i32, ctypes.POINTER(i32)],
    "culipx_blocking_generate": [i32, vp, vp, i32, i32, vp, i32, ctypes.POINTER(i32)],
    "culipx_normal_vector": [ctypes.c_ulonglong, i64, vp],
    "culipx_handle_create": [ctypes.POINTER(vp), i32, vp],
    "culipx_handle_destroy": [vp],
    "culipx_handle_set_stream": [vp, vp],
    "culipx_handle_set_memory_budget": [vp, i64],
    "culipx_handle_memory_used": [vp, ctypes.POINTER(i64)],
    "culipx_handle_synchronize": [vp],
    "culipx_handle_launch_count": [vp, ctypes.POINTER(i64), i32],
    "culipx_pattern_analyze": [vp, i32, vp, vp, i32, vp, i32, f64, i32, ctypes.POINTER(vp)],
    "culipx_pattern_analyze_systems": [vp, i32, vp, vp, i32, vp, i32, f64, i32, i32, vp, ctypes.POINTER(vp)],
    "culipx_pattern_destroy": [vp],
    "culipx_pattern_info": [vp, vp],
    "culipx_pattern_export": [vp] * 12,
    "culipx_factor_create": [vp, ctypes.POINTER(vp)],
    "culipx_factor_destroy": [vp],
    "culipx_factor_compute": [vp, vp, vp, i32, f64],
    "culipx_factor_compute_host": [vp, vp, vp, i32, f64],
    "culipx_factor_export_size": [vp, ctypes.POINTER(i64)],
    "culipx_factor_export": [vp] * 9,
    "culipx_factor_stats": [vp, ctypes.POINTER(f64), ctypes.POINTER(i32)],
    "culipx_factor_info": [vp, vp],
    "culipx_prec_apply": [vp, i32, vp, vp],
    "culipx_factor_set_solve_algorithm": [vp, i32, i32],
    "culipx_factor_set_pivot_fp64": [vp, f64],
    "culipx_permute_create": [vp, i32, i64, vp, vp, vp, vp, i32, ctypes.POINTER(vp)],
    "culipx_permute_destroy": [vp],
    "culipx_permute_structure": [vp, ctypes.POINTER(vp), ctypes.POINTER(vp)],
    "culipx_permute_apply": [vp, i32, vp, vp, vp, i32, vp],
    "culipx_permute_export": [vp, vp, vp],
    "culipx_csr_create": [vp, i32, i32, i64, vp, vp, vp, i32, i32, ctypes.POINTER(vp)],
    "culipx_csr_destroy": [vp],
    "culipx_spmv": [vp, vp, vp, f64, f64, i32],
    "culipx_batch_factor_solve_graph": [vp, vp, vp, vp, i32, f64, vp, vp, f64, i32, vp, vp, vp],
    "culipx_sprank": [i32, i32, vp, vp, vp, vp, ctypes.POINTER(i32)],
    "culipx_ordering_rcm": [i32, vp, vp, vp],
    "culipx_kkt_assembly_create": [vp, i32, i32, i64, vp, vp, ctypes.POINTER(vp)],
    "culipx_kkt_assembly_destroy": [vp],
    "culipx_kkt_assembly_size": [vp, ctypes.POINTER(i32), ctypes.POINTER(i64)],
    "culipx_kkt_assembly_structure": [vp, ctypes.POINTER(vp), ctypes.POINTER(vp)],
    "culipx_kkt_assembly_export": [vp, vp, vp],
    "culipx_kkt_assemble": [vp, vp, vp, vp, vp, f64, f64, i32, vp],
    "culipx_csr_set_format": [vp, i32],
    "culipx_csr_refresh": [vp],
    "culipx_sqmr_solve": [vp, vp, vp, vp, vp, f64, i32, ctypes.POINTER(f64), ctypes.POINTER(i32)],
    "culipx_sqmr_solve_noalloc": [vp, vp, vp, vp, vp, f64, i32, ctypes.POINTER(f64), ctypes.POINTER(i32)],
    "culipx_vec_dot": [vp, i32, i64, vp, vp, ctypes.POINTER(f64)],
    "culipx_vec_nrm2": [vp, i32, i64, vp, ctypes.POINTER(f64)],
    "culipx_vec_axpy": [vp, i32, i64, f64, vp, vp],
    "culipx_vec_scal": [vp, i32, i64, f64, vp],
    "culipx_vec_convert": [vp, i64, i32, vp, i32, vp],
    "culipx_batch_create": [vp, i32, vp, ctypes.POINTER(vp)],
    "culipx_batch_destroy": [vp],
    "culipx_batch_sqmr_solve": [vp, vp, vp, vp, vp, f64, i32, vp, vp, vp],
    "culipx_sqmr_solve_multi": [vp, vp, vp, i32, vp, vp, f64, i32, vp, vp, vp],
    "culipx_sqmr_refine_multi": [vp, vp, vp, i32, vp, vp, f64, f64, i32, i32, vp, vp, vp, vp],
    "culipx_sqmr_solve_many": [vp, i32, vp, vp, vp, vp, f64, i32, vp, vp, vp],
    "culipx_server_create": [i32, i64, i32, i32, f64, i32, ctypes.POINTER(vp)],
    "culipx_server_destroy": [vp],
    "culipx_server_add_pattern": [vp, i32, vp, vp, i32, vp, i32, ctypes.POINTER(i32)],
    "culipx_server_submit": [vp, i32, vp, i32, vp, ctypes.POINTER(i32)],
    "culipx_server_progress": [vp, i32, ctypes.POINTER(i32)],
    "culipx_server_result": [vp, i32, vp, vp, vp, ctypes.POINTER(f64)],
    "culipx_server_release": [vp, i32],
    "culipx_server_stats": [vp, vp],
    "culipx_server_set_large_rows": [vp, i32],
    "culipx_server_launch_count": [vp, vp],
    "culipx_server_set_refine": [vp, i32, f64],
    "culipx_factor_compute_graph": [vp, vp, i32, f64],
    "culipx_ldu_create": [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp],
    "culipx_ldu_apply": [vp, i32, vp, vp],
    "culipx_sqmr_solve_ldu": [vp, vp, vp, vp, vp, f64, i32, vp, vp],
    "culipx_ldu_destroy": [vp],
    "culipx_kkt_operator_create": [vp, i32, i32, i32, ctypes.c_longlong, vp, vp, vp, vp, f64, i32, vp, vp],
    "culipx_kkt_operator_multiply": [vp, vp, vp, f64, f64],
    "culipx_kkt_operator_destroy": [vp],
    "culipx_tune_kkt_block": [vp, i32, i32, vp, vp, vp, vp, i32, vp, i32, f64, i32, vp, vp, vp, vp, vp],
    "culipx_batch_sqmr_refine": [vp, vp, vp, vp, vp, f64, f64, i32, i32, vp, vp, vp, vp],
    "culipx_sqmr_refine": [vp, vp, vp, vp, vp, f64, f64, i32, i32, ctypes.POINTER(f64), ctypes.POINTER(i32),
                           ctypes.POINTER(i32)],
    "culipx_sqmr_profile": [vp, i32],
    "culipx_sqmr_set_wait_skew": [vp, ctypes.c_ulonglong],
    "culipx_sqmr_phase_times": [vp, vp, i32],
}

_lib = None


def load():
    """Loads libculipx.so; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python culip_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        L.culipx_last_error.restype = ctypes.c_char_p
        L.culipx_last_error.argtypes = []
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    return ["culipx_last_error", *_SIGS.keys()]


def check(status: int, allow=(OK,)) -> int:
    if status not in allow:
        msg = load().culipx_last_error().decode(errors="replace")
        raise CulipxError(status, msg)
    return status


def call(name: str, *args, allow=(OK,)) -> int:
    return check(getattr(load(), name)(*args), allow)
