"""ctypes binding of libmatops_b200.so (the C ABI declared in include/matops_b200.h).

The library is built in-tree by matops_b200/build.py.  There is no fallback: if the
shared library is missing or cannot be loaded, importing the bindings raises.
"""
from __future__ import annotations

import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmatops_b200.so")


class MoMatrix(ctypes.Structure):
    """mo_matrix: device column-major view (data, rows, cols, ld)."""
    _fields_ = [("data", ctypes.c_void_p), ("rows", ctypes.c_int64),
                ("cols", ctypes.c_int64), ("ld", ctypes.c_int64)]


class MoProfile(ctypes.Structure):
    """mo_profile: per-class launches, device ms, algorithmic flops and bytes."""
    _fields_ = [("launches", ctypes.c_int64 * 9), ("ms", ctypes.c_double * 9),
                ("flops", ctypes.c_double * 9), ("bytes", ctypes.c_double * 9)]


class MoIRInfo(ctypes.Structure):
    """mo_ir_info: outcome of mo_dsposv_ir."""
    _fields_ = [("iters", ctypes.c_int), ("gmres_iters", ctypes.c_int),
                ("converged", ctypes.c_int), ("fallback", ctypes.c_int),
                ("shifts", ctypes.c_int), ("method", ctypes.c_int), ("abandoned", ctypes.c_int),
                ("prec", ctypes.c_int),
                ("berr", ctypes.c_double), ("shift", ctypes.c_double),
                ("history", ctypes.c_double * 32)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m matops_b200.build` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    i, d, p, i64, sz = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64, ctypes.c_size_t
    M = MoMatrix
    sigs = {
        "mo_ctx_create": [i, ctypes.POINTER(p)],
        "mo_ctx_destroy": [p],
        "mo_set_stream": [p, p],
        "mo_sync": [p],
        "mo_blocking_params": [p, i, i, i],
        "mo_num_workers": [p, i],
        "mo_set_syrk_blas_beta": [p, i],
        "mo_set_spin_limit": [p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)],
        "mo_mult_sym": [p, M, M, M, d, d, i],
        "mo_mult_trm": [p, M, M, d, i],
        "mo_rank_update2_sym": [p, M, M, M, d, d, i],
        "mo_update_trm": [p, M, M, M, d, d, i],
        "mo_inverse_trm": [p, M, i, i],
        "mo_decompose_qrt": [p, M, M, M, i],
        "mo_decompose_qr": [p, M, M, M, i],
        "mo_build_t": [p, M, M, M],
        "mo_mult_qt": [p, M, M, M, M, i, i],
        "mo_mult_q": [p, M, M, M, M, i, i],
        "mo_solve_qrt": [p, M, M, M, M, i, i],
        "mo_solve_qr": [p, M, M, M, M, i, i],
        "mo_decompose_ldl_nopiv": [p, M, M, i, i],
        "mo_solve_ldl_nopiv": [p, M, M, i],
        "mo_decompose_ldl": [p, M, M, p, i64, i, i],
        "mo_solve_ldl": [p, M, M, p, i64, i],
        "mo_decompose_bk": [p, M, M, p, i64, i, i],
        "mo_solve_bk": [p, M, M, p, i64, i],
        "mo_build_q": [p, M, M, M, i],
        "mo_build_qt": [p, M, M, M, i],
        "mo_mirror_create": [p, p, i64, ctypes.POINTER(p)],
        "mo_mirror_destroy": [p],
        "mo_mirror_find": [p, ctypes.POINTER(p), ctypes.POINTER(i64)],
        "mo_mirror_view": [p, p, i64, i64, i64, i, ctypes.POINTER(M)],
        "mo_mirror_to_host": [p],
        "mo_mirror_host_modified": [p],
        "mo_mirror_state": [p],
        "mo_malloc": [p, ctypes.POINTER(p), sz],
        "mo_free": [p, p],
        "mo_upload": [p, M, p, i64],
        "mo_upload_tri": [p, M, p, i64, i],
        "mo_download": [p, p, i64, M],
        "mo_upload_bytes": [p, p, p, sz],
        "mo_download_bytes": [p, p, p, sz],
        "mo_mult": [p, M, M, M, d, d, i],
        "mo_rank_update_sym": [p, M, M, d, d, i],
        "mo_solve_trm": [p, M, M, d, i],
        "mo_decompose_chol": [p, M, i, i, ctypes.POINTER(d)],
        "mo_solve_chol": [p, M, M, i],
        "mo_decompose_lu": [p, M, p, i64, i],
        "mo_solve_lu": [p, M, M, p, i64, i],
        "mo_profile_enable": [p, i],
        "mo_profile_read": [p, ctypes.POINTER(MoProfile)],
        "mo_measure_fp64_peak": [p, d, ctypes.POINTER(d)],
        "mo_solve_trm_static": [M, M, d, i, p],
        "mo_dsposv_ir": [p, M, M, M, i, i, i, d, i, ctypes.POINTER(MoIRInfo)],
        "mo_decompose_chol_adjoint": [p, M, M, i],
        "mo_decompose_chol_adjoint_batched": [p, i, p, p, i],
        "mo_solve_chol_adjoint": [p, M, M, M, M, i],
        "mo_batch_create": [p, i, i, p, i, ctypes.POINTER(p)],
        "mo_batch_destroy": [p],
        "mo_batch_run": [p, p, p, p, p, p, p],
        "mo_batch_tune": [p, i, p],
        "mo_batch_schedule": [p, p, i],
        "mo_lp_gemm": [p, i, i64, i64, i64, ctypes.c_float, p, i64, p, i64, ctypes.c_float, p,
                       i64, i],
    }
    for name, args in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = i
    L.mo_strerror.argtypes = [i]
    L.mo_strerror.restype = ctypes.c_char_p
    _lib = L
    return L
