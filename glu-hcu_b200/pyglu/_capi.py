"""ctypes binding of the C ABI (include/glu_b200.h, include/glu_preprocess.h).

The shared libraries are built in-tree (glu-hcu_b200/lib) by
``make -C glu-hcu_b200/csrc``; there is no fallback implementation, so a
missing library is an ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lib")
ENGINE_PATH = os.path.join(LIB_DIR, "libglu_b200.so")
NICSLU_PATH = os.path.join(LIB_DIR, "libglu_nicslu.so")

GLU_OK = 0
GLU_ERR_ARG = -1
GLU_ERR_CUDA = -2
GLU_ERR_NOMEM = -3
GLU_ERR_SINGULAR = -4
GLU_ERR_TIMEOUT = -5
GLU_ERR_STATE = -6
GLU_ERR_NOT_CONVERGED = -7
GLU_ERR_NO_DEVICE = -8
GLU_ERR_UNSUPPORTED = -9
GLU_HOST = 0
GLU_DEVICE = 1
GLU_INJECT_ALLOC_FAILURES = 1
GLU_INJECT_UNSET_SOLVE_FLAG = 2

# Every symbol the engine exports (checked by the tests against the header).
ENGINE_SYMBOLS = [
    "glu_last_error", "glu_version", "glu_symbolic_analyze", "glu_symbolic_sizes",
    "glu_symbolic_export", "glu_symbolic_slots", "glu_predict_lu", "glu_symbolic_destroy",
    "glu_create", "glu_create_from_pattern", "glu_destroy", "glu_levels", "glu_set_transform",
    "glu_set_source", "glu_load_lu_values", "glu_store_lu_values", "glu_load_source_values",
    "glu_factor", "glu_solve", "glu_solve_transposed", "glu_solve_refined", "glu_get_stats",
    "glu_get_tuning", "glu_set_tuning", "glu_solve_noalloc", "glu_profile_enable", "glu_kernel_times",
    "glu_kernel_kind_name", "glu_measure_fp32_peak", "glu_set_wait_limit", "glu_debug_inject",
    "glu_factor_many", "glu_solve_refined_many",
]
GLU_KERNEL_KINDS = 16
PRE_SYMBOLS = [
    "glu_pre_analyze", "glu_pre_n", "glu_pre_nnz", "glu_pre_matrix", "glu_pre_transform",
    "glu_pre_source_map", "glu_pre_destroy", "glu_pre_read_mtx", "glu_pre_free",
]


class GLUError(RuntimeError):
    """A failed engine call; ``status`` is the glu_status code."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class SingularMatrixError(GLUError):
    """A zero or non-finite pivot was met during factorization."""


class NotConvergedError(GLUError):
    """Iterative refinement stopped above its tolerance."""


class RefineStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("residual", C.c_double), ("residual_inf", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("n", C.c_uint32), ("nnz_lu", C.c_uint32), ("batch", C.c_uint32), ("num_lev", C.c_int32),
                ("wide_levels", C.c_uint32), ("chain_segments", C.c_uint32), ("dense_tail", C.c_uint32),
                ("factor_flops", C.c_double), ("factor_launches", C.c_uint64),
                ("last_factor_ms", C.c_float), ("pert", C.c_float), ("supernodes", C.c_uint32),
                ("sn_levels", C.c_uint32), ("sn_update_flops", C.c_double), ("sn_update_bytes", C.c_double),
                ("sn_panel_bytes", C.c_double), ("sn_sweep_levels", C.c_uint32),
                ("dense_update_bytes", C.c_double), ("dense_update_flops", C.c_double),
                ("solve_launches", C.c_uint64), ("couple_columns", C.c_uint32), ("couple_groups", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("wide_work", C.c_uint32), ("chain_cluster", C.c_uint32), ("group_lanes", C.c_uint32),
                ("dense_tail_min", C.c_uint32), ("dense_tail_max", C.c_uint32), ("solve_thin", C.c_uint32),
                ("solve_cluster", C.c_uint32), ("sn_width", C.c_uint32),
                ("sn_small", C.c_uint32), ("dense_lookahead", C.c_uint32), ("dense_tc_min", C.c_uint32),
                ("dense_rate", C.c_uint32), ("sn_sweep_fused", C.c_uint32),
                ("batch_tile", C.c_uint32), ("defer_tail", C.c_uint32), ("dense_group", C.c_uint32)]


_vp = C.c_void_p
_u32 = C.c_uint32
_pu32 = C.POINTER(C.c_uint32)


def _load(path, what):
    if not os.path.exists(path):
        raise ImportError(f"{what} not built: {path} is missing (run make -C glu-hcu_b200/csrc)")
    return C.CDLL(path)


def load_engine():
    lib = _load(ENGINE_PATH, "GLU engine library")
    lib.glu_last_error.restype = C.c_char_p
    lib.glu_version.restype = C.c_char_p
    sig = {
        "glu_symbolic_analyze": [_u32, _u32, _vp, _vp, C.POINTER(_vp)],
        "glu_symbolic_sizes": [_vp, _pu32, _pu32],
        "glu_symbolic_export": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
        "glu_symbolic_slots": [_vp, _vp],
        "glu_predict_lu": [_vp, _vp, _vp],
        "glu_create": [_vp, C.c_int, _u32, C.POINTER(_vp)],
        "glu_create_from_pattern": [C.c_int, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _u32, C.POINTER(_vp)],
        "glu_levels": [_vp, C.POINTER(C.c_int32), _vp, _vp],
        "glu_set_transform": [_vp, _vp, _vp, _vp, _vp, _vp, C.c_int],
        "glu_set_source": [_vp, _u32, _vp, _vp, _vp, _vp],
        "glu_load_lu_values": [_vp, _u32, _u32, _vp, C.c_int, _vp],
        "glu_store_lu_values": [_vp, _u32, _u32, _vp, C.c_int, _vp],
        "glu_load_source_values": [_vp, _u32, _u32, _vp, C.c_int, _vp],
        "glu_factor": [_vp, _u32, _u32, C.c_int, _vp],
        "glu_solve": [_vp, _u32, _u32, _vp, _vp, C.c_int, _vp],
        "glu_solve_transposed": [_vp, _u32, _u32, _vp, _vp, C.c_int, _vp],
        "glu_solve_refined": [_vp, _u32, _u32, _u32, _vp, _vp, C.c_double, _u32, C.c_int, C.c_int,
                              C.POINTER(RefineStats), _vp],
        "glu_get_stats": [_vp, C.POINTER(Stats)],
        "glu_get_tuning": [_vp, C.POINTER(Tuning)],
        "glu_set_tuning": [_vp, C.POINTER(Tuning)],
        "glu_solve_noalloc": [_vp, _u32, _u32, _vp, _vp, _vp],
        "glu_profile_enable": [_vp, C.c_int],
        "glu_kernel_times": [_vp, _vp, _vp],
        "glu_measure_fp32_peak": [C.c_int, C.POINTER(C.c_double)],
        "glu_set_wait_limit": [_vp, _u32],
        "glu_debug_inject": [_vp, C.c_int, _u32],
        "glu_factor_many": [_u32, _vp, C.c_int, _vp, _u32],
        "glu_solve_refined_many": [_u32, _vp, _vp, _vp, _vp, C.c_double, _u32, C.c_int,
                                   C.POINTER(RefineStats), _vp, _u32],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.glu_symbolic_destroy.argtypes = [_vp]
    lib.glu_symbolic_destroy.restype = None
    lib.glu_destroy.argtypes = [_vp]
    lib.glu_destroy.restype = None
    lib.glu_kernel_kind_name.argtypes = [C.c_int]
    lib.glu_kernel_kind_name.restype = C.c_char_p
    return lib


def kernel_times(handle):
    """{kernel kind: (ms, launches)} of the last profiled glu_factor call."""
    lib = engine()
    ms = np.zeros(GLU_KERNEL_KINDS, np.float32)
    n = np.zeros(GLU_KERNEL_KINDS, np.uint32)
    check(lib.glu_kernel_times(handle, ptr(ms), ptr(n)), "kernel times")
    return {lib.glu_kernel_kind_name(k).decode(): (float(ms[k]), int(n[k])) for k in range(GLU_KERNEL_KINDS)}


def load_preprocess():
    lib = _load(NICSLU_PATH, "NICSLU preprocessing library")
    lib.glu_pre_analyze.argtypes = [_u32, _u32, _vp, _vp, _vp, C.POINTER(_vp)]
    lib.glu_pre_analyze.restype = C.c_int
    lib.glu_pre_n.argtypes = [_vp]
    lib.glu_pre_n.restype = _u32
    lib.glu_pre_nnz.argtypes = [_vp]
    lib.glu_pre_nnz.restype = _u32
    lib.glu_pre_matrix.argtypes = [_vp, _vp, _vp, _vp]
    lib.glu_pre_matrix.restype = None
    lib.glu_pre_transform.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_int)]
    lib.glu_pre_transform.restype = None
    lib.glu_pre_source_map.argtypes = [_vp, _vp, _vp]
    lib.glu_pre_source_map.restype = None
    lib.glu_pre_destroy.argtypes = [_vp]
    lib.glu_pre_destroy.restype = None
    lib.glu_pre_read_mtx.argtypes = [C.c_char_p, _pu32, _pu32, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]
    lib.glu_pre_read_mtx.restype = C.c_int
    lib.glu_pre_free.argtypes = [_vp]
    lib.glu_pre_free.restype = None
    return lib


_engine = None
_pre = None


def engine():
    global _engine
    if _engine is None:
        _engine = load_engine()
    return _engine


def pre():
    global _pre
    if _pre is None:
        _pre = load_preprocess()
    return _pre


def check(status, what="GLU call"):
    if status == GLU_OK:
        return
    msg = engine().glu_last_error().decode(errors="replace")
    text = f"{what} failed: {msg}"
    if status == GLU_ERR_ARG:
        raise ValueError(text)
    if status == GLU_ERR_SINGULAR:
        raise SingularMatrixError(status, text)
    if status == GLU_ERR_NOT_CONVERGED:
        raise NotConvergedError(status, text)
    raise GLUError(status, text)


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)
