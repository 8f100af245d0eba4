"""Oracle for the GLU numeric path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package.  It checks results and is never the thing measured or shipped.

Two parts:

* ``_bin/liboracle.so`` -- a plain-C restatement of the reference's numeric
  algorithm (glu_oracle.c): the right-looking column factorization of
  src/numeric.cu:36-89 / 204-345 run sequentially in level order, in FP32 and
  FP64; the triangular solve of src/symbolic.cc:200-251; the levelling of
  src/symbolic.cc:106-151; the fill-in of src/symbolic.cc:11-53; transposed
  solves, an FP64 CSC SpMV and FP64 iterative refinement for the new
  capabilities.
* ``_ref/libglu_ref.so`` -- the reference's own CPU code (NICSLU, preprocess.c,
  symbolic.cc) compiled from the reference tree by oracle/Makefile, driven
  through ref_harness.cpp.  It pins the restatement: pattern, permutations,
  levels and predictLU values are compared bit-exactly against it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

_ref = None
_orc = None


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libglu_ref.so"))


def _load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(os.path.join(HERE, "_ref", "libglu_ref.so"))
        lib.ref_create.restype = C.c_void_p
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_analyze.argtypes = [C.c_void_p, C.c_uint, C.c_uint, _f64p, _u32p, _u32p]
        lib.ref_analyze.restype = C.c_int
        lib.ref_n.argtypes = [C.c_void_p]
        lib.ref_n.restype = C.c_uint
        lib.ref_nnzA.argtypes = [C.c_void_p]
        lib.ref_nnzA.restype = C.c_uint
        lib.ref_get_dumped.argtypes = [C.c_void_p, _f64p, _u32p, _u32p]
        lib.ref_get_perm.argtypes = [C.c_void_p, _u32p, _u32p, _u32p, _u32p, _f64p, _f64p,
                                     _i32p, _i32p, C.POINTER(C.c_uint)]
        lib.ref_set_csc.argtypes = [C.c_void_p, C.c_uint, C.c_uint, _f64p, _u32p, _u32p]
        lib.ref_symbolic.argtypes = [C.c_void_p]
        lib.ref_lu_nnz.argtypes = [C.c_void_p]
        lib.ref_lu_nnz.restype = C.c_uint
        lib.ref_num_lev.argtypes = [C.c_void_p]
        lib.ref_num_lev.restype = C.c_int
        lib.ref_get_symbolic.argtypes = [C.c_void_p, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p,
                                         _f32p, _i32p, _i32p]
        lib.ref_solve.argtypes = [C.c_void_p, _f32p, _f32p, _f32p]
        lib.ref_set_val.argtypes = [C.c_void_p, _f32p]
        lib.ref_get_val.argtypes = [C.c_void_p, _f32p]
        lib.ref_nicslu_create.restype = C.c_void_p
        lib.ref_nicslu_create.argtypes = [C.c_uint, C.c_uint, _f64p, _u32p, _u32p, C.c_uint,
                                          _f64p, C.POINTER(C.c_int)]
        lib.ref_nicslu_threads.argtypes = [C.c_void_p]
        lib.ref_nicslu_threads.restype = C.c_uint
        lib.ref_nicslu_refactor.argtypes = [C.c_void_p, _f64p, C.c_uint, C.POINTER(C.c_double)]
        lib.ref_nicslu_solve.argtypes = [C.c_void_p, _f64p, C.POINTER(C.c_double)]
        lib.ref_nicslu_refine.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double, C.c_uint]
        lib.ref_nicslu_lu_nnz.argtypes = [C.c_void_p]
        lib.ref_nicslu_lu_nnz.restype = C.c_size_t
        lib.ref_nicslu_destroy.argtypes = [C.c_void_p]
        _ref = lib
    return _ref


class RefGLU:
    """The reference's preprocessing + symbolic phase on one matrix."""

    def __init__(self, data, indices, indptr, n, preprocessed=False):
        lib = _load_ref()
        self._lib = lib
        self._h = lib.ref_create()
        ax = np.ascontiguousarray(data, dtype=np.float64)
        ai = np.ascontiguousarray(indices, dtype=np.uint32)
        ap = np.ascontiguousarray(indptr, dtype=np.uint32)
        if preprocessed:
            lib.ref_set_csc(self._h, n, ax.size, ax, ai, ap)
            self.perm = None
        else:
            ret = lib.ref_analyze(self._h, n, ax.size, ax, ai, ap)
            if ret != 0:
                raise RuntimeError(f"reference preprocessing failed ({ret})")
            n = lib.ref_n(self._h)
            nz = lib.ref_nnzA(self._h)
            self.ax = np.empty(nz, np.float64)
            self.ai = np.empty(nz, np.uint32)
            self.ap = np.empty(n + 1, np.uint32)
            lib.ref_get_dumped(self._h, self.ax, self.ai, self.ap)
            p = {k: np.empty(n, np.uint32) for k in ("row_perm", "row_perm_inv", "col_perm", "col_perm_inv")}
            rs = np.empty(n, np.float64)
            cs = np.empty(n, np.float64)
            piv = np.empty(n, np.int32)
            pinv = np.empty(n, np.int32)
            flag = C.c_uint(0)
            lib.ref_get_perm(self._h, p["row_perm"], p["row_perm_inv"], p["col_perm"],
                             p["col_perm_inv"], rs, cs, piv, pinv, C.byref(flag))
            p.update(row_scale=rs, col_scale_perm=cs, pivot=piv, pivot_inv=pinv, mc64=int(flag.value))
            self.perm = p
        self.n = n
        self._sym = False

    def symbolic(self):
        lib = self._lib
        lib.ref_symbolic(self._h)
        n = self.n
        nnz = lib.ref_lu_nnz(self._h)
        nlev = lib.ref_num_lev(self._h)
        s = dict(sym_c_ptr=np.empty(n + 1, np.uint32), sym_r_idx=np.empty(nnz, np.uint32),
                 l_col_ptr=np.empty(n, np.uint32), csr_r_ptr=np.empty(n + 1, np.uint32),
                 csr_c_idx=np.empty(nnz, np.uint32), csr_diag_ptr=np.empty(n, np.uint32),
                 val=np.empty(nnz, np.float32), level_ptr=np.empty(nlev + 1, np.int32),
                 level_idx=np.empty(n, np.int32))
        lib.ref_get_symbolic(self._h, s["sym_c_ptr"], s["sym_r_idx"], s["l_col_ptr"],
                             s["csr_r_ptr"], s["csr_c_idx"], s["csr_diag_ptr"], s["val"],
                             s["level_ptr"], s["level_idx"])
        s["nnz"] = nnz
        s["num_lev"] = nlev
        self._sym = True
        self.sym = s
        return s

    def solve(self, luval, rhs):
        """Symbolic_Matrix::solve (FP32) with the given factor values."""
        x = np.empty(self.n, np.float32)
        self._lib.ref_solve(self._h, np.ascontiguousarray(luval, np.float32),
                            np.ascontiguousarray(rhs, np.float32), x)
        return x

    def __del__(self):
        try:
            self._lib.ref_destroy(self._h)
        except Exception:
            pass


class RefNicsLU:
    """NICSLU's own multi-threaded CPU factor / refactor / solve (the CPU baseline)."""

    def __init__(self, data, indices, indptr, n, threads):
        lib = _load_ref()
        self._lib = lib
        self.n = n
        self.threads = threads
        t = np.zeros(2)
        st = C.c_int(0)
        self._keep = (np.ascontiguousarray(data, np.float64), np.ascontiguousarray(indices, np.uint32),
                      np.ascontiguousarray(indptr, np.uint32))
        self._h = lib.ref_nicslu_create(n, data.size, *self._keep, threads, t, C.byref(st))
        if st.value != 0:
            raise RuntimeError(f"NICSLU factorization failed ({st.value})")
        self.t_analyze, self.t_factor = float(t[0]), float(t[1])
        self.threads_created = lib.ref_nicslu_threads(self._h)

    def refactor(self, data):
        t = C.c_double(0)
        ret = self._lib.ref_nicslu_refactor(self._h, np.ascontiguousarray(data, np.float64),
                                            self.threads, C.byref(t))
        if ret != 0:
            raise RuntimeError(f"NICSLU refactor failed ({ret})")
        return t.value

    def solve(self, b):
        x = np.array(b, dtype=np.float64, copy=True)
        t = C.c_double(0)
        ret = self._lib.ref_nicslu_solve(self._h, x, C.byref(t))
        if ret != 0:
            raise RuntimeError(f"NICSLU solve failed ({ret})")
        return x

    def refine(self, x, b, eps=1e-12, maxiter=10):
        x = np.ascontiguousarray(x, np.float64)
        self._lib.ref_nicslu_refine(self._h, x, np.ascontiguousarray(b, np.float64), eps, maxiter)
        return x

    def lu_nnz(self):
        return int(self._lib.ref_nicslu_lu_nnz(self._h))

    def __del__(self):
        try:
            self._lib.ref_nicslu_destroy(self._h)
        except Exception:
            pass


# ---------------------------------------------------------------------------
# The C restatement (liboracle.so)
def _load_orc():
    global _orc
    if _orc is None:
        path = os.path.join(HERE, "_bin", "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-C", HERE, "-s"], check=True)
        lib = C.CDLL(path)
        pat = [C.c_uint, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p, C.c_int, _i32p, _i32p]
        lib.orc_factor_f32.argtypes = pat + [_f32p, C.c_float]
        lib.orc_factor_f64.argtypes = pat + [_f64p, C.c_double]
        lib.orc_pert.argtypes = [C.c_uint, _u32p, _f32p]
        lib.orc_pert.restype = C.c_float
        lib.orc_solve_f32.argtypes = [C.c_uint, _u32p, _u32p, _u32p, _f32p, _u32p, _u32p, _i32p, _f64p, _f64p,
                                      C.c_int, _f32p, _f32p]
        lib.orc_sweeps_f32.argtypes = [C.c_uint, _u32p, _u32p, _u32p, _f32p, _f32p, C.c_int]
        lib.orc_sweeps_f64.argtypes = [C.c_uint, _u32p, _u32p, _u32p, _f64p, _f64p, C.c_int]
        lib.orc_leveling.argtypes = [C.c_uint, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p, _i32p, _i32p]
        lib.orc_leveling.restype = C.c_int
        lib.orc_fill_in.argtypes = [C.c_uint, _u32p, _u32p, C.c_uint, _u32p, _u32p, _u32p]
        lib.orc_fill_in.restype = C.c_uint
        _orc = lib
    return _orc


def _pat_args(p):
    return (p["sym_c_ptr"], p["sym_r_idx"], p["l_col_ptr"], p["csr_r_ptr"], p["csr_c_idx"], p["csr_diag_ptr"])


def leveling(p):
    """Symbolic_Matrix::leveling restated: (level_ptr, level_idx)."""
    lib = _load_orc()
    n = p["sym_c_ptr"].size - 1
    lp = np.empty(n + 1, np.int32)
    li = np.empty(n, np.int32)
    nl = lib.orc_leveling(n, *_pat_args(p), lp, li)
    return lp[: nl + 1].copy(), li


def factor(p, val, level_ptr, level_idx, dtype=np.float32, pert=0.0):
    """Right-looking column factorization in level order (numeric.cu semantics)."""
    lib = _load_orc()
    n = p["sym_c_ptr"].size - 1
    v = np.array(val, dtype=dtype, copy=True)
    lp = np.ascontiguousarray(level_ptr, np.int32)
    li = np.ascontiguousarray(level_idx, np.int32)
    f = lib.orc_factor_f32 if dtype == np.float32 else lib.orc_factor_f64
    f(n, *_pat_args(p), lp.size - 1, lp, li, v, pert)
    return v


def pert(p, val):
    return float(_load_orc().orc_pert(p["sym_c_ptr"].size - 1, p["sym_c_ptr"], np.ascontiguousarray(val, np.float32)))


def solve(p, val, tr, rhs):
    """Symbolic_Matrix::solve restated (FP32)."""
    lib = _load_orc()
    n = p["sym_c_ptr"].size - 1
    x = np.empty(n, np.float32)
    lib.orc_solve_f32(n, p["sym_c_ptr"], p["sym_r_idx"], p["l_col_ptr"], np.ascontiguousarray(val, np.float32),
                      tr["col_perm"], tr["row_perm_inv"], tr["pivot"], tr["col_scale_perm"], tr["row_scale"],
                      int(tr["mc64"]), np.ascontiguousarray(rhs, np.float32), x)
    return x


def sweeps(p, val, y, trans=False):
    """L then U sweeps (or U^T then L^T) on the permuted system."""
    lib = _load_orc()
    n = p["sym_c_ptr"].size - 1
    if np.asarray(val).dtype == np.float64:
        yy = np.array(y, np.float64, copy=True)
        lib.orc_sweeps_f64(n, p["sym_c_ptr"], p["sym_r_idx"], p["l_col_ptr"], np.ascontiguousarray(val), yy, int(trans))
    else:
        yy = np.array(y, np.float32, copy=True)
        lib.orc_sweeps_f32(n, p["sym_c_ptr"], p["sym_r_idx"], p["l_col_ptr"], np.ascontiguousarray(val, np.float32),
                           yy, int(trans))
    return yy


def fill_in(ap, ai, n, cap=50_000_000):
    """Symbolic_Matrix::fill_in restated (sorted-list merging)."""
    lib = _load_orc()
    cp = np.empty(n + 1, np.uint32)
    ri = np.empty(cap, np.uint32)
    dg = np.empty(n, np.uint32)
    nz = lib.orc_fill_in(n, np.ascontiguousarray(ap, np.uint32), np.ascontiguousarray(ai, np.uint32), cap, cp, ri, dg)
    if nz == 0:
        raise MemoryError("fill-in exceeds the oracle's capacity")
    return cp, ri[:nz].copy(), dg


# ---------------------------------------------------------------------------
# The reference's own GPU numeric factorization (src/numeric.cu LUonDevice),
# built for sm_100a into oracle/_ref/libglu_ref_gpu.so.
_refgpu = None


def ref_gpu_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libglu_ref_gpu.so"))


def _load_ref_gpu():
    global _refgpu
    if _refgpu is None:
        ref = _load_ref()
        ref.ref_load_pattern.argtypes = [C.c_void_p, C.c_uint, C.c_uint, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p,
                                         _f32p, C.c_int, _i32p, _i32p]
        lib = C.CDLL(os.path.join(HERE, "_ref", "libglu_ref_gpu.so"))
        lib.ref_gpu_luondevice.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.POINTER(C.c_float), C.c_char_p,
                                           C.c_int]
        lib.ref_gpu_luondevice.restype = C.c_int
        lib.ref_gpu_copy_span.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_float)]
        lib.ref_gpu_copy_span.restype = C.c_int
        _refgpu = lib
    return _refgpu


def ref_luondevice(pattern, val, level_ptr, level_idx, perturb=False, keep_free_bytes=0, copy_span=None):
    """Run the reference's LUonDevice on the given Symbolic_Matrix arrays.

    Returns (factor values, the reference's own "Total GPU time" in ms, which
    includes its allocations and copies).  keep_free_bytes > 0 holds a ballast
    allocation so that only that much device memory is free during the call
    (bounds the scratch the reference sizes from free memory).  With
    ``copy_span`` a list, the span of the same allocations and copies without
    the factorization (ref_gpu_copy_span) is measured afterwards, with the same
    ballast, and appended to it in ms.
    """
    lib = _load_ref_gpu()
    ref = _load_ref()
    h = ref.ref_create()
    try:
        p = {k: np.ascontiguousarray(pattern[k], np.uint32) for k in
             ("sym_c_ptr", "sym_r_idx", "l_col_ptr", "csr_r_ptr", "csr_c_idx", "csr_diag_ptr")}
        n = p["sym_c_ptr"].size - 1
        nnz = p["sym_r_idx"].size
        lp = np.ascontiguousarray(level_ptr, np.int32)
        li = np.ascontiguousarray(level_idx, np.int32)
        ref.ref_load_pattern(h, n, nnz, p["sym_c_ptr"], p["sym_r_idx"], p["l_col_ptr"], p["csr_r_ptr"],
                             p["csr_c_idx"], p["csr_diag_ptr"], np.ascontiguousarray(val, np.float32),
                             lp.size - 1, lp, li)
        ms = C.c_float(0)
        err = C.create_string_buffer(1024)
        st = lib.ref_gpu_luondevice(h, int(perturb), int(keep_free_bytes), C.byref(ms), err, 1024)
        if st != 0:
            raise RuntimeError(f"reference LUonDevice failed: {err.value.decode(errors='replace')}")
        out = np.empty(nnz, np.float32)
        ref.ref_get_val(h, out)
        if copy_span is not None:
            cs = C.c_float(0)
            if lib.ref_gpu_copy_span(h, int(keep_free_bytes), C.byref(cs)) != 0:
                raise RuntimeError("reference copy span failed")
            copy_span.append(float(cs.value))
        return out, float(ms.value)
    finally:
        ref.ref_destroy(h)
