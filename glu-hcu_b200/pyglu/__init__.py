"""pyglu -- Python interface of the B200 GLU sparse LU engine.

Same surface as the reference's pyglu (pyglu/__init__.py, src/glu_binding.cpp):

    lu = pyglu.splu(A)            # factorize (returns GLUFactorization)
    x  = lu.solve(b)              # solve Ax = b
    x  = pyglu.spsolve(A, b)      # factorize and solve in one call

A is any scipy sparse matrix or a (data, indices, indptr, shape) CSC tuple.
As in the reference, the factors and the plain solve are FP32 (inputs and
outputs are float64, converted at the boundary); unlike the reference the
solve runs on the GPU.  Additions:

* ``lu.solve(b, refine=True, tol=1e-10)`` -- FP64 iterative refinement on the
  GPU (residuals with the original FP64 matrix), reaching FP64-level residuals;
* ``lu.refactor(data)`` -- new values, same pattern, no new analysis;
* ``lu.solve(b, trans='T')`` -- solves with A^T;
* :class:`BatchedGLU` -- many value sets of one pattern factored and solved
  together;
* :func:`sparse_solve` -- differentiable solve (torch.autograd.Function) with
  a hand-written adjoint;
* :func:`tune` -- the schedule autotuner.
"""
from __future__ import annotations

import numpy as np

try:
    import scipy.sparse as _sp

    _HAS_SCIPY = True
except ImportError:  # pragma: no cover
    _HAS_SCIPY = False

from . import _capi
from ._capi import GLUError, NotConvergedError, SingularMatrixError, check, ptr

__all__ = ["splu", "spsolve", "GLUFactorization", "BatchedGLU", "UnevenBatch", "sparse_solve", "tune",
           "GLUError", "SingularMatrixError", "NotConvergedError", "read_mtx"]


def _csc_parts(A):
    """(data, indices, indptr, shape) of a scipy sparse matrix or a CSC tuple."""
    if isinstance(A, tuple) and len(A) == 4:
        return A
    if _HAS_SCIPY and _sp.issparse(A):
        M = A.tocsc()  # a copy for any other format; canonicalised below
        if M is A:
            M = A.copy()
        M.sum_duplicates()
        M.sort_indices()
        return M.data, M.indices, M.indptr, M.shape
    raise TypeError("A must be a scipy sparse matrix or a "
                    "(data, indices, indptr, shape) tuple in CSC format")


def _to_csc_arrays(A):
    """Return (data_f64, indices_i32, indptr_i32, n) of a square sparse matrix.

    Accepts what the reference's pyglu accepts (pyglu/__init__.py:28-63) and
    raises the same exception types with the same messages, so that callers
    matching on them keep working.
    """
    data, indices, indptr, shape = _csc_parts(A)
    rows, cols = shape
    if rows != cols:
        raise ValueError(f"Matrix must be square, got shape {shape}")
    arrays = [np.ascontiguousarray(a, dtype=t)
              for a, t in ((data, np.float64), (indices, np.int32), (indptr, np.int32))]
    if arrays[2].shape[0] != rows + 1:
        raise ValueError(f"indptr length {arrays[2].shape[0]} inconsistent with n={rows}")
    if rows == 0:
        raise ValueError("Matrix dimension must be > 0")
    return arrays[0], arrays[1], arrays[2], rows


def _validate(data, indices, indptr, n):
    """Checks of the reference binding (src/glu_binding.cpp:51-77)."""
    if n <= 0:
        raise ValueError("n must be positive")
    data = np.ascontiguousarray(data, dtype=np.float64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    indptr = np.ascontiguousarray(indptr, dtype=np.int32)
    if indices.shape[0] != data.shape[0]:
        raise ValueError("data and indices length mismatch")
    if indptr.shape[0] != n + 1:
        raise ValueError("indptr length must be n+1")
    if (indices < 0).any():
        raise ValueError("Negative row index in CSC matrix")
    if (indptr < 0).any():
        raise ValueError("Negative indptr value")
    return data, indices.astype(np.uint32), indptr.astype(np.uint32)


class Analysis:
    """NICSLU preprocessing plus the symbolic phase of one sparsity pattern.

    Holds the preprocessed matrix, the permutations/scalings used by the
    solves, the map from the input matrix's entries into the LU layout, and
    the L+U pattern (the reference's Symbolic_Matrix arrays).
    """

    def __init__(self, data, indices, indptr, n):
        data, ai, ap = _validate(data, indices, indptr, n)
        if data.size == 0:
            raise RuntimeError("GLU preprocessing failed (error -1)")
        pre = _capi.pre()
        h = _capi.C.c_void_p()
        ret = pre.glu_pre_analyze(n, data.size, ptr(data), ptr(ai), ptr(ap), _capi.C.byref(h))
        if ret != 0:
            raise RuntimeError(f"GLU preprocessing failed (error {ret})")
        try:
            nz = pre.glu_pre_nnz(h)
            self.n = n
            self.nnz_a = nz
            self.pax = np.empty(nz, np.float64)
            self.pai = np.empty(nz, np.uint32)
            self.pap = np.empty(n + 1, np.uint32)
            pre.glu_pre_matrix(h, ptr(self.pax), ptr(self.pai), ptr(self.pap))
            self.col_perm = np.empty(n, np.uint32)
            self.row_perm_inv = np.empty(n, np.uint32)
            self.pivot = np.empty(n, np.int32)
            self.col_scale_perm = np.empty(n, np.float64)
            self.row_scale = np.empty(n, np.float64)
            mc = _capi.C.c_int(0)
            pre.glu_pre_transform(h, ptr(self.col_perm), ptr(self.row_perm_inv), ptr(self.pivot),
                                  ptr(self.col_scale_perm), ptr(self.row_scale), _capi.C.byref(mc))
            self.mc64 = int(mc.value)
            self.src_pos = np.empty(nz, np.uint32)
            self.src_scale = np.empty(nz, np.float64)
            pre.glu_pre_source_map(h, ptr(self.src_pos), ptr(self.src_scale))
        finally:
            pre.glu_pre_destroy(h)
        self.data, self.ai, self.ap = data, ai, ap
        eng = _capi.engine()
        self._sym = _capi.C.c_void_p()
        check(eng.glu_symbolic_analyze(n, nz, ptr(self.pap), ptr(self.pai), _capi.C.byref(self._sym)),
              "symbolic analysis")
        nlu = _capi.C.c_uint32(0)
        eng.glu_symbolic_sizes(self._sym, None, _capi.C.byref(nlu))
        self.nnz_lu = int(nlu.value)
        slots = np.empty(nz, np.uint32)
        eng.glu_symbolic_slots(self._sym, ptr(slots))
        self.slots = slots
        self.src_slot = np.ascontiguousarray(slots[self.src_pos])

    def pattern(self):
        """The L+U pattern: dict of the Symbolic_Matrix arrays (include/symbolic.h:15-21)."""
        n, z = self.n, self.nnz_lu
        out = dict(sym_c_ptr=np.empty(n + 1, np.uint32), sym_r_idx=np.empty(z, np.uint32),
                   l_col_ptr=np.empty(n, np.uint32), csr_r_ptr=np.empty(n + 1, np.uint32),
                   csr_c_idx=np.empty(z, np.uint32), csr_diag_ptr=np.empty(n, np.uint32))
        _capi.engine().glu_symbolic_export(self._sym, *(ptr(out[k]) for k in (
            "sym_c_ptr", "sym_r_idx", "l_col_ptr", "csr_r_ptr", "csr_c_idx", "csr_diag_ptr")))
        return out

    def predict_lu(self, pax=None):
        """predictLU (src/symbolic.cc:82-103): FP32 LU values from the preprocessed FP64 values."""
        pax = self.pax if pax is None else np.ascontiguousarray(pax, np.float64)
        val = np.empty(self.nnz_lu, np.float32)
        _capi.engine().glu_predict_lu(self._sym, ptr(pax), ptr(val))
        return val

    def __del__(self):
        try:
            _capi.engine().glu_symbolic_destroy(self._sym)
        except Exception:
            pass


def _torch():
    import torch

    return torch


def _stream():
    torch = _torch()
    return _capi.C.c_void_p(torch.cuda.current_stream().cuda_stream)


class _Engine:
    """A device handle for `batch` value sets of one analysed pattern."""

    def __init__(self, an: Analysis, batch=1, device=0):
        eng = _capi.engine()
        self.an = an
        self.batch = batch
        self.device = device
        self._h = _capi.C.c_void_p()
        check(eng.glu_create(an._sym, device, batch, _capi.C.byref(self._h)), "device setup")
        check(eng.glu_set_transform(self._h, ptr(an.col_perm), ptr(an.row_perm_inv), ptr(an.pivot),
                                    ptr(an.col_scale_perm), ptr(an.row_scale), an.mc64), "transform setup")
        check(eng.glu_set_source(self._h, an.nnz_a, ptr(an.ap), ptr(an.ai), ptr(an.src_slot),
                                 ptr(an.src_scale)), "source setup")

    def __del__(self):
        try:
            _capi.engine().glu_destroy(self._h)
        except Exception:
            pass


def _check_device_tensor(t, name, dtype, numel, device):
    """The engine reads and writes device pointers as raw arrays: refuse any
    tensor whose memory is not exactly what the call will touch."""
    if not _is_cuda_tensor(t):
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.device.index != device:
        raise ValueError(f"{name} is on cuda:{t.device.index}, the factorization on cuda:{device}")
    if str(t.dtype) != f"torch.{dtype}":
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.numel() != numel:
        raise ValueError(f"{name} must hold {numel} values, got {t.numel()}")


def _is_cuda_tensor(x):
    return hasattr(x, "is_cuda") and x.is_cuda


class GLUFactorization:
    """GPU LU factorization of a sparse matrix (same constructor as the reference).

    Constructed by :func:`splu`.  Call ``.solve(b)`` to solve ``Ax = b``.
    """

    def __init__(self, data, indices, indptr, n, perturb=False, device=0):
        self._setup(Analysis(data, indices, indptr, n), perturb, device)

    def _setup(self, an, perturb, device):
        self._an = an
        self._eng = _Engine(self._an, 1, device)
        self.perturb = bool(perturb)
        self._factor_values(self._an.data)

    @classmethod
    def _from_analysis(cls, an, perturb=False, device=0):
        """A factorization of an already analysed matrix."""
        obj = cls.__new__(cls)
        obj._setup(an, perturb, device)
        return obj

    # -- reference surface -------------------------------------------------
    @property
    def n(self):
        """Matrix dimension."""
        return self._an.n

    def solve(self, b, refine=False, tol=1e-10, maxiter=10, trans="N"):
        """Solve ``A x = b`` (``trans='T'``: ``A^T x = b``).

        b has shape (n,) or (n, k).  Without ``refine`` this is the reference's
        FP32 solve (b cast to float32, result returned as float64); with it,
        FP64 iterative refinement to relative residual ``tol``.
        """
        b = np.asarray(b, dtype=np.float64)
        n = self.n
        if b.shape[0] != n:
            raise ValueError(f"RHS length {b.shape[0]} != matrix dimension {n}")
        vec = b.ndim == 1
        bm = np.ascontiguousarray(b.reshape(n, -1).T)  # (k, n)
        k = bm.shape[0]
        t = 1 if str(trans).upper() in ("T", "H") else 0
        eng = _capi.engine()
        if refine:
            x = np.empty_like(bm)
            st = _capi.RefineStats()
            s = eng.glu_solve_refined(self._eng._h, 0, 1, k, ptr(bm), ptr(x), float(tol), int(maxiter), t,
                                      _capi.GLU_HOST, _capi.C.byref(st), None)
            self.last_refine = dict(iterations=st.iterations, residual=st.residual,
                                    residual_inf=st.residual_inf)
            if s != _capi.GLU_ERR_NOT_CONVERGED:
                check(s, "refined solve")
        else:
            bf = bm.astype(np.float32)
            xf = np.empty_like(bf)
            fn = eng.glu_solve_transposed if t else eng.glu_solve
            check(fn(self._eng._h, 0, k, ptr(bf), ptr(xf), _capi.GLU_HOST, None), "solve")
            x = xf.astype(np.float64)
        x = x.T
        return np.ascontiguousarray(x[:, 0] if vec else x)

    # -- additions ---------------------------------------------------------
    def _factor_values(self, data):
        eng = _capi.engine()
        data = np.ascontiguousarray(data, dtype=np.float64)
        if data.shape != (self._an.nnz_a,):
            raise ValueError(f"expected {self._an.nnz_a} values, got shape {data.shape}")
        check(eng.glu_load_source_values(self._eng._h, 0, 1, ptr(data), _capi.GLU_HOST, None), "value upload")
        check(eng.glu_factor(self._eng._h, 0, 1, 1 if self.perturb else 0, None), "GPU factorization")

    def refactor(self, data):
        """Refactorize with new values of the same pattern (the data array of
        the CSC matrix in the same order as the one given to the constructor)."""
        self._factor_values(data)
        return self

    def refactor_device(self, data, stream=None):
        """Refactorize from a CUDA float64 tensor of values (no host round trip)."""
        _check_device_tensor(data, "data", "float64", self._an.nnz_a, self._eng.device)
        eng = _capi.engine()
        st = stream if stream is not None else _stream()
        check(eng.glu_load_source_values(self._eng._h, 0, 1, _capi.C.c_void_p(data.data_ptr()),
                                         _capi.GLU_DEVICE, st), "value upload")
        check(eng.glu_factor(self._eng._h, 0, 1, 1 if self.perturb else 0, st), "GPU factorization")

    def solve_device(self, b, x, refine=True, tol=1e-10, maxiter=10, trans="N", stream=None):
        """Solve with CUDA float64 tensors b, x of shape (k, n) (refined) or
        float32 (plain); returns the refinement statistics."""
        k = b.shape[0] if b.dim() == 2 else 1
        dtype = "float64" if refine else "float32"
        _check_device_tensor(b, "b", dtype, k * self.n, self._eng.device)
        _check_device_tensor(x, "x", dtype, k * self.n, self._eng.device)
        eng = _capi.engine()
        st = stream if stream is not None else _stream()
        t = 1 if str(trans).upper() in ("T", "H") else 0
        bp = _capi.C.c_void_p(b.data_ptr())
        xp = _capi.C.c_void_p(x.data_ptr())
        if refine:
            rs = _capi.RefineStats()
            s = eng.glu_solve_refined(self._eng._h, 0, 1, k, bp, xp, float(tol), int(maxiter), t,
                                      _capi.GLU_DEVICE, _capi.C.byref(rs), st)
            if s != _capi.GLU_ERR_NOT_CONVERGED:
                check(s, "refined solve")
            return dict(iterations=rs.iterations, residual=rs.residual, residual_inf=rs.residual_inf)
        fn = eng.glu_solve_transposed if t else eng.glu_solve
        check(fn(self._eng._h, 0, k, bp, xp, _capi.GLU_DEVICE, st), "solve")
        return None

    def lu_values(self):
        """FP32 factor values in the Symbolic_Matrix::val layout."""
        val = np.empty(self._an.nnz_lu, np.float32)
        check(_capi.engine().glu_store_lu_values(self._eng._h, 0, 1, ptr(val), _capi.GLU_HOST, None), "read values")
        return val

    def pattern(self):
        return self._an.pattern()

    def levels(self):
        """(level_ptr, level_idx) built on the GPU."""
        eng = _capi.engine()
        nl = _capi.C.c_int32(0)
        eng.glu_levels(self._eng._h, _capi.C.byref(nl), None, None)
        lp = np.empty(nl.value + 1, np.int32)
        li = np.empty(self.n, np.int32)
        eng.glu_levels(self._eng._h, None, ptr(lp), ptr(li))
        return lp, li

    @property
    def stats(self):
        st = _capi.Stats()
        _capi.engine().glu_get_stats(self._eng._h, _capi.C.byref(st))
        return {k: getattr(st, k) for k, _ in _capi.Stats._fields_}

    @property
    def analysis(self):
        return self._an

    @property
    def handle(self):
        return self._eng._h


def splu(A, perturb=False, device=0):
    """Compute the sparse LU factorization of A on the GPU.

    Parameters
    ----------
    A : scipy.sparse matrix (any format) or (data, indices, indptr, shape) tuple
    perturb : bool, optional -- GESP diagonal perturbation for tiny pivots.

    Raises ValueError for a non-square or inconsistent matrix, RuntimeError when
    preprocessing or the GPU factorization fails.
    """
    data, indices, indptr, n = _to_csc_arrays(A)
    return GLUFactorization(data, indices, indptr, n, perturb, device)


def spsolve(A, b, perturb=False, refine=False, tol=1e-10):
    """Solve the sparse linear system Ax = b on the GPU."""
    b = np.asarray(b, dtype=np.float64)
    return splu(A, perturb=perturb).solve(b, refine=refine, tol=tol)


class BatchedGLU:
    """Many value sets of one sparsity pattern, factored and solved together.

    ``values`` has shape (B, nnz) in the data order of the CSC pattern
    (data, indices, indptr).  NICSLU's ordering and scaling are computed once
    from ``values[0]`` and reused for every set, as NICSLU's own refactor does
    (NicsLU_ResetMatrixValues, nicslu_matrix.c:244-269).
    """

    def __init__(self, indices, indptr, n, values, perturb=False, device=0):
        values = np.ascontiguousarray(values, dtype=np.float64)
        if values.ndim != 2:
            raise ValueError("values must have shape (B, nnz)")
        self._an = Analysis(values[0], indices, indptr, n)
        self.batch = values.shape[0]
        self._eng = _Engine(self._an, self.batch, device)
        self.perturb = bool(perturb)
        self.refactor(values)

    @property
    def n(self):
        return self._an.n

    def refactor(self, values):
        eng = _capi.engine()
        values = np.ascontiguousarray(values, dtype=np.float64)
        if values.shape != (self.batch, self._an.nnz_a):
            raise ValueError(f"values must have shape ({self.batch}, {self._an.nnz_a})")
        check(eng.glu_load_source_values(self._eng._h, 0, self.batch, ptr(values), _capi.GLU_HOST, None),
              "value upload")
        status = eng.glu_factor(self._eng._h, 0, self.batch, 1 if self.perturb else 0, None)
        check(status, "GPU factorization")

    def solve(self, b, tol=1e-10, maxiter=10, refine=True):
        """b: (B, k, n) float64 -> x (B, k, n), FP64-refined."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if b.ndim == 2:
            b = b[:, None, :]
        B, k, n = b.shape
        if B != self.batch or n != self.n:
            raise ValueError("b must have shape (B, k, n)")
        x = np.empty_like(b)
        st = _capi.RefineStats()
        s = _capi.engine().glu_solve_refined(self._eng._h, 0, B, k, ptr(b), ptr(x), float(tol), int(maxiter),
                                             0, _capi.GLU_HOST, _capi.C.byref(st), None)
        self.last_refine = dict(iterations=st.iterations, residual=st.residual, residual_inf=st.residual_inf)
        if s != _capi.GLU_ERR_NOT_CONVERGED:
            check(s, "refined solve")
        return x

    @property
    def handle(self):
        return self._eng._h

    @property
    def stats(self):
        st = _capi.Stats()
        _capi.engine().glu_get_stats(self._eng._h, _capi.C.byref(st))
        return {k: getattr(st, k) for k, _ in _capi.Stats._fields_}


class UnevenBatch:
    """Independent systems of different sizes and patterns, each with its own
    right-hand sides, refactored and solved together.

    ``systems`` is a list of CSC matrices ``(data, indices, indptr, n)``.  Each
    system keeps its own analysis and handle; refactorization and refined
    solves go through glu_factor_many / glu_solve_refined_many: every system's
    kernels are enqueued on one of ``streams`` CUDA streams from one host
    thread, and the host waits once per factorization round and once per
    refinement step for all systems together.  The analyses (NICSLU
    preprocessing and the symbolic phase, on the host) run in ``workers``
    threads.  ``refactor`` keeps each system's ordering and scaling, as a
    refactorization does.
    """

    def __init__(self, systems, perturb=False, device=0, streams=16, workers=8):
        import concurrent.futures as cf

        torch = _torch()
        systems = list(systems)
        with cf.ThreadPoolExecutor(max(1, min(int(workers), len(systems)))) as ex:
            analyses = list(ex.map(lambda s_: Analysis(*s_), systems))
        self.lus = [GLUFactorization._from_analysis(an, perturb=perturb, device=device) for an in analyses]
        self._streams = [torch.cuda.Stream(device=device) for _ in range(max(1, min(int(streams), len(self.lus))))]
        self._stream_ptrs = (_capi.C.c_void_p * len(self._streams))(*[s_.cuda_stream for s_ in self._streams])
        self._handles = (_capi.C.c_void_p * len(self.lus))(*[lu.handle.value for lu in self.lus])
        self.perturb = bool(perturb)
        self.last_refine = None

    def __len__(self):
        return len(self.lus)

    def analysis(self, i):
        """The NICSLU preprocessing and symbolic phase of system i."""
        return self.lus[i].analysis

    def lu_values(self, i):
        """FP32 factor values of system i (Symbolic_Matrix::val layout)."""
        return self.lus[i].lu_values()

    def refactor(self, values):
        """New values for every system (a list of data arrays, CSC order)."""
        eng = _capi.engine()
        if len(values) != len(self.lus):
            raise ValueError(f"expected {len(self.lus)} value arrays, got {len(values)}")
        vals = [np.ascontiguousarray(v, dtype=np.float64) for v in values]
        for v, lu in zip(vals, self.lus):
            if v.shape != (lu._an.nnz_a,):
                raise ValueError(f"expected {lu._an.nnz_a} values, got shape {v.shape}")
        ns = len(self._streams)
        for i, (v, lu) in enumerate(zip(vals, self.lus)):
            check(eng.glu_load_source_values(lu._eng._h, 0, 1, ptr(v), _capi.GLU_HOST,
                                             _capi.C.c_void_p(self._stream_ptrs[i % ns])), "value upload")
        check(eng.glu_factor_many(len(self.lus), self._handles, 1 if self.perturb else 0, self._stream_ptrs, ns),
              "GPU factorization")
        return self

    def solve(self, bs, tol=1e-10, maxiter=10):
        """FP64-refined solves: ``bs[i]`` has shape (n_i,) or (n_i, k_i);
        returns the list of solutions in the same shapes."""
        eng = _capi.engine()
        if len(bs) != len(self.lus):
            raise ValueError(f"expected {len(self.lus)} right-hand sides, got {len(bs)}")
        vecs, mats, xs = [], [], []
        for b, lu in zip(bs, self.lus):
            b = np.asarray(b, dtype=np.float64)
            if b.shape[0] != lu.n:
                raise ValueError(f"RHS length {b.shape[0]} != matrix dimension {lu.n}")
            bm = np.ascontiguousarray(b.reshape(lu.n, -1).T)  # (k, n)
            vecs.append(b.ndim == 1)
            mats.append(bm)
            xs.append(np.empty_like(bm))
        count = len(self.lus)
        nrhs = (_capi.C.c_uint32 * count)(*[m.shape[0] for m in mats])
        bp = (_capi.C.c_void_p * count)(*[m.ctypes.data for m in mats])
        xp = (_capi.C.c_void_p * count)(*[x.ctypes.data for x in xs])
        stats = (_capi.RefineStats * count)()
        s = eng.glu_solve_refined_many(count, self._handles, nrhs, bp, xp, float(tol), int(maxiter), _capi.GLU_HOST,
                                       stats, self._stream_ptrs, len(self._streams))
        if s != _capi.GLU_ERR_NOT_CONVERGED:
            check(s, "refined solve")
        self.last_refine = [dict(iterations=st.iterations, residual=st.residual, residual_inf=st.residual_inf)
                            for st in stats]
        out = []
        for vec, x in zip(vecs, xs):
            x = x.T
            out.append(np.ascontiguousarray(x[:, 0] if vec else x))
        return out


def write_mtx(path, data, indices, indptr, n):
    """Write a CSC matrix as a Matrix Market 'coordinate real general' file with
    triplets column by column -- the order lu_cmd's reader requires
    (src/nicslu/util/nicslu_readfile.c:98-228).  Values round-trip exactly."""
    data = np.asarray(data, np.float64)
    rows = np.asarray(indices, np.int64) + 1
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(np.asarray(indptr, np.int64))) + 1
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n} {n} {data.size}\n")
        for r, c, v in zip(rows.tolist(), cols.tolist(), data.tolist()):
            f.write(f"{r} {c} {v!r}\n")


def read_mtx(path):
    """Matrix Market file -> (data, indices, indptr, n) with NICSLU's reader."""
    import ctypes as C

    pre = _capi.pre()
    n = C.c_uint32(0)
    nz = C.c_uint32(0)
    ax, ai, ap = C.c_void_p(), C.c_void_p(), C.c_void_p()
    ret = pre.glu_pre_read_mtx(str(path).encode(), C.byref(n), C.byref(nz), C.byref(ax), C.byref(ai), C.byref(ap))
    if ret != 0:
        raise RuntimeError(f"cannot read {path} (NICSLU error {ret})")
    try:
        data = np.ctypeslib.as_array(C.cast(ax, C.POINTER(C.c_double)), (nz.value,)).copy()
        indices = np.ctypeslib.as_array(C.cast(ai, C.POINTER(C.c_uint32)), (nz.value,)).astype(np.int32)
        indptr = np.ctypeslib.as_array(C.cast(ap, C.POINTER(C.c_uint32)), (n.value + 1,)).astype(np.int32)
    finally:
        for p in (ax, ai, ap):
            pre.glu_pre_free(p)
    return data, indices, indptr, int(n.value)


from .autograd import sparse_solve  # noqa: E402
from .autotune import tune  # noqa: E402
