"""Host-side input checks that run before any device work.

glu_create_from_pattern validates every pointer and index array of the
Symbolic_Matrix pattern before any of them is used to index another (the
planners and the level kernel read them without bounds checks); a malformed
array is GLU_ERR_ARG, on a machine with or without a GPU.  pyglu's device
entry points refuse tensors whose memory is not exactly what the engine will
read and write.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from pyglu import _capi, synth

KEYS = ("sym_c_ptr", "sym_r_idx", "l_col_ptr", "csr_r_ptr", "csr_c_idx", "csr_diag_ptr")


@pytest.fixture(scope="module")
def pattern():
    import pyglu

    an = pyglu.Analysis(*synth.nodal(200, seed=1))
    return an.pattern()


def _create(p):
    eng = _capi.engine()
    h = C.c_void_p()
    n = p["sym_c_ptr"].size - 1
    nnz = p["sym_r_idx"].size
    arr = [np.ascontiguousarray(p[k], np.uint32) for k in KEYS]
    st = eng.glu_create_from_pattern(0, n, nnz, *(a.ctypes.data_as(C.c_void_p) for a in arr), 1, C.byref(h))
    if st == _capi.GLU_OK:
        eng.glu_destroy(h)
    return st, eng.glu_last_error().decode()


def _bad(p, key, fn):
    q = {k: np.array(v, copy=True) for k, v in p.items()}
    fn(q[key])
    return q


def test_valid_pattern_passes_the_checks(pattern):
    st, _ = _create(pattern)
    # without a GPU the call gets past validation and stops at the device
    assert st in (_capi.GLU_OK, _capi.GLU_ERR_NO_DEVICE)


@pytest.mark.parametrize("key,mutate,msg", [
    ("csr_diag_ptr", lambda a: a.__setitem__(3, a[3] + 1), "diagonal pointer of row"),
    ("csr_diag_ptr", lambda a: a.__setitem__(5, 0xFFFFFFF0), "diagonal pointer of row"),
    ("csr_r_ptr", lambda a: a.__setitem__(7, a[8] + 3), "csr_r_ptr decreases"),
    ("csr_r_ptr", lambda a: a.__setitem__(0, 1), "inconsistent pattern"),
    ("sym_c_ptr", lambda a: a.__setitem__(4, 0x7FFFFFFF), "sym_c_ptr decreases"),
    ("l_col_ptr", lambda a: a.__setitem__(2, a[2] + 1), "diagonal pointer of column"),
    ("csr_c_idx", lambda a: a.__setitem__(len(a) // 2, 10 ** 6), "out of range"),
])
def test_malformed_pattern_is_an_argument_error(pattern, key, mutate, msg):
    st, err = _create(_bad(pattern, key, mutate))
    assert st == _capi.GLU_ERR_ARG, (st, err)
    assert msg in err, err


def test_row_index_out_of_range_is_an_argument_error(pattern):
    q = {k: np.array(v, copy=True) for k, v in pattern.items()}
    cp, dg = q["sym_c_ptr"], q["l_col_ptr"]
    j = int(np.argmax(cp[1:] - dg >= 2))  # a column with an L part; its last row goes out of range
    q["sym_r_idx"][int(cp[j + 1]) - 1] = 10 ** 6
    st, err = _create(q)
    assert st == _capi.GLU_ERR_ARG, (st, err)
    assert "out of range" in err, err


def test_unsorted_rows_are_an_argument_error(pattern):
    q = {k: np.array(v, copy=True) for k, v in pattern.items()}
    cp = q["sym_c_ptr"]
    j = int(np.argmax(np.diff(cp.astype(np.int64)) >= 3))
    a, b = int(cp[j]), int(cp[j + 1])
    q["sym_r_idx"][a:b] = q["sym_r_idx"][a:b][::-1]
    st, err = _create(q)
    assert st == _capi.GLU_ERR_ARG, (st, err)


def test_transpose_mismatch_is_an_argument_error(pattern):
    q = {k: np.array(v, copy=True) for k, v in pattern.items()}
    # swap two column indices inside one CSR row that keeps its diagonal
    rp, ci, rd = q["csr_r_ptr"], q["csr_c_idx"], q["csr_diag_ptr"]
    for r in range(len(rp) - 1):
        if rp[r + 1] - rd[r] >= 3:
            p0 = int(rd[r]) + 1
            ci[p0], ci[p0 + 1] = ci[p0 + 1], ci[p0]
            break
    st, err = _create(q)
    assert st == _capi.GLU_ERR_ARG, (st, err)
    assert "transpose" in err


class _FakeTensor:
    """Stand-in for a CUDA tensor (no GPU here): just the attributes checked."""

    def __init__(self, dtype="float64", numel=10, contiguous=True, device=0, cuda=True):
        import torch

        self.is_cuda = cuda
        self.dtype = getattr(torch, dtype)
        self._n = numel
        self._c = contiguous
        self.device = type("D", (), {"index": device})()

    def numel(self):
        return self._n

    def is_contiguous(self):
        return self._c


@pytest.mark.parametrize("kw,msg", [
    (dict(cuda=False), "CUDA tensor"),
    (dict(device=1), "cuda:1"),
    (dict(dtype="float32"), "float64"),
    (dict(contiguous=False), "contiguous"),
    (dict(numel=9), "10 values"),
])
def test_device_entry_points_refuse_mismatched_tensors(kw, msg):
    import pyglu

    with pytest.raises(ValueError, match=msg):
        pyglu._check_device_tensor(_FakeTensor(**kw), "x", "float64", 10, 0)
    pyglu._check_device_tensor(_FakeTensor(), "x", "float64", 10, 0)  # the matching tensor passes


def test_oracle_unaffected_by_checks(pattern):
    """The oracle reads the same arrays; a valid pattern still levels."""
    lp, li = oracle.leveling(pattern)
    assert lp[-1] == pattern["sym_c_ptr"].size - 1
    assert np.array_equal(np.sort(li), np.arange(li.size))


def test_failure_injection_arguments():
    eng = _capi.engine()
    assert eng.glu_debug_inject(None, 99, 0) == _capi.GLU_ERR_ARG
    assert eng.glu_debug_inject(None, _capi.GLU_INJECT_UNSET_SOLVE_FLAG, 0) == _capi.GLU_ERR_ARG
    assert eng.glu_set_wait_limit(None, 10) == _capi.GLU_ERR_ARG
    assert eng.glu_debug_inject(None, _capi.GLU_INJECT_ALLOC_FAILURES, 3) == _capi.GLU_OK
    assert eng.glu_debug_inject(None, _capi.GLU_INJECT_ALLOC_FAILURES, 0) == _capi.GLU_OK
