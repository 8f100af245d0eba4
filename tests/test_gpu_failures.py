"""Failure detection, with failures made on the host or a flag nothing sets.

* A device-side wait that runs out: the dense-tail solve sweeps are told to
  start their block tickets at 1 (GLU_INJECT_UNSET_SOLVE_FLAG), so no block
  sets the first block's completion flag; with a short wait limit every wait
  on it gives up, the kernel finishes, the call returns GLU_ERR_TIMEOUT, and
  the same handle then solves correctly.  Nothing faults or hangs the GPU.
* Device allocation failure: the library's next allocations are made to fail
  (GLU_INJECT_ALLOC_FAILURES); handle creation and a solve that needs larger
  working vectors return GLU_ERR_NOMEM, and the handle stays usable.

The reference reports neither: its waits are cudaDeviceSynchronize
(src/numeric.cu:615-616) and its CUDA errors go to a text stream
(numeric.cu:354-429).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _oracle_x(lu, b):
    an = lu.analysis
    tr = dict(col_perm=an.col_perm, row_perm_inv=an.row_perm_inv, pivot=an.pivot,
              col_scale_perm=an.col_scale_perm, row_scale=an.row_scale, mc64=an.mc64)
    return oracle.solve(lu.pattern(), lu.lu_values(), tr, b)


def _solve_status(lu, b):
    from pyglu import _capi

    bf = np.ascontiguousarray(b, np.float32)
    xf = np.empty_like(bf)
    st = _capi.engine().glu_solve(lu.handle, 0, 1, _capi.ptr(bf), _capi.ptr(xf), _capi.GLU_HOST, None)
    return st, xf


def test_solve_wait_runs_out_and_handle_stays_usable():
    import pyglu
    from pyglu import _capi, synth

    A = synth.config0()
    lu = pyglu.GLUFactorization(*A)
    assert lu.stats["dense_tail"] > 64 * 2  # several dense blocks wait on the first
    eng = _capi.engine()
    b = synth.rhs_uniform(A[3], 1, seed=4)[0]
    try:
        _capi.check(eng.glu_set_wait_limit(lu.handle, 20000))
        _capi.check(eng.glu_debug_inject(lu.handle, _capi.GLU_INJECT_UNSET_SOLVE_FLAG, 0))
        st, _ = _solve_status(lu, b)
        assert st == _capi.GLU_ERR_TIMEOUT, st
        assert b"timed out" in eng.glu_last_error()
    finally:
        _capi.check(eng.glu_set_wait_limit(lu.handle, 0))
    # the injection was for one solve: the next one completes and is right
    st, x = _solve_status(lu, b)
    assert st == _capi.GLU_OK
    xo = _oracle_x(lu, b)
    assert np.abs(x - xo).max() <= 1e-4 * np.abs(xo).max()


def test_unset_flag_injection_needs_a_dense_block():
    import pyglu
    from pyglu import _capi, autotune, synth

    A = synth.nodal(300, seed=3)
    lu = pyglu.GLUFactorization(*A)
    autotune._set(lu.handle, {"dense_tail_min": 1 << 31})
    assert lu.stats["dense_tail"] == 0
    assert _capi.engine().glu_debug_inject(lu.handle, _capi.GLU_INJECT_UNSET_SOLVE_FLAG, 0) == \
        _capi.GLU_ERR_UNSUPPORTED


def test_device_allocation_failure_is_nomem_and_recoverable():
    import pyglu
    from pyglu import _capi, synth

    eng = _capi.engine()
    A = synth.nodal(1500, seed=2)
    try:
        # creation: the first device allocation fails
        _capi.check(eng.glu_debug_inject(None, _capi.GLU_INJECT_ALLOC_FAILURES, 1))
        with pytest.raises(pyglu.GLUError) as ei:
            pyglu.GLUFactorization(*A)
        assert ei.value.status == _capi.GLU_ERR_NOMEM
        # nothing pending any more: creation succeeds
        lu = pyglu.GLUFactorization(*A)
        b = synth.rhs_uniform(A[3], 6, seed=5)  # (6, n): more right-hand sides than any solve before
        lu.solve(b[0])
        # a solve that needs larger working vectors
        _capi.check(eng.glu_debug_inject(None, _capi.GLU_INJECT_ALLOC_FAILURES, 1))
        bf = np.ascontiguousarray(b, np.float32)
        xf = np.empty_like(bf)
        st = eng.glu_solve(lu.handle, 0, 6, _capi.ptr(bf), _capi.ptr(xf), _capi.GLU_HOST, None)
        assert st == _capi.GLU_ERR_NOMEM, st
    finally:
        eng.glu_debug_inject(None, _capi.GLU_INJECT_ALLOC_FAILURES, 0)
    # the handle is still usable
    _capi.check(eng.glu_solve(lu.handle, 0, 6, _capi.ptr(bf), _capi.ptr(xf), _capi.GLU_HOST, None))
    for k in range(6):
        xo = _oracle_x(lu, b[k])
        assert np.abs(xf[k] - xo).max() <= 1e-4 * np.abs(xo).max()
