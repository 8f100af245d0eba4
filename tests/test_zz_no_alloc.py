"""glu_solve_noalloc: the FP32 solve for callers that cannot allocate device
memory (a simulator whose device memory a framework owns and pools, a
real-time loop that must not stall in the allocator).  Call after call it must
give what glu_solve gives and what the oracle's sweeps give on the same
factors, using the library's fixed device array instead of allocated working
vectors.

Kept in a file of its own that pytest collects last; it passes alone in a fresh
process and after the other tests.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-4  # relative to max |x|, as the other FP32 solve comparisons
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cases():
    from pyglu import synth

    return [synth.nodal(1500, seed=2), synth.grid_mesh(side=40, seed=1, n_long=20)]


def _oracle_x(lu, b):
    """Symbolic_Matrix::solve restated, on the GPU's own factors."""
    an = lu.analysis
    tr = dict(col_perm=an.col_perm, row_perm_inv=an.row_perm_inv, pivot=an.pivot,
              col_scale_perm=an.col_scale_perm, row_scale=an.row_scale, mc64=an.mc64)
    p, v = lu.pattern(), lu.lu_values()
    return np.stack([oracle.solve(p, v, tr, bi) for bi in b])


@pytest.mark.parametrize("case", [0, 1], ids=["nodal_dense_tail", "mesh"])
def test_noalloc_solve_matches_glu_solve_and_oracle(case):
    import torch

    import pyglu
    from pyglu import _capi

    A = _cases()[case]
    n = A[3]
    lu = pyglu.GLUFactorization(*A)
    eng = _capi.engine()
    h = lu.handle
    stream = _capi.C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(5 + case)
    for call, nrhs in enumerate((1, 3)):  # two calls in a row, the second with other sizes
        b = torch.tensor(rng.uniform(-1, 1, (nrhs, n)), dtype=torch.float32, device="cuda")
        x_ref = torch.empty_like(b)
        x_na = torch.full_like(b, float("nan"))
        _capi.check(eng.glu_solve(h, 0, nrhs, _capi.C.c_void_p(b.data_ptr()), _capi.C.c_void_p(x_ref.data_ptr()),
                                  _capi.GLU_DEVICE, stream), "glu_solve")
        _capi.check(eng.glu_solve_noalloc(h, 0, nrhs, _capi.C.c_void_p(b.data_ptr()),
                                          _capi.C.c_void_p(x_na.data_ptr()), stream), "glu_solve_noalloc")
        torch.cuda.synchronize()
        xr, xn = x_ref.cpu().numpy(), x_na.cpu().numpy()
        assert np.isfinite(xn).all(), call
        assert np.abs(xn - xr).max() <= TOL * np.abs(xr).max(), call
        xo = _oracle_x(lu, b.cpu().numpy())
        assert np.abs(xn - xo).max() <= TOL * np.abs(xo).max(), call


def test_noalloc_rejects_sizes_beyond_its_array():
    import torch

    import pyglu
    from pyglu import _capi, synth

    A = synth.nodal(300, seed=3)
    lu = pyglu.GLUFactorization(*A)
    eng = _capi.engine()
    b = torch.zeros(8, dtype=torch.float32, device="cuda")
    nrhs = (1 << 20) // A[3] + 1  # n * nrhs just above the limit; rejected before any access
    st = eng.glu_solve_noalloc(lu.handle, 0, nrhs, _capi.C.c_void_p(b.data_ptr()), _capi.C.c_void_p(b.data_ptr()),
                               None)
    assert st == _capi.GLU_ERR_UNSUPPORTED
    assert b"static scratch" in eng.glu_last_error()


_TAIL_LIMIT_CHILD = r"""
import sys
sys.path.insert(0, {pkg!r})
import torch
import pyglu
from pyglu import _capi, synth
A = synth.nodal(1500, seed=2)
lu = pyglu.GLUFactorization(*A)
m = lu.stats["dense_tail"]
assert m > 64 * 3, m  # more 64-row blocks than the lowered limit below allows
b = torch.zeros(A[3], dtype=torch.float32, device="cuda")
eng = _capi.engine()
st = eng.glu_solve_noalloc(lu.handle, 0, 1, _capi.C.c_void_p(b.data_ptr()), _capi.C.c_void_p(b.data_ptr()), None)
assert st == _capi.GLU_ERR_UNSUPPORTED, st
assert b"dense trailing block" in eng.glu_last_error()
print("rejected", m)
"""


def test_noalloc_rejects_dense_tail_beyond_its_array():
    """The dense-tail bound (order <= 262,080) is checked before any device
    access; the block limit is lowered through the environment so that a small
    matrix reaches the same rejection path."""
    code = _TAIL_LIMIT_CHILD.format(pkg=os.path.join(ROOT, "glu-hcu_b200"))
    env = dict(os.environ, GLU_NOALLOC_BLOCK_LIMIT="4")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "rejected" in r.stdout
