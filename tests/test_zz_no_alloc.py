"""glu_solve_noalloc: the FP32 solve for callers that cannot allocate device
memory (framework-owned memory pools, code running under CUDA graph capture,
real-time loops).  It must give what glu_solve gives, call after call, from the
library's fixed device array instead of allocated working vectors.

Kept in a file of its own that pytest collects last; it passes alone in a fresh
process and after the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4  # relative to max |x|, as the other FP32 solve comparisons


def _cases():
    from pyglu import synth

    return [synth.nodal(1500, seed=2), synth.grid_mesh(side=40, seed=1, n_long=20)]


@pytest.mark.parametrize("case", [0, 1], ids=["nodal_dense_tail", "mesh"])
def test_noalloc_solve_matches_glu_solve(case):
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
