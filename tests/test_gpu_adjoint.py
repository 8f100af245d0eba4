"""The differentiable solve (pyglu.sparse_solve) on the differentiation
configuration's generator (band 24, 5% unsymmetric rows), at sizes beyond
the small-matrix check in test_gpu_parity.

* n = 2,000: the adjoint gradients of loss = w.x with respect to every
  nonzero of A and every entry of b against the gradients of a dense
  torch.linalg.solve (FP64) of the same system, 1e-6 relative.
* n = 20,000: FP64 central differences (relative step 1e-6) on 16 nonzeros
  and 16 entries of b, 1e-6 relative.  The function values come from the
  engine's FP64-refined solve (relative residual 1e-15 asked); the
  differences are taken on the entries of largest relative sensitivity
  |v_q g_q| / |f|: a central difference at relative step h resolves a
  gradient to about (forward error of f) / (h * sensitivity), so only the
  most sensitive entries of a system this size are resolved to 1e-6 by FP64.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _loss_and_grads(A, seed, device="cuda"):
    import torch

    import pyglu

    data, indices, indptr, n = A
    lu = pyglu.GLUFactorization(*A)
    rng = np.random.default_rng(seed)
    w = torch.tensor(rng.standard_normal(n), dtype=torch.float64, device=device)
    vals = torch.tensor(data, dtype=torch.float64, device=device, requires_grad=True)
    b = torch.tensor(rng.uniform(-1, 1, n), dtype=torch.float64, device=device, requires_grad=True)
    x = pyglu.sparse_solve(vals, b, lu, tol=1e-15, maxiter=40)
    loss = (w * x).sum()
    loss.backward()
    return lu, w, b.detach(), float(loss.detach()), vals.grad.cpu().numpy(), b.grad.cpu().numpy()


def test_adjoint_matches_dense_gradient_n2000():
    import scipy.sparse as sp
    import torch

    from pyglu import synth

    A = synth.config4(n=2000, seed=1)
    data, indices, indptr, n = A
    lu, w, b, loss, gv, gb = _loss_and_grads(A, seed=3)
    M = torch.tensor(sp.csc_matrix((data, indices, indptr), shape=(n, n)).toarray(), dtype=torch.float64,
                     requires_grad=True)
    bb = b.cpu().clone().requires_grad_(True)
    xd = torch.linalg.solve(M, bb)
    (w.cpu() * xd).sum().backward()
    cols = np.repeat(np.arange(n), np.diff(indptr))
    gdense = M.grad.numpy()[indices, cols]
    assert np.allclose(gv, gdense, rtol=1e-6, atol=1e-9 * np.abs(gdense).max())
    assert np.allclose(gb, bb.grad.numpy(), rtol=1e-6, atol=1e-9 * np.abs(gb).max())


def test_adjoint_matches_central_differences_n20000():
    import torch

    from pyglu import synth

    A = synth.config4(n=20000, seed=2)
    data, indices, indptr, n = A
    lu, w, b, loss, gv, gb = _loss_and_grads(A, seed=4)
    wn = w.cpu().numpy()
    bn = b.cpu().numpy()

    def f(v, bb):
        lu.refactor(v)
        x = lu.solve(bb, refine=True, tol=1e-15, maxiter=40)
        return float(wn @ x)

    rng = np.random.default_rng(5)
    f0 = abs(loss)
    sens = np.abs(data * gv) / f0
    cand = np.argsort(sens)[-64:]  # the 64 most sensitive nonzeros
    assert sens[cand].min() >= 1e-3
    for q in rng.choice(cand, 16, replace=False):
        h = 1e-6 * abs(data[q])
        vp, vm = data.copy(), data.copy()
        vp[q] += h
        vm[q] -= h
        fd = (f(vp, bn) - f(vm, bn)) / (2 * h)
        assert abs(fd - gv[q]) <= 1e-6 * abs(fd), (q, fd, gv[q])
    lu.refactor(data)
    sb = np.abs(bn * gb) / f0
    cand_b = np.argsort(sb)[-64:]
    assert sb[cand_b].min() >= 1e-3
    for i in rng.choice(cand_b, 16, replace=False):
        h = 1e-6 * abs(bn[i])
        bp, bm = bn.copy(), bn.copy()
        bp[i] += h
        bm[i] -= h
        x_p = lu.solve(bp, refine=True, tol=1e-15, maxiter=40)
        x_m = lu.solve(bm, refine=True, tol=1e-15, maxiter=40)
        fd = (float(wn @ x_p) - float(wn @ x_m)) / (2 * h)
        assert abs(fd - gb[i]) <= 1e-6 * abs(fd), (i, fd, gb[i])
    assert torch.cuda.is_available()
