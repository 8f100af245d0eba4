"""The differentiable solve (pyglu.sparse_solve) on the differentiation
configuration's generator (band 24, 5% unsymmetric rows).

* n = 2,000: the adjoint gradients of loss = w.x with respect to every
  nonzero of A and every entry of b against the gradients of a dense
  torch.linalg.solve (FP64) of the same system, 1e-6 relative.
* n = 100,000: FP64 central differences at relative step 1e-6 on 16 random
  nonzeros and 64 random entries of b, 1e-6 relative (bench.py --workload
  adjoint runs the same check on 64 nonzeros; at this size the pattern fills
  to 1.4e9 LU entries with a 36,784-wide dense tail, and every nonzero costs
  two refactorizations).  Each quotient
  (f(v + h) - f(v - h)) / 2h is evaluated without subtracting the two
  function values, which at this size agree to more digits than FP64 holds
  (the 2-norm condition number is about 1e8):
    - nonzero q = (i, j), A(+-) = A(v) +- h e_i e_j^T:  A(+)(x(+) - x(-)) =
      -2h e_i x(-)_j, hence  f(+) - f(-) = -2h x(-)_j lambda(+)_i  with
      x(-) = A(-)^-1 b and lambda(+) = A(+)^-T w -- an identity, so the quotient
      is -x(-)_j lambda(+)_i exactly: two refactorizations at the perturbed
      values, a refined solve and a refined transposed solve;
    - entry i of b: f is linear in b, so the quotient is w . A^-1 e_i exactly,
      one refined (non-transposed) solve of e_i -- independent of the
      transposed solve the adjoint uses.
  The identity itself is checked on the CPU against plainly subtracted
  function values (tests/test_cpu_adjoint_quotient.py).
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


def test_adjoint_matches_central_differences_n100000():
    import torch

    from pyglu import synth

    A = synth.config4(n=100_000, seed=2)
    data, indices, indptr, n = A
    lu, w, b, loss, gv, gb = _loss_and_grads(A, seed=4)
    wn = w.cpu().numpy()
    bn = b.cpu().numpy()
    cols = np.repeat(np.arange(n), np.diff(indptr))
    rng = np.random.default_rng(5)
    # FP64 refinement stalls near 1e-15 on this system: a few steps past 1e-14
    # change nothing measurable
    kw = dict(refine=True, tol=1e-14, maxiter=10)

    worst = 0.0
    atol = 1e-9 * np.abs(gv).max()
    for q in rng.choice(len(data), 16, replace=False):
        i, j = indices[q], cols[q]
        h = 1e-6 * abs(data[q])
        vp, vm = data.copy(), data.copy()
        vp[q] += h
        vm[q] -= h
        lam_p = lu.refactor(vp).solve(wn, trans="T", **kw)
        x_m = lu.refactor(vm).solve(bn, **kw)
        fd = -x_m[j] * lam_p[i]  # == (f(v + h) - f(v - h)) / 2h
        assert abs(fd - gv[q]) <= 1e-6 * abs(fd) + atol, (q, fd, gv[q])
        worst = max(worst, abs(fd - gv[q]) / max(abs(fd), 1e-300))
    print(f"nonzeros: max relative difference {worst:.2e}")

    lu.refactor(data)
    idx = rng.choice(n, 64, replace=False)
    E = np.zeros((n, 64))
    E[idx, np.arange(64)] = 1.0
    fd_b = wn @ lu.solve(E, **kw)  # (f(b + h e_i) - f(b - h e_i)) / 2h, exact for a linear f
    atol_b = 1e-9 * np.abs(gb).max()
    assert np.all(np.abs(fd_b - gb[idx]) <= 1e-6 * np.abs(fd_b) + atol_b), \
        np.max(np.abs(fd_b - gb[idx]) / np.abs(fd_b))
    print(f"b: max relative difference {np.max(np.abs(fd_b - gb[idx]) / np.abs(fd_b)):.2e}")
    assert torch.cuda.is_available()
