"""The identities the n = 100,000 finite-difference check evaluates its central
quotients with, on small dense FP64 systems where subtracting the two
function values loses nothing:

* A(+-) = A +- h e_i e_j^T:  (f(+) - f(-)) / 2h == -x(-)_j lambda(+)_i with
  f = w . A^-1 b, x(-) = A(-)^-1 b, lambda(+) = A(+)^-T w;
* f linear in b:  (f(b + h e_i) - f(b - h e_i)) / 2h == w . A^-1 e_i.
"""
import numpy as np


def _system(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + n * np.eye(n)
    return A, rng.standard_normal(n), rng.standard_normal(n)


def test_nonzero_quotient_identity():
    for seed in range(5):
        A, b, w = _system(12, seed)
        f = lambda M: w @ np.linalg.solve(M, b)  # noqa: E731
        for i, j in [(0, 0), (3, 7), (11, 2)]:
            h = 1e-2 * abs(A[i, j])  # a large step: the plain difference is accurate
            Ap, Am = A.copy(), A.copy()
            Ap[i, j] += h
            Am[i, j] -= h
            fp, fm = f(Ap), f(Am)
            plain = (fp - fm) / (2 * h)
            x_m = np.linalg.solve(Am, b)
            lam_p = np.linalg.solve(Ap.T, w)
            # the plain difference is good to a few units of FP64 in f, / 2h
            bound = 1e-12 * abs(plain) + 64 * np.finfo(float).eps * max(abs(fp), abs(fm)) / (2 * h)
            assert abs(plain - (-x_m[j] * lam_p[i])) <= bound


def test_rhs_quotient_identity():
    A, b, w = _system(10, 7)
    f = lambda bb: w @ np.linalg.solve(A, bb)  # noqa: E731
    for i in range(10):
        h = 0.5
        e = np.zeros(10)
        e[i] = 1.0
        plain = (f(b + h * e) - f(b - h * e)) / (2 * h)
        assert abs(plain - w @ np.linalg.solve(A, e)) <= 1e-12 * abs(plain)
