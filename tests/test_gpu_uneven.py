"""Uneven batch: independent systems of different sizes and patterns, each
with its own right-hand sides, refactored and solved together on separate
streams (the uneven-batch configuration at reduced sizes)."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _systems(count=6, seed=3):
    from pyglu import synth

    out = []
    for n, k, s in synth.config3_systems(count=count, seed=seed, n_range=(400, 2500), rhs_range=(1, 6)):
        A = synth.nodal(n, seed=s)
        out.append((A, synth.rhs_uniform(n, k, seed=s).T))  # b: (n, k)
    return out


def test_uneven_batch_refined_solves():
    import pyglu

    cases = _systems()
    ub = pyglu.UnevenBatch([A for A, _ in cases], workers=4)
    assert len(ub) == len(cases)
    xs = ub.solve([b for _, b in cases], tol=1e-12, maxiter=30)
    for (A, b), x in zip(cases, xs):
        n = A[3]
        M = sp.csc_matrix(A[:3], shape=(n, n))
        assert x.shape == b.shape
        r = np.linalg.norm(M @ x - b, axis=0) / np.linalg.norm(b, axis=0)
        assert r.max() <= 1e-10, r
    assert all(s["residual"] <= 1e-10 for s in ub.last_refine)


def test_uneven_batch_refactor_matches_oracle():
    """A refactor keeps each system's ordering and scaling: every member's
    factors of its new values agree with the oracle's FP32 column algorithm on
    the same values placed into the same pattern."""
    import pyglu
    from pyglu import synth

    import oracle

    cases = _systems(count=4, seed=5)
    ub = pyglu.UnevenBatch([A for A, _ in cases], workers=3)
    new_vals = [synth.perturb_values(*A, count=1, seed=9)[0] for A, _ in cases]
    ub.refactor(new_vals)
    for i, v in enumerate(new_vals):
        an = ub.analysis(i)
        p = an.pattern()
        lp, li = oracle.leveling(p)
        placed = np.zeros(an.nnz_lu, np.float32)
        placed[an.src_slot] = (v * an.src_scale).astype(np.float32)
        ref = oracle.factor(p, placed, lp, li, np.float32).astype(np.float64)
        a = ub.lu_values(i).astype(np.float64)
        cp = p["sym_c_ptr"].astype(np.int64)
        nz = np.diff(cp) > 0
        scale = np.maximum.reduceat(np.abs(ref), cp[:-1][nz])
        err = np.maximum.reduceat(np.abs(a - ref), cp[:-1][nz]) / np.where(scale > 0, scale, 1)
        assert err.max() <= 1e-4, (i, err.max())
