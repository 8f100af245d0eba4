"""The schedule autotuner on the default (supernodal) path.

tune() must pick a schedule that refactors no slower than the engine's
defaults (timed in the same search), leave factors that still match the
oracle, and round-trip its cache: a second call, and a new handle of the same
pattern, get the stored schedule without timing.
"""
import numpy as np
import pytest

import oracle

from test_gpu_parity import FACTOR_TOL, col_max_rel

pytestmark = pytest.mark.gpu


def test_tune_config0_default_path(tmp_path):
    import pyglu
    from pyglu import autotune, synth

    A = synth.config0()
    lu = pyglu.GLUFactorization(*A)
    assert autotune.current(lu.handle)["sn_width"] > 0  # the supernodal default path
    cache = str(tmp_path / "tune.json")
    best, ms, rep = pyglu.tune(lu, cache=cache, repeats=3, passes=1)
    assert not rep["cached"]
    assert ms <= rep["default_ms"]
    assert {k for k, _, _ in rep["trials"]} <= set(autotune.SUPERNODAL_SPACE)
    assert autotune.current(lu.handle) == best
    # the tuned handle's factors against the oracle
    p = lu.pattern()
    lp, li = lu.levels()
    ref = oracle.factor(p, lu.analysis.predict_lu(), lp, li, np.float32)
    assert col_max_rel(lu.lu_values(), ref, p["sym_c_ptr"]) <= FACTOR_TOL
    # cache: the same handle, then a new handle of the same pattern
    best2, ms2, rep2 = pyglu.tune(lu, cache=cache)
    assert rep2["cached"] and best2 == best and ms2 == ms
    lu2 = pyglu.GLUFactorization(*A)
    pyglu.tune(lu2, cache=cache)
    assert autotune.current(lu2.handle) == best


def test_tune_batch(tmp_path):
    import pyglu
    from pyglu import synth

    A = synth.nodal(2000, seed=12, band=32, n_long=2, unsym_frac=0.1)
    vals = synth.perturb_values(*A, count=4, seed=1)
    bl = pyglu.BatchedGLU(A[1], A[2], A[3], vals)
    space = {"dense_tc_min": [0, 512], "dense_lookahead": [0, 1024]}
    best, ms, rep = pyglu.tune(bl, data=vals, cache=str(tmp_path / "t.json"), space=space, repeats=2)
    assert ms <= rep["default_ms"]
    b = synth.rhs_uniform(A[3], 2, seed=3)
    X = bl.solve(np.broadcast_to(b, (4, 2, A[3])).copy(), tol=1e-12, maxiter=30)
    import scipy.sparse as sp

    for z in range(4):
        M = sp.csc_matrix((vals[z], A[1], A[2]), shape=(A[3], A[3]))
        for k in range(2):
            assert np.linalg.norm(M @ X[z, k] - b[k]) / np.linalg.norm(b[k]) <= 1e-10
