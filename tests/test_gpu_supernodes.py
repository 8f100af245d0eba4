"""GPU parity of the supernodal sparse factorization against the oracle.

The supernodal path groups runs of columns with nested lower patterns and a
dense diagonal block (widths 1..64) and levels them by the reference's column
dependencies.  Every width limit (20 and 40 end inside a 16-column chunk of
the diagonal-block LU and the row solves), with and without the dense
trailing block, must reproduce the oracle's FP32 column algorithm
(src/numeric.cu) within the factor tolerance: per-column max-relative
difference <= 1e-4.
"""
import numpy as np
import pytest

import oracle

from test_gpu_parity import FACTOR_TOL, col_max_rel

pytestmark = pytest.mark.gpu

NO_TAIL = 1 << 31


def _matrices():
    from pyglu import synth

    return {
        "config0": synth.config0(),
        "mesh90": synth.grid_mesh(side=90, seed=3, n_long=40),
        "nodal2500": synth.nodal(2500, seed=9),
    }


_CACHE = {}


def _matrix(name):
    if name not in _CACHE:
        _CACHE[name] = _matrices()[name]
    return _CACHE[name]


def _factor(A, perturb=False, **tune):
    import pyglu
    from pyglu import autotune

    lu = pyglu.GLUFactorization(*A, perturb=perturb)
    autotune._set(lu.handle, tune)
    lu.refactor(A[0])
    return lu


def _reference(lu, perturb=False):
    p = lu.pattern()
    lp, li = lu.levels()
    v0 = lu.analysis.predict_lu()
    pert = oracle.pert(p, v0) if perturb else 0.0
    return oracle.factor(p, v0, lp, li, np.float32, pert), p


@pytest.mark.parametrize("name", ["config0", "mesh90", "nodal2500"])
@pytest.mark.parametrize("width", [0, 1, 3, 20, 40, 64])
@pytest.mark.parametrize("tail", ["tail", "notail"])
def test_supernode_width_matches_oracle(name, width, tail):
    A = _matrix(name)
    tune = {"sn_width": width}
    if tail == "notail":
        tune["dense_tail_min"] = NO_TAIL
    lu = _factor(A, **tune)
    st = lu.stats
    if width:
        assert st["supernodes"] > 0 and st["sn_levels"] > 0 and st["sn_sweep_levels"] > 0
        assert st["sn_levels"] <= lu.analysis.n
    else:
        assert st["supernodes"] == 0 and st["sn_sweep_levels"] == 0
    if tail == "notail":
        assert st["dense_tail"] == 0
    v = lu.lu_values()
    assert np.isfinite(v).all()
    ref, p = _reference(lu)
    err = col_max_rel(v, ref, p["sym_c_ptr"])
    assert err <= FACTOR_TOL, (name, width, tail, err)
    # the sweeps of this schedule (supernodal when width > 0): FP64-refined solve
    import scipy.sparse as sp
    from pyglu import synth

    n = A[3]
    b = synth.rhs_uniform(n, 1, seed=5)[0]
    x = lu.solve(b, refine=True, tol=1e-12, maxiter=30)
    M = sp.csc_matrix(A[:3], shape=(n, n))
    assert np.linalg.norm(M @ x - b) / np.linalg.norm(b) <= 1e-10


def test_supernodes_cut_the_level_count():
    """The mesh's wide supernodes collapse thousands of column levels."""
    A = _matrix("mesh90")
    lu = _factor(A, sn_width=64, dense_tail_min=NO_TAIL)
    assert lu.stats["sn_levels"] * 4 < lu.stats["num_lev"]
    assert lu.stats["sn_sweep_levels"] * 2 < lu.stats["num_lev"]


@pytest.mark.parametrize("width", [3, 64])
def test_supernodes_perturbed_match_oracle(width):
    A = _matrix("nodal2500")
    lu = _factor(A, perturb=True, sn_width=width, dense_tail_min=NO_TAIL)
    ref, p = _reference(lu, perturb=True)
    err = col_max_rel(lu.lu_values(), ref, p["sym_c_ptr"])
    assert err <= FACTOR_TOL, err


def test_supernodes_refined_solve():
    import scipy.sparse as sp
    from pyglu import synth

    A = _matrix("mesh90")
    lu = _factor(A, sn_width=64)
    n = A[3]
    b = synth.rhs_loads(n, seed=2)
    x = lu.solve(b, refine=True, tol=1e-12, maxiter=30)
    M = sp.csc_matrix(A[:3], shape=(n, n))
    assert np.linalg.norm(M @ x - b) / np.linalg.norm(b) <= 1e-10


@pytest.mark.parametrize("small", [0, 1])
@pytest.mark.parametrize("width", [3, 4])
def test_small_supernode_grouping_matches_oracle(small, width):
    """Supernodes with few rows and targets run one per warp (sn_small = 1) or a
    block each (0); both must match the oracle, including the last pivots of a
    dense trailing region cut into narrow supernodes."""
    A = _matrix("nodal2500")
    lu = _factor(A, sn_width=width, dense_tail_min=NO_TAIL, sn_small=small)
    ref, p = _reference(lu)
    err = col_max_rel(lu.lu_values(), ref, p["sym_c_ptr"])
    assert err <= FACTOR_TOL, (small, width, err)


@pytest.mark.parametrize("name", ["config0", "mesh90"])
def test_dense_lookahead_matches_oracle(name):
    """The dense trailing block with the next panel factored during the
    current update (forced on these small tails) against the oracle, and the
    refined solve."""
    import scipy.sparse as sp
    from pyglu import synth

    A = _matrix(name)
    lu = _factor(A, dense_lookahead=64)
    assert lu.stats["dense_tail"] > 64
    ref, p = _reference(lu)
    err = col_max_rel(lu.lu_values(), ref, p["sym_c_ptr"])
    assert err <= FACTOR_TOL, err
    n = A[3]
    b = synth.rhs_uniform(n, 1, seed=6)[0]
    x = lu.solve(b, refine=True, tol=1e-12, maxiter=30)
    M = sp.csc_matrix(A[:3], shape=(n, n))
    assert np.linalg.norm(M @ x - b) / np.linalg.norm(b) <= 1e-10
