"""The supernodal solve sweeps in both launch forms against the oracle.

sn_sweep_fused = 0 (default): one launch per sweep level.  sn_sweep_fused = 1:
each sweep is one launch; blocks draw tickets in level order and wait, with a
bounded wait, until every supernode they solve has been released by the
blocks that update it.  Both must give Symbolic_Matrix::solve's result on the
same factors (src/symbolic.cc:200-251) within the FP32 solve tolerance, for
one and for several right-hand sides, and for several value sets at once.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _oracle_x(lu, b):
    an = lu.analysis
    tr = dict(col_perm=an.col_perm, row_perm_inv=an.row_perm_inv, pivot=an.pivot,
              col_scale_perm=an.col_scale_perm, row_scale=an.row_scale, mc64=an.mc64)
    p, v = lu.pattern(), lu.lu_values()
    return np.stack([oracle.solve(p, v, tr, bi) for bi in b])


@pytest.mark.parametrize("fused", [1, 0], ids=["fused", "per_level"])
@pytest.mark.parametrize("name", ["mesh90", "config0"])
def test_sweeps_match_oracle(name, fused):
    import pyglu
    from pyglu import autotune, synth

    A = synth.grid_mesh(side=90, seed=3, n_long=40) if name == "mesh90" else synth.config0()
    lu = pyglu.GLUFactorization(*A)
    autotune._set(lu.handle, {"sn_sweep_fused": fused})
    lu.refactor(A[0])
    assert lu.stats["sn_sweep_levels"] > 0
    b = synth.rhs_uniform(A[3], 3, seed=7)
    x = lu.solve(b.T).T  # (3, n)
    xo = _oracle_x(lu, b)
    assert np.abs(x - xo).max() <= TOL * np.abs(xo).max()


def split_levels(lu):
    """Levels of the last plain solve whose small-supernode groups had a launch
    of their own: the solve's launches less one per sweep level, the two
    transforms, the two sweeps' copies of the solved unknowns and, with a dense
    tail, its two triangular sweeps and the tail coupling."""
    st = lu.stats
    base = 2 + st["sn_sweep_levels"] + 2 + (3 if st["dense_tail"] else 0)
    return st["solve_launches"] - base


def test_per_level_sweeps_with_small_group_launches_match_oracle():
    """The 300 x 300 mesh (n = 90,000; tens of thousands of leaf supernodes):
    the per-level sweeps run the small-supernode groups of the wide levels in
    their own warp-per-supernode launches, the rest in the full kernel."""
    import pyglu
    from pyglu import autotune, synth

    A = synth.config1(side=300)
    lu = pyglu.GLUFactorization(*A)
    autotune._set(lu.handle, {"sn_sweep_fused": 0})
    lu.refactor(A[0])
    b = synth.rhs_uniform(A[3], 2, seed=9)
    x = lu.solve(b.T).T
    splits = split_levels(lu)
    print("levels with small-group launches:", splits)
    assert splits >= 0, splits
    xo = _oracle_x(lu, b)
    rel = np.abs(x - xo).max() / np.abs(xo).max()
    print(f"max difference relative to max |x|: {rel:.3e}")
    assert rel <= TOL, (rel, splits)


def test_fused_sweeps_over_value_sets():
    import scipy.sparse as sp

    import pyglu
    from pyglu import autotune, synth

    A = synth.grid_mesh(side=60, seed=5, n_long=20)
    vals = synth.perturb_values(*A, count=3, seed=2)
    bl = pyglu.BatchedGLU(A[1], A[2], A[3], vals)
    autotune._set(bl.handle, {"sn_sweep_fused": 1})
    bl.refactor(vals)
    b = synth.rhs_uniform(A[3], 2, seed=4)
    X = bl.solve(np.broadcast_to(b, (3, 2, A[3])).copy(), tol=1e-12, maxiter=30)
    for z in range(3):
        M = sp.csc_matrix((vals[z], A[1], A[2]), shape=(A[3], A[3]))
        for k in range(2):
            assert np.linalg.norm(M @ X[z, k] - b[k]) / np.linalg.norm(b[k]) <= 1e-10
