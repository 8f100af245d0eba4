"""The tensor-core trailing update of the dense tail (tcgen05, three-part BF16 split) against
the oracle's FP32 column algorithm.

The tensor-core path is forced on small trailing blocks (dense_tc_min low) so
that partial 128 x 128 tiles, a short last panel, the panel pairs of the
look-ahead (forced with dense_lookahead) and both tail layouts (in place in the
CSC values, and the gathered buffer of the mesh) are exercised; each must stay
within the factor tolerance (factor_parity: per-column max-relative
difference <= 1e-4, or as close to the FP64 factors as the reference
algorithm's FP32 ones where FP32 cannot resolve 1e-4) and the profile must
show the tensor-core kernel ran (regions of less than
dense_tc_min^2 entries stay on the FP32 FMA kernel).
"""
import numpy as np
import pytest

import oracle

from test_gpu_parity import factor_parity

pytestmark = pytest.mark.gpu


def _factor(A, perturb=False, **tune):
    import pyglu
    from pyglu import _capi, autotune

    lu = pyglu.GLUFactorization(*A, perturb=perturb)
    autotune._set(lu.handle, tune)
    eng = _capi.engine()
    _capi.check(eng.glu_profile_enable(lu.handle, 1))
    lu.refactor(A[0])
    kt = _capi.kernel_times(lu.handle)
    _capi.check(eng.glu_profile_enable(lu.handle, 0))
    return lu, kt


def _check(lu, perturb=False):
    """factor_parity of the handle's factors against the oracle's FP32 and FP64
    column algorithm on the same input."""
    p = lu.pattern()
    lp, li = lu.levels()
    v0 = lu.analysis.predict_lu()
    pert = oracle.pert(p, v0) if perturb else 0.0
    ref = oracle.factor(p, v0, lp, li, np.float32, pert)
    ref64 = oracle.factor(p, v0, lp, li, np.float64, pert)
    v = lu.lu_values()
    assert np.isfinite(v).all()
    return factor_parity(v, ref, ref64, p["sym_c_ptr"])


CASES = {
    # name: (generator, tuning)
    "nodal1500_tc": (lambda s: s.nodal(1500, seed=2), {"dense_tc_min": 128}),
    "nodal2500_tc_pairs": (lambda s: s.nodal(2500, seed=9), {"dense_tc_min": 128, "dense_lookahead": 256}),
    "config0_tc_pairs": (lambda s: s.config0(), {"dense_tc_min": 128, "dense_lookahead": 512}),
    "mesh90_buffer_tc": (lambda s: s.grid_mesh(side=90, seed=3, n_long=40), {"dense_tc_min": 64}),
    "nodal_band32_tc_pairs": (lambda s: s.nodal(3000, seed=12, band=32, n_long=2, unsym_frac=0.1),
                              {"dense_tc_min": 128, "dense_lookahead": 256}),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tensor_core_update_matches_oracle(name):
    from pyglu import synth

    gen, tune = CASES[name]
    A = gen(synth)
    lu, kt = _factor(A, **tune)
    m = lu.stats["dense_tail"]
    assert m >= tune["dense_tc_min"], m
    assert kt["k_dense_update_tc"][1] > 0 and kt["k_dense_pack"][1] > 0, kt
    ok, err, over, ratio = _check(lu)
    print(f"{name}: m={m} max column relative difference {err:.3e} ({over} columns over, FP64 ratio {ratio:.2f})")
    assert ok, (err, over, ratio)


def test_tensor_core_update_with_gesp():
    from pyglu import synth

    A = synth.nodal(2000, seed=4)
    lu, kt = _factor(A, perturb=True, dense_tc_min=128, dense_lookahead=256)
    assert kt["k_dense_update_tc"][1] > 0
    ok, err, over, ratio = _check(lu, perturb=True)
    assert ok, (err, over, ratio)


def test_tensor_core_batch_of_value_sets():
    """Several value sets in one launch sequence (blockIdx.z of the packs and
    the tile index of the persistent update): every set against the oracle."""
    import pyglu
    from pyglu import _capi, autotune, synth

    A = synth.nodal(2000, seed=12, band=32, n_long=2, unsym_frac=0.1)
    vals = synth.perturb_values(*A, count=3, seed=1)
    bl = pyglu.BatchedGLU(A[1], A[2], A[3], vals)
    autotune._set(bl.handle, {"dense_tc_min": 128, "dense_lookahead": 256})
    bl.refactor(vals)
    an = bl._an
    p = an.pattern()
    lp, li = oracle.leveling(p)
    for z in range(3):
        placed = np.zeros(an.nnz_lu, np.float32)
        placed[an.src_slot] = (vals[z] * an.src_scale).astype(np.float32)
        ref = oracle.factor(p, placed, lp, li, np.float32)
        ref64 = oracle.factor(p, placed, lp, li, np.float64)
        v = np.empty(an.nnz_lu, np.float32)
        _capi.check(_capi.engine().glu_store_lu_values(bl.handle, z, 1, _capi.ptr(v), _capi.GLU_HOST, None))
        ok, err, over, ratio = factor_parity(v, ref, ref64, p["sym_c_ptr"])
        assert ok, (z, err, over, ratio)


def test_fma_path_still_selectable():
    from pyglu import synth

    A = synth.nodal(2500, seed=9)
    lu, kt = _factor(A, dense_tc_min=0)
    assert kt["k_dense_update_tc"][1] == 0 and kt["k_dense_update"][1] > 0
    assert _check(lu)[0]


COUPLE_CASES = {
    # name: (generator, tuning); defer_tail > 1 makes the coupling products
    # cheap in the cost model, so that small blocks defer columns too
    "nodal3000_band32": (lambda s: s.nodal(3000, seed=12, band=32, n_long=2, unsym_frac=0.1),
                         {"dense_tc_min": 128, "dense_lookahead": 256, "defer_tail": 64}),
    "config0_many_groups": (lambda s: s.config0(), {"dense_tc_min": 128, "defer_tail": 100000}),
    "mesh90_buffer": (lambda s: s.grid_mesh(side=90, seed=3, n_long=40), {"dense_tc_min": 64, "defer_tail": 100000}),
}


@pytest.mark.parametrize("name", sorted(COUPLE_CASES))
def test_deferred_coupling_matches_oracle(name):
    """Sparse supernodes leave their update of the dense tail to tensor-core
    products after the sparse part (k_couple_pack, then the tensor-core update
    over the whole block); the factors stay within the factor tolerance of the
    oracle's column algorithm, for the in-place tail and the buffered one."""
    from pyglu import synth

    gen, tune = COUPLE_CASES[name]
    A = gen(synth)
    lu, kt = _factor(A, **tune)
    cols, groups = lu.stats["couple_columns"], lu.stats["couple_groups"]
    assert cols > 0 and groups == (cols + 127) // 128, (cols, groups)
    assert kt["k_couple_pack"][1] == groups, kt
    ok, err, over, ratio = _check(lu)
    lu0, kt0 = _factor(A, **{**tune, "defer_tail": 0})
    assert lu0.stats["couple_columns"] == 0 and kt0["k_couple_pack"][1] == 0
    ok0, err0, over0, ratio0 = _check(lu0)
    print(f"{name}: m={lu.stats['dense_tail']} deferred columns {cols} in {groups} products: max column "
          f"relative difference {err:.3e} ({over} columns over, FP64 ratio {ratio:.2f}); not deferred "
          f"{err0:.3e} ({over0}, {ratio0:.2f})")
    assert ok, (err, over, ratio)


def test_deferred_coupling_over_value_sets():
    import pyglu
    from pyglu import _capi, autotune, synth

    A = synth.nodal(2000, seed=12, band=32, n_long=2, unsym_frac=0.1)
    vals = synth.perturb_values(*A, count=3, seed=1)
    bl = pyglu.BatchedGLU(A[1], A[2], A[3], vals)
    autotune._set(bl.handle, {"dense_tc_min": 128, "dense_lookahead": 256, "defer_tail": 64})
    assert bl.stats["couple_columns"] > 0
    bl.refactor(vals)
    an = bl._an
    p = an.pattern()
    lp, li = oracle.leveling(p)
    for z in range(3):
        placed = np.zeros(an.nnz_lu, np.float32)
        placed[an.src_slot] = (vals[z] * an.src_scale).astype(np.float32)
        ref = oracle.factor(p, placed, lp, li, np.float32)
        ref64 = oracle.factor(p, placed, lp, li, np.float64)
        v = np.empty(an.nnz_lu, np.float32)
        _capi.check(_capi.engine().glu_store_lu_values(bl.handle, z, 1, _capi.ptr(v), _capi.GLU_HOST, None))
        ok, err, over, ratio = factor_parity(v, ref, ref64, p["sym_c_ptr"])
        assert ok, (z, err, over, ratio)


@pytest.mark.parametrize("group", [2, 3, 4])
@pytest.mark.parametrize("tc", [128, 0], ids=["tensor_cores", "fma"])
def test_lookahead_groups_match_oracle(group, tc):
    """Look-ahead groups of 2..4 panels: panel j's strips take K = 64 j, the
    rest K = 64 x group (up to 256 pack slots on the tensor-core path; the FMA
    kernel in 64-wide chunks)."""
    from pyglu import synth

    A = synth.nodal(3000, seed=12, band=32, n_long=2, unsym_frac=0.1)
    lu, kt = _factor(A, dense_tc_min=tc, dense_lookahead=256, dense_group=group, defer_tail=0)
    assert lu.stats["dense_tail"] > 4 * 64
    if tc:
        assert kt["k_dense_update_tc"][1] > 0
    ok, err, over, ratio = _check(lu)
    print(f"group {group} {'tc' if tc else 'fma'}: max column relative difference {err:.3e} ({over}, {ratio:.2f})")
    assert ok, (err, over, ratio)
