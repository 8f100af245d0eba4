"""CPU tests: the oracle pinned against the golden fixtures and the reference,
and the product's host logic (preprocessing, symbolic phase, value maps)."""
import glob
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

import oracle

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
PATTERN_KEYS = ("sym_c_ptr", "sym_r_idx", "l_col_ptr", "csr_r_ptr", "csr_c_idx", "csr_diag_ptr")


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def inputs(g):
    return g["data"], g["indices"], g["indptr"], int(g["n"])


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)


@pytest.fixture(params=FIXTURES, ids=[os.path.basename(f)[:-4] for f in FIXTURES])
def golden(request):
    return load(request.param)


# ------------------------------------------------------------- oracle pins --
def test_oracle_leveling_matches_golden(golden):
    lp, li = oracle.leveling(golden)
    assert np.array_equal(lp, golden["level_ptr"])
    assert np.array_equal(li, golden["level_idx"])


def test_oracle_fill_in_matches_golden(golden):
    cp, ri, dg = oracle.fill_in(golden["pap"], golden["pai"], int(golden["n"]))
    assert np.array_equal(cp, golden["sym_c_ptr"])
    assert np.array_equal(ri, golden["sym_r_idx"])
    assert np.array_equal(dg, golden["l_col_ptr"])


def test_oracle_factor_is_deterministic_and_matches_golden(golden):
    lu = oracle.factor(golden, golden["val"], golden["level_ptr"], golden["level_idx"], np.float32)
    assert np.array_equal(bits(lu), bits(golden["lu32"]))
    lu64 = oracle.factor(golden, golden["val"].astype(np.float64), golden["level_ptr"], golden["level_idx"],
                         np.float64)
    assert np.array_equal(bits(lu64), bits(golden["lu64"]))
    pert = oracle.pert(golden, golden["val"])
    assert np.float32(pert) == golden["pert"]
    lup = oracle.factor(golden, golden["val"], golden["level_ptr"], golden["level_idx"], np.float32, pert=pert)
    assert np.array_equal(bits(lup), bits(golden["lu32_pert"]))


def test_oracle_solve_matches_reference_solve(golden):
    tr = {k: golden[k] for k in ("col_perm", "row_perm_inv", "pivot", "col_scale_perm", "row_scale")}
    tr["mc64"] = int(golden["mc64"])
    x = oracle.solve(golden, golden["lu32"], tr, golden["b"])
    assert np.array_equal(bits(x), bits(golden["x_ref"]))


def test_oracle_factors_reproduce_matrix(golden):
    """L*U equals the preprocessed matrix (FP64 factors, FP64 check)."""
    import scipy.sparse as sp

    n = int(golden["n"])
    cp = golden["sym_c_ptr"].astype(np.int64)
    ri = golden["sym_r_idx"].astype(np.int64)
    dg = golden["l_col_ptr"].astype(np.int64)
    v = golden["lu64"]
    cols = np.repeat(np.arange(n), np.diff(cp))
    lower = ri > cols
    L = sp.csc_matrix((v[lower], (ri[lower], cols[lower])), shape=(n, n)) + sp.eye(n)
    U = sp.csc_matrix((v[~lower], (ri[~lower], cols[~lower])), shape=(n, n))
    # the factors start from predictLU's FP32 values
    A = sp.csc_matrix((golden["pax"].astype(np.float32).astype(np.float64), golden["pai"], golden["pap"]),
                      shape=(n, n))
    err = abs(L @ U - A).max()
    assert err <= 1e-9 * abs(A).max()
    assert np.array_equal(dg, golden["l_col_ptr"])


@pytest.mark.ref
def test_golden_fixtures_reproduce_with_live_reference(golden):
    """The fixtures are what the reference computes today (same build, same inputs)."""
    r = oracle.RefGLU(*inputs(golden))
    s = r.symbolic()
    for k in PATTERN_KEYS + ("level_ptr", "level_idx"):
        assert np.array_equal(s[k], golden[k]), k
    assert np.array_equal(bits(s["val"]), bits(golden["val"]))
    assert np.array_equal(bits(r.ax), bits(golden["pax"]))
    assert np.array_equal(bits(r.solve(golden["lu32"], golden["b"])), bits(golden["x_ref"]))


# ----------------------------------------------------- product host logic --
def test_analysis_matches_reference_preprocessing_and_symbolic(golden):
    import pyglu

    an = pyglu.Analysis(*inputs(golden))
    assert np.array_equal(bits(an.pax), bits(golden["pax"]))
    assert np.array_equal(an.pai, golden["pai"])
    assert np.array_equal(an.pap, golden["pap"])
    for k in ("col_perm", "row_perm_inv", "pivot"):
        assert np.array_equal(getattr(an, k), golden[k]), k
    for k in ("col_scale_perm", "row_scale"):
        assert np.array_equal(bits(getattr(an, k)), bits(golden[k])), k
    p = an.pattern()
    for k in PATTERN_KEYS:
        assert np.array_equal(p[k], golden[k]), k
    assert np.array_equal(bits(an.predict_lu()), bits(golden["val"]))


def test_source_map_places_values_bit_exactly(golden):
    """New values of A go straight into the LU layout: ax * scale is what NICSLU
    computes in place, and the slot is where predictLU puts it."""
    import pyglu

    an = pyglu.Analysis(*inputs(golden))
    d = golden["data"]
    placed = d * an.src_scale
    assert np.array_equal(bits(placed), bits(an.pax[an.src_pos]))
    val = np.zeros(an.nnz_lu, np.float32)
    val[an.src_slot] = placed.astype(np.float32)
    assert np.array_equal(bits(val), bits(golden["val"]))


def test_symbolic_against_oracle_on_meshes():
    """Fast fill-in equals the merge restatement on patterns with long paths."""
    import pyglu
    from pyglu import synth

    for side in (8, 17, 30):
        A = synth.grid_mesh(side=side, seed=side, n_long=side)
        an = pyglu.Analysis(*A)
        p = an.pattern()
        cp, ri, dg = oracle.fill_in(an.pap, an.pai, an.n)
        assert np.array_equal(p["sym_c_ptr"], cp)
        assert np.array_equal(p["sym_r_idx"], ri)
        assert np.array_equal(p["l_col_ptr"], dg)


@pytest.mark.ref
def test_symbolic_bit_exact_with_reference_config0():
    """The full-size n=4,960 nodal matrix: pattern and CSR identical."""
    import pyglu
    from pyglu import synth

    A = synth.config0()
    r = oracle.RefGLU(*A)
    s = r.symbolic()
    an = pyglu.Analysis(*A)
    p = an.pattern()
    for k in PATTERN_KEYS:
        assert np.array_equal(p[k], s[k]), k
    assert np.array_equal(bits(an.predict_lu()), bits(s["val"]))


def test_unpreprocessed_pattern_symbolic_matches_oracle():
    """Symbolic phase on an arbitrary unsymmetric pattern (no NICSLU)."""
    import ctypes as C

    from pyglu import _capi

    rng = np.random.default_rng(11)
    n = 150
    rows, cols = [], []
    for j in range(n):
        k = rng.integers(1, 5)
        rr = np.unique(np.concatenate([[j], rng.integers(0, n, k)]))
        rows.append(rr)
        cols.append(np.full(rr.size, j))
    ai = np.concatenate(rows).astype(np.uint32)
    ap = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.uint32)
    eng = _capi.engine()
    h = C.c_void_p()
    _capi.check(eng.glu_symbolic_analyze(n, ai.size, _capi.ptr(ap), _capi.ptr(ai), C.byref(h)))
    nz = C.c_uint32()
    eng.glu_symbolic_sizes(h, None, C.byref(nz))
    cp = np.empty(n + 1, np.uint32)
    ri = np.empty(nz.value, np.uint32)
    dg = np.empty(n, np.uint32)
    eng.glu_symbolic_export(h, _capi.ptr(cp), _capi.ptr(ri), _capi.ptr(dg), None, None, None)
    eng.glu_symbolic_destroy(h)
    ocp, ori, odg = oracle.fill_in(ap, ai, n)
    assert np.array_equal(cp, ocp) and np.array_equal(ri, ori) and np.array_equal(dg, odg)


# ------------------------------------------------------------------- C ABI --
def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(glu_\w+)\s*\(", txt)))


def test_c_abi_exports_every_declared_symbol():
    from pyglu import _capi

    eng = _capi.engine()
    pre = _capi.pre()
    for name in _declared("glu_b200.h"):
        assert hasattr(eng, name), name
    for name in _declared("glu_preprocess.h"):
        assert hasattr(pre, name), name
    assert sorted(_declared("glu_b200.h")) == sorted(_capi.ENGINE_SYMBOLS)
    assert sorted(_declared("glu_preprocess.h")) == sorted(_capi.PRE_SYMBOLS)


def test_engine_reports_no_device_without_gpu():
    """Creating a device handle fails cleanly (status, message) without a GPU."""
    from conftest import HAS_GPU

    if HAS_GPU:
        pytest.skip("GPU present")
    import ctypes as C

    import pyglu
    from pyglu import _capi, synth

    an = pyglu.Analysis(*synth.nodal(100, seed=1))
    h = C.c_void_p()
    st = _capi.engine().glu_create(an._sym, 0, 1, C.byref(h))
    assert st == _capi.GLU_ERR_NO_DEVICE
    assert b"device" in _capi.engine().glu_last_error()
    with pytest.raises(pyglu.GLUError):
        pyglu.splu(__import__("scipy.sparse", fromlist=["x"]).eye(4, format="csc") * 2.0)


# ------------------------------------------------- reference error behaviour --
def test_input_validation_like_reference():
    import scipy.sparse as sp

    import pyglu

    with pytest.raises(ValueError):
        pyglu._to_csc_arrays(sp.random(3, 4, density=0.5, format="csc"))
    with pytest.raises(TypeError):
        pyglu._to_csc_arrays(np.eye(3))
    with pytest.raises(ValueError):
        pyglu._to_csc_arrays((np.ones(1), np.zeros(1), np.zeros(3), (3, 3)))
    with pytest.raises(ValueError):
        pyglu._to_csc_arrays((np.ones(0), np.zeros(0), np.zeros(1), (0, 0)))
    with pytest.raises(ValueError):
        pyglu.GLUFactorization(np.ones(2), np.array([0, -1]), np.array([0, 1, 2]), 2)
    with pytest.raises(ValueError):
        pyglu.GLUFactorization(np.ones(2), np.array([0, 1]), np.array([0, 1]), 2)


def test_structurally_singular_matrix_fails_in_preprocessing():
    import pyglu

    # column 1 empty -> MC64 finds rank < n (nicslu_analyze.c:149-155)
    data = np.array([1.0, 2.0])
    indices = np.array([0, 1])
    indptr = np.array([0, 2, 2])
    with pytest.raises(RuntimeError, match="preprocessing failed"):
        pyglu.Analysis(data, indices, indptr, 2)


def test_duplicate_entries_rejected_by_preprocessing():
    import pyglu

    data = np.array([1.0, 2.0, 3.0])
    indices = np.array([0, 0, 1])
    indptr = np.array([0, 2, 3])
    with pytest.raises(RuntimeError, match="preprocessing failed"):
        pyglu.Analysis(data, indices, indptr, 2)


def test_scipy_duplicates_are_summed_like_reference():
    import scipy.sparse as sp

    import pyglu

    A = sp.coo_matrix((np.array([1.0, 2.0, 3.0, 4.0]), (np.array([0, 0, 1, 1]), np.array([0, 0, 1, 1]))),
                      shape=(2, 2))
    data, indices, indptr, n = pyglu._to_csc_arrays(A)
    assert np.array_equal(data, [3.0, 7.0])
    an = pyglu.Analysis(data, indices, indptr, n)
    assert an.nnz_lu == 2
