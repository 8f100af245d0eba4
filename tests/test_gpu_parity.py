"""GPU parity tests: the CUDA path against the golden fixtures and the oracle.

Tolerances (FP32 factors computed in a different order than the reference's
own nondeterministic atomics): per-column max-relative difference of the L+U
values <= 1e-4 (|a - b| / max_col |b|) -- for the tensor-core and deferred
coupling paths (factor_parity), on columns where the reference's FP32 factors
are themselves farther than that from the FP64 factors, at least as close to
the FP64 factors as the reference's FP32 ones, up to a factor of 2; level sets
and everything symbolic bit-exact; FP64-refined solves to relative residual
<= 1e-10.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

import oracle

pytestmark = pytest.mark.gpu

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
FACTOR_TOL = 1e-4
REFINE_TOL = 1e-10


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def inputs(g):
    return g["data"], g["indices"], g["indptr"], int(g["n"])


def col_rel(a, b, cptr):
    """Per column: max_i |a_i - b_i| / max_i |b_i| (LU values, CSC; nonempty
    columns)."""
    cptr = np.asarray(cptr, np.int64)
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    m = np.abs(b.astype(np.float64))
    starts = cptr[:-1]
    nz = np.diff(cptr) > 0
    dmax = np.maximum.reduceat(d, starts[nz])
    bmax = np.maximum.reduceat(m, starts[nz])
    return np.where(bmax > 0, dmax / np.where(bmax > 0, bmax, 1), dmax)


def col_max_rel(a, b, cptr):
    """Max over columns of max_i |a_i - b_i| / max_i |b_i| (LU values, CSC)."""
    return float(col_rel(a, b, cptr).max())


FP64_SLACK = 2.0


def factor_parity(v, ref32, ref64, cptr, tol=FACTOR_TOL):
    """Factor parity of FP32 factors v against the oracle's FP32 factors ref32
    of the same input, ref64 the oracle's FP64 factors of it.

    Every column must be within tol (per-column max-relative) of ref32.  On
    columns where FP32 itself cannot resolve tol -- where the two FP32 orders
    differ by more -- v must be at least as close to the FP64 factors as
    ref32 is, up to FP64_SLACK: the reference algorithm's own FP32 error then
    bounds ours.  Returns (passed, max difference to ref32, columns over tol,
    worst ratio of the two FP64 errors over those columns)."""
    d32 = col_rel(v, ref32, cptr)
    over = d32 > tol
    if not over.any():
        return True, float(d32.max()), 0, 0.0
    e_ours = col_rel(v, ref64, cptr)[over]
    e_ref = col_rel(ref32, ref64, cptr)[over]
    ratio = float((e_ours / np.maximum(e_ref, 1e-300)).max())
    return ratio <= FP64_SLACK, float(d32.max()), int(over.sum()), ratio


def rel_residual(g, x, b):
    import scipy.sparse as sp

    n = int(g["n"])
    A = sp.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n))
    return np.linalg.norm(A @ x - b) / np.linalg.norm(b)


@pytest.fixture(params=FIXTURES, ids=[os.path.basename(f)[:-4] for f in FIXTURES])
def golden(request):
    return load(request.param)


def test_levels_built_on_gpu_are_bit_exact(golden):
    import pyglu

    lu = pyglu.GLUFactorization(*inputs(golden))
    lp, li = lu.levels()
    assert np.array_equal(lp, golden["level_ptr"])
    assert np.array_equal(li, golden["level_idx"])


def test_factor_matches_reference_fp32(golden):
    import pyglu

    lu = pyglu.GLUFactorization(*inputs(golden))
    v = lu.lu_values()
    assert np.isfinite(v).all()
    err32 = col_max_rel(v, golden["lu32"], golden["sym_c_ptr"])
    assert err32 <= FACTOR_TOL, err32


def test_factor_perturbed_matches_reference(golden):
    import pyglu

    lu = pyglu.GLUFactorization(*inputs(golden), perturb=True)
    assert abs(lu.stats["pert"] - float(golden["pert"])) <= 1e-7 * float(golden["pert"])
    v = lu.lu_values()
    err = col_max_rel(v, golden["lu32_pert"], golden["sym_c_ptr"])
    assert err <= FACTOR_TOL, err


def test_plain_solve_matches_reference_solve(golden):
    """GPU FP32 solve vs Symbolic_Matrix::solve on the same GPU factors."""
    import pyglu

    lu = pyglu.GLUFactorization(*inputs(golden))
    v = lu.lu_values()
    b = golden["b"]
    x = lu.solve(b.astype(np.float64))
    tr = {k: golden[k] for k in ("col_perm", "row_perm_inv", "pivot", "col_scale_perm", "row_scale")}
    tr["mc64"] = int(golden["mc64"])
    x_ref = oracle.solve(golden, v, tr, b).astype(np.float64)
    scale = np.abs(x_ref).max()
    assert np.abs(x - x_ref).max() <= 1e-4 * scale


def test_refined_solve_reaches_fp64_residual(golden):
    import pyglu

    lu = pyglu.GLUFactorization(*inputs(golden))
    b = golden["b"].astype(np.float64)
    x = lu.solve(b, refine=True, tol=1e-14, maxiter=30)
    res = rel_residual(golden, x, b)
    assert res <= REFINE_TOL, (res, lu.last_refine)
    assert lu.last_refine["residual"] <= REFINE_TOL
    # forward error against the FP64 oracle of the same matrix
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    n = int(golden["n"])
    A = sp.csc_matrix((golden["data"], golden["indices"], golden["indptr"]), shape=(n, n))
    x64 = spl.spsolve(A, b)
    assert np.linalg.norm(x - x64) <= 1e-6 * np.linalg.norm(x64)


def test_transposed_solves(golden):
    import scipy.sparse as sp

    import pyglu

    n = int(golden["n"])
    A = sp.csc_matrix((golden["data"], golden["indices"], golden["indptr"]), shape=(n, n))
    lu = pyglu.GLUFactorization(*inputs(golden))
    b = golden["b"].astype(np.float64)
    x = lu.solve(b, refine=True, tol=1e-14, maxiter=30, trans="T")
    assert np.linalg.norm(A.T @ x - b) / np.linalg.norm(b) <= REFINE_TOL
    xt = lu.solve(b, trans="T")  # FP32 transposed sweeps
    assert np.linalg.norm(A.T @ xt - b) / np.linalg.norm(b) <= 1e-2


def test_multiple_rhs(golden):
    import scipy.sparse as sp

    import pyglu

    n = int(golden["n"])
    A = sp.csc_matrix((golden["data"], golden["indices"], golden["indptr"]), shape=(n, n))
    lu = pyglu.GLUFactorization(*inputs(golden))
    B = np.random.default_rng(1).uniform(-1, 1, (n, 5))
    X = lu.solve(B, refine=True, tol=1e-13, maxiter=30)
    assert X.shape == (n, 5)
    for k in range(5):
        assert np.linalg.norm(A @ X[:, k] - B[:, k]) / np.linalg.norm(B[:, k]) <= REFINE_TOL
    X1 = lu.solve(B)
    x0 = lu.solve(B[:, 0])
    assert np.allclose(X1[:, 0], x0, rtol=1e-5, atol=1e-6 * np.abs(x0).max())


def test_c_abi_from_raw_pattern(golden):
    """glu_create_from_pattern + load + factor + store, plain C-ABI calls."""
    import ctypes as C

    from pyglu import _capi

    eng = _capi.engine()
    n = int(golden["n"])
    z = golden["sym_r_idx"].size
    arrs = [np.ascontiguousarray(golden[k]) for k in ("sym_c_ptr", "sym_r_idx", "l_col_ptr", "csr_r_ptr",
                                                      "csr_c_idx", "csr_diag_ptr")]
    h = C.c_void_p()
    _capi.check(eng.glu_create_from_pattern(0, n, z, *(_capi.ptr(a) for a in arrs), 1, C.byref(h)))
    try:
        val = np.ascontiguousarray(golden["val"])
        _capi.check(eng.glu_load_lu_values(h, 0, 1, _capi.ptr(val), _capi.GLU_HOST, None))
        _capi.check(eng.glu_factor(h, 0, 1, 0, None))
        out = np.empty(z, np.float32)
        _capi.check(eng.glu_store_lu_values(h, 0, 1, _capi.ptr(out), _capi.GLU_HOST, None))
        assert col_max_rel(out, golden["lu32"], golden["sym_c_ptr"]) <= FACTOR_TOL
        nl = C.c_int32()
        lp = np.empty(golden["level_ptr"].size, np.int32)
        li = np.empty(n, np.int32)
        _capi.check(eng.glu_levels(h, C.byref(nl), _capi.ptr(lp), _capi.ptr(li)))
        assert nl.value + 1 == lp.size and np.array_equal(lp, golden["level_ptr"])
        # solve in the preprocessed system (no transform): L U y = b
        b = golden["b"].copy()
        y = np.empty_like(b)
        _capi.check(eng.glu_solve(h, 0, 1, _capi.ptr(b), _capi.ptr(y), _capi.GLU_HOST, None))
        y_orc = oracle.sweeps(golden, out, b)
        assert np.abs(y - y_orc).max() <= 1e-4 * np.abs(y_orc).max()
    finally:
        eng.glu_destroy(h)


def test_bad_calls_return_status():
    import ctypes as C

    from pyglu import _capi

    eng = _capi.engine()
    assert eng.glu_factor(None, 0, 1, 0, None) == _capi.GLU_ERR_ARG
    h = C.c_void_p()
    one = np.array([0, 1], np.uint32)
    zero = np.array([0], np.uint32)
    # diagonal pointer does not point at the diagonal
    st = eng.glu_create_from_pattern(0, 1, 1, _capi.ptr(one), _capi.ptr(np.array([0], np.uint32)),
                                     _capi.ptr(np.array([5], np.uint32)), _capi.ptr(one), _capi.ptr(zero),
                                     _capi.ptr(zero), 1, C.byref(h))
    assert st == _capi.GLU_ERR_ARG


def _raw_handle(A):
    """Symbolic phase + device handle for an already-ordered matrix (no NICSLU)."""
    import ctypes as C

    from pyglu import _capi

    eng = _capi.engine()
    A = A.tocsc()
    A.sort_indices()
    ap = A.indptr.astype(np.uint32)
    ai = A.indices.astype(np.uint32)
    ax = A.data.astype(np.float64)
    sym = C.c_void_p()
    _capi.check(eng.glu_symbolic_analyze(A.shape[0], ai.size, _capi.ptr(ap), _capi.ptr(ai), C.byref(sym)))
    nz = C.c_uint32()
    eng.glu_symbolic_sizes(sym, None, C.byref(nz))
    val = np.empty(nz.value, np.float32)
    eng.glu_predict_lu(sym, _capi.ptr(ax), _capi.ptr(val))
    h = C.c_void_p()
    _capi.check(eng.glu_create(sym, 0, 1, C.byref(h)))
    return eng, sym, h, val


def test_zero_pivot_reported_and_gesp_replaces_it():
    """[[1,1,0],[1,1,1],[0,1,2]] in natural order: column 1 meets a zero pivot
    and has an L part.  Plain factorization reports it; GESP replaces it by
    pert = 3.45e-4 * ||A||_1 (numeric.cu:490-506, 139-140)."""
    import scipy.sparse as sp

    from pyglu import _capi

    A = sp.csc_matrix(np.array([[1.0, 1.0, 0.0], [1.0, 1.0, 1.0], [0.0, 1.0, 2.0]]))
    eng, sym, h, val = _raw_handle(A)
    try:
        _capi.check(eng.glu_load_lu_values(h, 0, 1, _capi.ptr(val), _capi.GLU_HOST, None))
        assert eng.glu_factor(h, 0, 1, 0, None) == _capi.GLU_ERR_SINGULAR
        _capi.check(eng.glu_load_lu_values(h, 0, 1, _capi.ptr(val), _capi.GLU_HOST, None))
        _capi.check(eng.glu_factor(h, 0, 1, 1, None))
        out = np.empty_like(val)
        _capi.check(eng.glu_store_lu_values(h, 0, 1, _capi.ptr(out), _capi.GLU_HOST, None))
        pert = np.float32(3.45e-4) * np.float32(3.0)
        # column 1 = rows {0,1,2}: U(0,1), pivot, L(2,1)
        assert out[3] == pert
        assert np.isclose(out[4], 1.0 / pert, rtol=1e-6)
        st = _capi.Stats()
        eng.glu_get_stats(h, _capi.C.byref(st))
        assert st.pert == pert
    finally:
        eng.glu_destroy(h)
        eng.glu_symbolic_destroy(sym)


def test_singular_matrix_through_splu_raises():
    import scipy.sparse as sp

    import pyglu

    # two identical columns: structurally full rank, numerically singular
    A = sp.csc_matrix(np.array([[1.0, 1.0, 0.0], [1.0, 1.0, 0.0], [0.0, 0.0, 1.0]]))
    with pytest.raises((pyglu.SingularMatrixError, RuntimeError)):
        pyglu.splu(A)


# ------------------------------------------------------------ larger cases --
def _oracle_check(A, tol=FACTOR_TOL):
    import pyglu

    lu = pyglu.GLUFactorization(*A)
    p = lu.pattern()
    lp, li = oracle.leveling(p)
    glp, gli = lu.levels()
    assert np.array_equal(lp, glp) and np.array_equal(li, gli)
    v0 = lu.analysis.predict_lu()
    ref = oracle.factor(p, v0, lp, li, np.float32)
    v = lu.lu_values()
    err = col_max_rel(v, ref, p["sym_c_ptr"])
    assert err <= tol, err
    return lu


def test_config0_full_size_against_oracle():
    """n = 4,960 nodal matrix (dense trailing block of ~1.8k columns)."""
    from pyglu import synth

    A = synth.config0()
    lu = _oracle_check(A)
    st = lu.stats
    assert st["dense_tail"] > 1000
    b = synth.rhs_uniform(A[3], 1, seed=0)[0]
    x = lu.solve(b, refine=True, tol=1e-12, maxiter=30)
    import scipy.sparse as sp

    M = sp.csc_matrix(A[:3], shape=(A[3], A[3]))
    assert np.linalg.norm(M @ x - b) / np.linalg.norm(b) <= REFINE_TOL


def test_mesh_against_oracle():
    """Power-grid mesh (narrow levels, cluster kernel, small dense tail)."""
    from pyglu import synth

    _oracle_check(synth.grid_mesh(side=90, seed=3, n_long=40))


def test_refactor_with_new_values_matches_oracle():
    from pyglu import synth

    import pyglu

    A = synth.nodal(2500, seed=9)
    lu = pyglu.GLUFactorization(*A)
    vals = synth.perturb_values(*A, count=1, seed=4)[0]
    lu.refactor(vals)
    an = lu.analysis
    placed = np.zeros(an.nnz_lu, np.float32)
    placed[an.src_slot] = (vals * an.src_scale).astype(np.float32)
    p = an.pattern()
    lp, li = lu.levels()
    ref = oracle.factor(p, placed, lp, li, np.float32)
    assert col_max_rel(lu.lu_values(), ref, p["sym_c_ptr"]) <= FACTOR_TOL


def test_batched_same_pattern():
    import scipy.sparse as sp

    import pyglu
    from pyglu import synth

    A = synth.nodal(1500, seed=12, band=32, n_long=2, unsym_frac=0.1)
    vals = synth.perturb_values(*A, count=5, seed=1)
    bl = pyglu.BatchedGLU(A[1], A[2], A[3], vals)
    b = synth.rhs_uniform(A[3], 3, seed=2)
    B = np.broadcast_to(b, (5, 3, A[3])).copy()
    X = bl.solve(B, tol=1e-12, maxiter=30)
    for i in range(5):
        M = sp.csc_matrix((vals[i], A[1], A[2]), shape=(A[3], A[3]))
        for k in range(3):
            assert np.linalg.norm(M @ X[i, k] - b[k]) / np.linalg.norm(b[k]) <= REFINE_TOL
    # every value set's factors against the oracle's FP32 column algorithm
    from pyglu import _capi

    an = bl._an
    p = an.pattern()
    lp, li = oracle.leveling(p)
    for z in (0, 4):
        placed = np.zeros(an.nnz_lu, np.float32)
        placed[an.src_slot] = (vals[z] * an.src_scale).astype(np.float32)
        ref = oracle.factor(p, placed, lp, li, np.float32)
        vz = np.empty(an.nnz_lu, np.float32)
        _capi.check(_capi.engine().glu_store_lu_values(bl.handle, z, 1, _capi.ptr(vz), _capi.GLU_HOST, None))
        assert col_max_rel(vz, ref, p["sym_c_ptr"]) <= FACTOR_TOL, z


def test_adjoint_gradient_matches_finite_differences():
    import torch

    import pyglu
    from pyglu import synth

    A = synth.nodal(120, seed=21)
    data, indices, indptr, n = A
    lu = pyglu.GLUFactorization(*A)
    rng = np.random.default_rng(3)
    w = torch.tensor(rng.standard_normal(n), dtype=torch.float64)
    vals = torch.tensor(data, dtype=torch.float64, requires_grad=True)
    b = torch.tensor(rng.uniform(-1, 1, n), dtype=torch.float64, requires_grad=True)
    x = pyglu.sparse_solve(vals, b, lu)
    loss = (w * x).sum()
    loss.backward()
    gv, gb = vals.grad.numpy().copy(), b.grad.numpy().copy()

    # FP64 central differences with a direct FP64 solver, step 1e-6 relative.
    # Cancellation limits an FP64 difference quotient to about
    # 1e-10 * |f| / |v_q g_q| relative error, so entries are drawn among those
    # whose relative sensitivity |v_q g_q| / |f| is at least 1e-3.
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    bn = b.detach().numpy()
    wn = w.numpy()

    def f(v, bb):
        M = sp.csc_matrix((v, indices, indptr), shape=(n, n))
        return float(wn @ spl.spsolve(M, bb))

    f0 = abs(float(loss))
    sens = np.abs(data * gv) / f0
    cand = np.nonzero(sens >= 1e-3)[0]
    assert cand.size >= 8
    for q in rng.choice(cand, min(16, cand.size), replace=False):
        h = 1e-6 * abs(data[q])
        vp, vm = data.copy(), data.copy()
        vp[q] += h
        vm[q] -= h
        fd = (f(vp, bn) - f(vm, bn)) / (2 * h)
        assert abs(fd - gv[q]) <= 1e-6 * abs(fd), (q, fd, gv[q])
    for i in rng.choice(n, 16, replace=False):
        h = 1e-6 * max(abs(bn[i]), 1e-3)
        bp, bm = bn.copy(), bn.copy()
        bp[i] += h
        bm[i] -= h
        fd = (f(data, bp) - f(data, bm)) / (2 * h)
        assert abs(fd - gb[i]) <= 1e-6 * max(abs(fd), 1e-8 * np.abs(gb).max()), (i, fd, gb[i])
    # dense torch.linalg.solve gradient
    import scipy.sparse as sp

    M = torch.tensor(sp.csc_matrix((data, indices, indptr), shape=(n, n)).toarray(), requires_grad=True)
    bb = b.detach().clone().requires_grad_(True)
    xd = torch.linalg.solve(M, bb)
    (w * xd).sum().backward()
    rows = indices
    cols = np.repeat(np.arange(n), np.diff(indptr))
    gdense = M.grad.numpy()[rows, cols]
    assert np.allclose(gv, gdense, rtol=1e-6, atol=1e-9 * np.abs(gdense).max())
    assert np.allclose(gb, bb.grad.numpy(), rtol=1e-6, atol=1e-12)
