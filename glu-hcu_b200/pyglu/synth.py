"""Seeded synthetic circuit and power-grid matrices.

These stand in for the circuit matrices the reference is benchmarked on.  Each
generator returns an n x n CSC matrix as ``(data f64, indices i32, indptr i32,
n)`` with sorted row indices and no duplicates, which is the form
``pyglu._to_csc_arrays`` produces from a scipy matrix (pyglu/__init__.py:30-63
in the reference).

* :func:`nodal` -- a nodal-analysis matrix: every node is linked to
  ``n_band`` neighbours within ``|i-j| <= band`` plus ``n_long`` uniformly
  random nodes; each link stamps a conductance ``g`` (log-uniform in
  ``g_range``) as ``-g`` at (i,j) and (j,i); a fraction ``unsym_frac`` of the
  rows gets one extra controlled-source entry of random sign and magnitude
  log-uniform in ``cs_range``; the diagonal is the sum of the absolute row
  off-diagonals plus a shunt log-uniform in ``shunt_range``.
* :func:`grid_mesh` -- a ``side x side`` resistive power grid (5-point
  stencil), a fraction of via/pad nodes tied to ground and a number of
  uniformly random long-range couplings.
* :func:`perturb_values` -- same-pattern value sets for batched
  refactorization: every nonzero times an independent lognormal factor, with
  diagonal dominance re-imposed.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _log_uniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


def _to_csc(rows, cols, vals, n):
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsc()
    A.sum_duplicates()
    A.sort_indices()
    return (np.ascontiguousarray(A.data, dtype=np.float64),
            np.ascontiguousarray(A.indices, dtype=np.int32),
            np.ascontiguousarray(A.indptr, dtype=np.int32), n)


def nodal(n: int, seed: int = 0, band: int = 16, n_band: int = 2, n_long: int = 1,
          unsym_frac: float = 0.05, g_range=(1e-6, 1e2), shunt_range=(1e-9, 1e-3),
          cs_range=(1e-4, 1e1)):
    """Synthetic nodal-analysis matrix (see module docstring)."""
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.int64)
    src, dst = [], []
    for _ in range(n_band):
        off = rng.integers(1, band + 1, n) * rng.choice(np.array([-1, 1]), n)
        j = i + off
        j = np.where((j < 0) | (j >= n), i - off, j)  # reflect at the ends
        src.append(i)
        dst.append(j)
    for _ in range(n_long):
        j = rng.integers(0, n - 1, n)
        j = j + (j >= i)  # uniform over the other nodes
        src.append(i)
        dst.append(j)
    src = np.concatenate(src)
    dst = np.concatenate(dst)
    keep = (src != dst) & (dst >= 0) & (dst < n)
    src, dst = src[keep], dst[keep]
    g = _log_uniform(rng, g_range[0], g_range[1], src.size)
    rows = np.concatenate([src, dst])
    cols = np.concatenate([dst, src])
    vals = -np.concatenate([g, g])
    # controlled sources: one unsymmetric entry in a fraction of the rows
    ncs = int(round(unsym_frac * n))
    cs_rows = rng.choice(n, size=ncs, replace=False)
    cs_off = rng.integers(1, band + 1, ncs) * rng.choice(np.array([-1, 1]), ncs)
    cs_cols = cs_rows + cs_off
    cs_cols = np.where((cs_cols < 0) | (cs_cols >= n), cs_rows - cs_off, cs_cols)
    cs_vals = _log_uniform(rng, cs_range[0], cs_range[1], ncs) * rng.choice(np.array([-1.0, 1.0]), ncs)
    rows = np.concatenate([rows, cs_rows])
    cols = np.concatenate([cols, cs_cols])
    vals = np.concatenate([vals, cs_vals])
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    A.sum_duplicates()
    rowabs = np.asarray(abs(A).sum(axis=1)).ravel()
    shunt = _log_uniform(rng, shunt_range[0], shunt_range[1], n)
    A = (A + sp.diags(rowabs + shunt)).tocoo()
    return _to_csc(A.row, A.col, A.data, n)


def grid_mesh(side: int = 700, seed: int = 0, seg_range=(1.0, 1e3), via_frac=0.005,
              via_range=(1e2, 1e4), n_long: int = 2000, long_range=(1e-3, 1.0)):
    """Resistive power-grid mesh (5-point stencil) with vias and long couplings."""
    rng = np.random.default_rng(seed)
    n = side * side
    idx = np.arange(n, dtype=np.int64).reshape(side, side)
    h_a, h_b = idx[:, :-1].ravel(), idx[:, 1:].ravel()
    v_a, v_b = idx[:-1, :].ravel(), idx[1:, :].ravel()
    a = np.concatenate([h_a, v_a])
    b = np.concatenate([h_b, v_b])
    g = _log_uniform(rng, seg_range[0], seg_range[1], a.size)
    la = rng.integers(0, n, n_long)
    lb = rng.integers(0, n - 1, n_long)
    lb = lb + (lb >= la)
    lg = _log_uniform(rng, long_range[0], long_range[1], n_long)
    a = np.concatenate([a, la])
    b = np.concatenate([b, lb])
    g = np.concatenate([g, lg])
    diag = np.zeros(n)
    np.add.at(diag, a, g)
    np.add.at(diag, b, g)
    nvia = int(round(via_frac * n))
    vias = rng.choice(n, size=nvia, replace=False)
    diag[vias] += _log_uniform(rng, via_range[0], via_range[1], nvia)
    rows = np.concatenate([a, b, np.arange(n)])
    cols = np.concatenate([b, a, np.arange(n)])
    vals = np.concatenate([-g, -g, diag])
    return _to_csc(rows, cols, vals, n)


def perturb_values(data, indices, indptr, n, count: int, seed: int = 0, sigma: float = 0.2):
    """``count`` value sets on the pattern of (data, indices, indptr).

    Every nonzero is multiplied by an independent lognormal(0, sigma) factor;
    then diagonal dominance is re-imposed: each diagonal becomes the absolute
    sum of its row's (perturbed) off-diagonals plus the row's original excess
    (diagonal minus absolute off-diagonal sum: the shunt, or the via
    conductance) times its own lognormal factor.  Returns shape (count, nnz).
    """
    rng = np.random.default_rng(seed)
    nnz = data.size
    cols = np.repeat(np.arange(n), np.diff(indptr))
    rows = indices.astype(np.int64)
    is_diag = rows == cols
    off0 = np.bincount(rows, weights=np.where(is_diag, 0.0, np.abs(data)), minlength=n)
    diag0 = np.zeros(n)
    diag0[rows[is_diag]] = data[is_diag]
    excess0 = np.maximum(diag0 - off0, 0.0)
    out = np.empty((count, nnz), dtype=np.float64)
    for b in range(count):
        f = rng.lognormal(0.0, sigma, nnz)
        v = data * f
        rowabs = np.bincount(rows, weights=np.where(is_diag, 0.0, np.abs(v)), minlength=n)
        d = rows[is_diag]
        v[is_diag] = rowabs[d] + excess0[d] * f[is_diag]
        out[b] = v
    return out


def rhs_uniform(n: int, nrhs: int = 1, seed: int = 0):
    """Right-hand sides uniform in [-1, 1], shape (nrhs, n)."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, (nrhs, n))


def rhs_loads(n: int, seed: int = 0, mean: float = 1e-3):
    """Current loads: negated exponential with the given mean."""
    return -np.random.default_rng(seed).exponential(mean, n)


# Workload presets with the sizes the benchmarks use.
def config0(seed: int = 0):
    """Nodal matrix, n=4,960, band 16, 2 band links + 1 long link, 5% unsymmetric rows."""
    return nodal(4960, seed=seed, band=16, n_band=2, n_long=1, unsym_frac=0.05)


def config1(seed: int = 0, side: int = 700):
    """700 x 700 power-grid mesh, n=490,000."""
    return grid_mesh(side=side, seed=seed)


def config2_pattern(seed: int = 0, n: int = 20000):
    """Nodal matrix, n=20,000, band 32, 2 band links + 2 long links, 10% unsymmetric rows."""
    return nodal(n, seed=seed, band=32, n_band=2, n_long=2, unsym_frac=0.10)


def config3_systems(count: int = 64, seed: int = 0, n_range=(2000, 50000), rhs_range=(1, 64)):
    """``count`` nodal systems with n log-uniform in n_range and 1..64 right-hand sides."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]), count)).astype(np.int64)
    nrhs = rng.integers(rhs_range[0], rhs_range[1] + 1, count)
    return [(int(ns[s]), int(nrhs[s]), seed * 1000 + s) for s in range(count)]


def config4(seed: int = 0, n: int = 100000):
    """Nodal matrix, n=100,000, band 24, 5% unsymmetric rows."""
    return nodal(n, seed=seed, band=24, n_band=2, n_long=1, unsym_frac=0.05)
