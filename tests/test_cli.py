"""lu_cmd (the reference's CLI surface, src/lu_cmd.cpp) and the drop-in build of
the reference's own lu_cmd.cpp + symbolic.cc against the engine through
include/glu_luondevice.hpp."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

LU_CMD = os.path.join(ROOT, "glu-hcu_b200", "bin", "lu_cmd")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "lu_cmd_dropin")


def run(cmd, cwd):
    return subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600)


def test_usage_and_bad_arguments(tmp_path):
    r = run([LU_CMD], tmp_path)
    assert r.returncode == 255 and "Usage" in r.stdout
    r = run([LU_CMD, "-x", "y"], tmp_path)
    assert r.returncode == 255
    r = run([LU_CMD, "-i", str(tmp_path / "missing.mtx")], tmp_path)
    assert r.returncode == 255 and "File cannot open" in r.stderr
    assert not (tmp_path / "x.dat").exists()


def test_mtx_round_trip(tmp_path):
    import pyglu
    from pyglu import synth

    A = synth.nodal(300, seed=4)
    p = tmp_path / "a.mtx"
    pyglu.write_mtx(p, *A)
    data, indices, indptr, n = pyglu.read_mtx(p)
    assert n == A[3]
    assert np.array_equal(indptr, A[2]) and np.array_equal(indices, A[1])
    assert np.array_equal(data, A[0])


def _mtx(tmp_path, n=1500, seed=8):
    import pyglu
    from pyglu import synth

    A = synth.nodal(n, seed=seed)
    p = tmp_path / "a.mtx"
    pyglu.write_mtx(p, *A)
    return A, p


def _residual(A, x):
    import scipy.sparse as sp

    M = sp.csc_matrix(A[:3], shape=(A[3], A[3]))
    b = np.ones(A[3])
    return np.linalg.norm(M @ x - b) / np.linalg.norm(b)


@pytest.mark.gpu
def test_lu_cmd_solves_and_writes_x(tmp_path):
    A, p = _mtx(tmp_path)
    r = run([LU_CMD, "-i", str(p)], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "Total GPU time" in r.stdout and "Number of levels" in r.stdout
    # x.dat keeps 6 significant digits (default stream formatting), so compare
    # values, not residuals
    import pyglu
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    x = np.loadtxt(tmp_path / "x.dat")
    assert x.shape == (A[3],)
    x32 = pyglu.splu(A[:3] + ((A[3], A[3]),)).solve(np.ones(A[3]))
    assert np.abs(x - x32).max() <= 1e-4 * np.abs(x32).max()
    r = run([LU_CMD, "-i", str(p), "-r", "-t", "1e-12"], tmp_path)
    assert r.returncode == 0, r.stderr
    x = np.loadtxt(tmp_path / "x.dat")
    x64 = spl.spsolve(sp.csc_matrix(A[:3], shape=(A[3], A[3])), np.ones(A[3]))
    assert np.abs(x - x64).max() <= 1e-5 * np.abs(x64).max()
    r = run([LU_CMD, "-i", str(p), "-p"], tmp_path)
    assert r.returncode == 0 and "GESP" in r.stdout


@pytest.mark.gpu
def test_reference_lu_cmd_links_against_engine(tmp_path):
    """The reference's unmodified lu_cmd.cpp and symbolic.cc, with LUonDevice
    from the shim: same outputs as the engine's own CLI."""
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in build not present")
    A, p = _mtx(tmp_path)
    d1 = tmp_path / "ref"
    d2 = tmp_path / "ours"
    d1.mkdir()
    d2.mkdir()
    r = run([DROPIN, "-i", str(p)], d1)
    assert r.returncode == 0, r.stderr
    assert "Total GPU time" in r.stdout
    r2 = run([LU_CMD, "-i", str(p)], d2)
    assert r2.returncode == 0, r2.stderr
    x_ref = np.loadtxt(d1 / "x.dat")
    x_ours = np.loadtxt(d2 / "x.dat")
    assert np.isfinite(x_ref).all() and _residual(A, x_ref) <= 5e-2  # 6-digit output
    assert np.abs(x_ref - x_ours).max() <= 1e-3 * np.abs(x_ref).max()
    for line in ("Symbolic nonzero", "Number of levels"):
        a = [l for l in r.stdout.splitlines() if line in l]
        b = [l for l in r2.stdout.splitlines() if line in l]
        assert a and b and a[0].split(":")[1].strip() == b[0].split(":")[1].strip(), line
