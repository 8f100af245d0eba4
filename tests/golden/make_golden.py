"""Generate the golden fixtures in tests/golden/ (run here, where the reference
is built into oracle/_ref).

Each case stores a seeded synthetic matrix and what the reference's own CPU
code computes for it -- NICSLU's preprocessed matrix, permutations and scales,
the Symbolic_Matrix pattern, levels and predictLU values, and
Symbolic_Matrix::solve on the oracle's FP32 factors -- together with the
oracle's FP32 and FP64 factors (numeric.cu semantics, sequential in level
order) and the GESP-perturbed FP32 factors.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "glu-hcu_b200"))

import oracle  # noqa: E402
from pyglu import synth  # noqa: E402

CASES = {
    "nodal_n200": lambda: synth.nodal(200, seed=3),
    "nodal_n600": lambda: synth.nodal(600, seed=4, band=16, n_long=1),
    "nodal_n1200": lambda: synth.nodal(1200, seed=5, band=24, n_long=1, unsym_frac=0.1),
    "mesh_24": lambda: synth.grid_mesh(side=24, seed=6, n_long=12),
    "nodal2_n500": lambda: synth.nodal(500, seed=7, band=32, n_band=2, n_long=2, unsym_frac=0.1),
}


def make(name, A):
    data, indices, indptr, n = A
    r = oracle.RefGLU(data, indices, indptr, n)
    s = r.symbolic()
    lu32 = oracle.factor(s, s["val"], s["level_ptr"], s["level_idx"], np.float32)
    lu64 = oracle.factor(s, s["val"].astype(np.float64), s["level_ptr"], s["level_idx"], np.float64)
    pert = oracle.pert(s, s["val"])
    lu32p = oracle.factor(s, s["val"], s["level_ptr"], s["level_idx"], np.float32, pert=pert)
    rng = np.random.default_rng(100 + n)
    b = rng.uniform(-1, 1, n).astype(np.float32)
    x_ref = r.solve(lu32, b)
    out = dict(data=data, indices=indices, indptr=indptr, n=np.int64(n),
               pax=r.ax, pai=r.ai, pap=r.ap, b=b, x_ref=x_ref, lu32=lu32, lu64=lu64,
               lu32_pert=lu32p, pert=np.float32(pert))
    for k in ("col_perm", "row_perm_inv", "pivot", "col_scale_perm", "row_scale", "row_perm"):
        out[k] = r.perm[k]
    out["mc64"] = np.int64(r.perm["mc64"])
    for k in ("sym_c_ptr", "sym_r_idx", "l_col_ptr", "csr_r_ptr", "csr_c_idx", "csr_diag_ptr", "val",
              "level_ptr", "level_idx"):
        out[k] = s[k]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: n={n} nnzA={data.size} nnzLU={s['nnz']} levels={s['num_lev']}")


if __name__ == "__main__":
    for name, gen in CASES.items():
        make(name, gen())
