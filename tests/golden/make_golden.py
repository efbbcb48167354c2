"""Generates tests/golden/oracle_golden.npz from the oracle (the reference's OpenMP backend
compiled in place; see oracle/Makefile). Run from the repository root:

    python tests/golden/make_golden.py

Contents (fixed seeds): for bs in {1, 2, 4, 8, 16}, inputs X, Y (n=37 x bs), W (bs x bs) and
the reference's BlockView::dot / mult outputs (impl/openmp/blockview.hh:104-182) and the
restated orthonormalize (evp_base.hh:39-71) on X; and one full BlockLanczos solve of the
16x16 2-D Laplacian (bs=4, nev=6, ncv=24, tol 1e-10) — eigenvalues and restart count.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from trl_b200 import problems as P  # noqa: E402


def main():
    if not O.available():
        O.build()
    out = {}
    rng = np.random.default_rng(2024)
    for bs in (1, 2, 4, 8, 16):
        X = rng.standard_normal((37, bs))
        Y = rng.standard_normal((37, bs))
        W = rng.standard_normal((bs, bs))
        out[f"X_{bs}"], out[f"Y_{bs}"], out[f"W_{bs}"] = X, Y, W
        R = np.zeros((bs, bs))
        O.block_view_op(bs, O.OP_DOT, X.copy(), Y.copy(), R)
        out[f"dot_{bs}"] = R
        Z = np.zeros_like(X)
        O.block_view_op(bs, O.OP_MULT, X.copy(), Z, W.copy())
        out[f"mult_{bs}"] = Z
        V = X.copy()
        out[f"orth_R_{bs}"] = O.orthonormalize(V)
        out[f"orth_V_{bs}"] = V
    A = P.laplace2d(16)
    X0 = np.random.default_rng(7).standard_normal((A.n, 4))
    r = O.solve_csr(A, 4, 6, 24, X0, tol=1e-10)
    out["solve_X0"] = X0
    out["solve_evals"] = r["evals"][:6]
    out["solve_iterations"] = np.array(r["iterations"])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, "solve:", r["iterations"], "restarts", r["evals"][:6])


if __name__ == "__main__":
    main()
