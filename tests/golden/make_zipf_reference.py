"""Runs the oracle (the reference's OpenMP BlockLanczos, default ModifiedGS, single-pass
CholQR) to convergence on the Zipf(1.5) random symmetric pattern with n = 524,288 rows
(problems.zipf_symmetric(524288, seed=42), degrees capped at 512, N(0,1) values mirrored):
bs 8, nev 100 (largest magnitude, both ends of an indefinite spectrum), ncv 256, tol 1e-10,
start block problems.initial_block(n, 8, seed=42). Writes
tests/golden/zipf524k_b8_reference.json: restart and operator-apply counts, the largest
true residual ||Ax - theta x|| / |theta| of the reference's Ritz pairs, and the 100
eigenvalues. Takes about 11 minutes on 8 host cores.

    python tests/golden/make_zipf_reference.py
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from trl_b200 import problems as P  # noqa: E402


def main():
    n, bs, nev, ncv = 524288, 8, 100, 256
    A = P.zipf_symmetric(n, seed=42)
    X0 = P.initial_block(n, bs, seed=42)
    t = time.time()
    r = O.solve_csr(A, bs, nev, ncv, X0, tol=1e-10, max_restarts=3000, ritz=True)
    wall = time.time() - t
    ev = r["evals"][:nev]
    X = r["ritz"]
    res = np.linalg.norm(A.matmat(X) - X * ev, axis=0) / np.linalg.norm(X, axis=0) / np.abs(ev)
    out = {"workload": f"zipf_symmetric n={n} nnz={A.nnz} seed 42, bs {bs}, nev {nev}, ncv {ncv}, tol 1e-10, start block seed 42",
           "converged": bool(r["converged"]), "restarts": r["iterations"], "n_op_apply": r["n_op_apply"], "solve_seconds": r["seconds"],
           "wall_seconds": wall, "threads": O.num_threads(), "max_theta_residual": float(res.max()), "evals": [float(x) for x in ev]}
    with open(os.path.join(ROOT, "tests", "golden", "zipf524k_b8_reference.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({k: v for k, v in out.items() if k != "evals"}))


if __name__ == "__main__":
    main()
