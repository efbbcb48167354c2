"""Runs the oracle (the reference's OpenMP BlockLanczos, default ModifiedGS, single-pass
CholQR) to convergence on the 96^3 anisotropic Laplacian with axis coefficients (1, 10, 100):
bs 8, nev 32, ncv 384, tol 1e-10, start block problems.initial_block(n, 8, seed=42).
Writes tests/golden/aniso96_reference.json: restart and operator-apply counts, wall time and
thread count of this host, and the 32 eigenvalues.

    OMP_NUM_THREADS=8 python tests/golden/make_aniso96_reference.py
"""
import json
import os
import platform
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from trl_b200 import problems as P  # noqa: E402


def main():
    A = P.anisotropic3d(96)
    X0 = P.initial_block(A.n, 8, seed=42)
    t = time.time()
    r = O.solve_csr(A, 8, 32, 384, X0, tol=1e-10, max_restarts=1000)
    wall = time.time() - t
    exact = P.anisotropic3d_eigenvalues(96, k=32)
    cpu = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            cpu = next(line.split(":", 1)[1].strip() for line in f if line.startswith("model name"))
    except Exception:
        pass
    out = {
        "workload": "anisotropic3d 96^3 coef (1,10,100), bs 8, nev 32, ncv 384, tol 1e-10, seed 42",
        "converged": r["converged"],
        "restarts": r["iterations"],
        "n_op_apply": r["n_op_apply"],
        "solve_seconds": r["seconds"],
        "wall_seconds": wall,
        "threads": O.num_threads(),
        "cpu": cpu,
        "host": platform.node(),
        "evals": r["evals"][:32].tolist(),
        "max_rel_err_vs_analytic": float(np.max(np.abs(r["evals"][:32] - exact) / exact)),
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "aniso96_reference.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({k: v for k, v in out.items() if k != "evals"}))


if __name__ == "__main__":
    main()
