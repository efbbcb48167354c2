"""The CPU oracle, pinned before it is trusted.

The oracle runs the reference's own code (lanczos.hh + the OpenMP backend, compiled in place)
on an Eigen-free restatement of evp_base.hh. It is pinned by
  * the reference's own test programs (tests/openmp/test_lanczos_{convergence,extend}.cc),
    compiled unchanged against the restatement: every case must pass;
  * the analytic spectra the reference tests use and that the benchmark configs have;
  * the dense routines against numpy (LAPACK) on random symmetric matrices;
  * committed golden vectors (tests/golden/) produced by the oracle at fixed seeds.
"""
import os
import subprocess

import numpy as np
import pytest

from trl_b200 import problems as P

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_reference_test_programs_pass(oracle):
    for exe in oracle.REF_TESTS:
        assert os.path.exists(exe), exe
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300, env=dict(os.environ, OMP_NUM_THREADS="4"))
        assert r.returncode == 0, r.stdout[-2000:]
        assert "not passed" not in r.stdout.lower()


def test_reference_convergence_program_output(oracle):
    exe = oracle.REF_TESTS[0]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300, env=dict(os.environ, OMP_NUM_THREADS="4"))
    # 8 cases: Diagonal and Laplace1D at bs 1, 2, 4, 8 (tests/openmp/test_lanczos_convergence.cc:69-78)
    assert r.stdout.count(" passed.") == 8
    assert "ALL PASSED" in r.stdout


@pytest.mark.parametrize("n", [1, 2, 5, 17, 64])
def test_dense_symmetric_eigen_matches_lapack(oracle, n):
    rng = np.random.default_rng(n)
    M = rng.standard_normal((n, n))
    A = M + M.T
    w, V = oracle.symmetric_eigen(A)
    wr = np.linalg.eigvalsh(A)
    assert np.allclose(w, wr, rtol=0, atol=1e-12 * max(1.0, np.abs(wr).max()))
    assert np.allclose(A @ V, V * w, atol=1e-11 * max(1.0, np.abs(wr).max()))
    assert np.allclose(V.T @ V, np.eye(n), atol=1e-12)


def test_dense_eigen_reads_lower_triangle(oracle):
    rng = np.random.default_rng(3)
    M = rng.standard_normal((6, 6))
    L = np.tril(M)
    w, _ = oracle.symmetric_eigen(L + np.triu(rng.standard_normal((6, 6)), 1) * 100)  # upper garbage ignored
    assert np.allclose(w, np.linalg.eigvalsh(np.tril(L) + np.tril(L, -1).T), atol=1e-12)


def test_dense_eigen_degenerate(oracle):
    A = np.diag([3.0, 1.0, 3.0, 2.0, 1.0])
    w, V = oracle.symmetric_eigen(A)
    assert np.allclose(w, [1, 1, 2, 3, 3])
    assert np.allclose(V.T @ V, np.eye(5), atol=1e-14)


@pytest.mark.parametrize("bs", [1, 2, 4, 8, 16])
def test_orthonormalize_is_cholqr(oracle, bs):
    rng = np.random.default_rng(bs)
    V = rng.standard_normal((257, bs))
    V0 = V.copy()
    R = oracle.orthonormalize(V)
    assert np.allclose(V.T @ V, np.eye(bs), atol=1e-12)
    assert np.allclose(np.tril(R, -1), 0)
    assert np.allclose(V @ R, V0, atol=1e-12)  # V_old = V_new R (concepts.hh:153-155)


def test_orthonormalize_breakdown_raises(oracle):
    V = np.zeros((50, 4))
    with pytest.raises(RuntimeError, match="Cholesky"):
        oracle.orthonormalize(V)


def test_small_dense_order_and_count(oracle):
    rng = np.random.default_rng(7)
    bs, nblk = 4, 6
    N = bs * nblk
    M = rng.standard_normal((N, N))
    D = M + M.T
    T = D.reshape(nblk, bs, nblk, bs).transpose(0, 2, 1, 3).copy()
    beta = np.triu(rng.standard_normal((bs, bs))) * 1e-9
    evals, evecs, nconv = oracle.solve_small_dense(T, beta, bs, nev=8, tol=1e-6)
    wr = np.linalg.eigvalsh(D)
    assert np.allclose(np.sort(np.abs(evals))[::-1], np.abs(evals))  # |theta| descending (evp_base.hh:103)
    assert np.allclose(np.sort(evals), wr, atol=1e-12)
    Y = evecs.transpose(0, 2, 1, 3).reshape(N, N)
    assert np.allclose(D @ Y, Y * evals, atol=1e-11)
    assert nconv == 8


def test_oracle_solves_laplace128_to_analytic(oracle):
    A = P.laplace2d(128)
    X0 = P.initial_block(A.n, 4, seed=42)
    r = oracle.solve_csr(A, 4, 10, 160, X0, tol=1e-8)
    assert r["converged"]
    exact = P.laplace2d_eigenvalues(128)[:10]
    assert np.max(np.abs(r["evals"][:10] - exact) / exact) < 1e-10


def test_golden_vectors(oracle):
    """Re-run the oracle on the committed golden inputs and compare bit-for-bit-ish."""
    path = os.path.join(GOLDEN, "oracle_golden.npz")
    g = np.load(path)
    for bs in (1, 2, 4, 8, 16):
        X = g[f"X_{bs}"].copy()
        Y = g[f"Y_{bs}"].copy()
        W = g[f"W_{bs}"].copy()
        R = np.zeros((bs, bs))
        oracle.block_view_op(bs, oracle.OP_DOT, X, Y, R)
        assert np.allclose(R, g[f"dot_{bs}"], rtol=1e-13, atol=1e-13)
        Z = np.zeros_like(X)
        oracle.block_view_op(bs, oracle.OP_MULT, X, Z, W)
        assert np.allclose(Z, g[f"mult_{bs}"], rtol=1e-13, atol=1e-13)
        V = X.copy()
        Rq = oracle.orthonormalize(V)
        assert np.allclose(V, g[f"orth_V_{bs}"], atol=1e-12)
        assert np.allclose(Rq, g[f"orth_R_{bs}"], atol=1e-12)
    A = P.laplace2d(16)
    r = oracle.solve_csr(A, 4, 6, 24, g["solve_X0"], tol=1e-10)
    assert np.allclose(r["evals"][:6], g["solve_evals"], rtol=1e-12)
    assert r["iterations"] == int(g["solve_iterations"])


def test_oracle_minner_solves_the_generalised_problem(oracle):
    """The reference driver with dot = V^T (M W) (examples/openmp/csrevp.hh:89-97) on
    op = M^{-1} K with a non-diagonal SPD M gives the generalised eigenpairs of (K, M) with
    M-orthonormal Ritz vectors."""
    import scipy.linalg as sl

    K, M = P.diffusion2d_consistent_mass(12, seed=3)
    Kd, Md = K.to_dense(), M.to_dense()
    Op = P.dense_csr(np.linalg.solve(Md, Kd))
    X0 = P.initial_block(K.n, 4, seed=5)
    r = oracle.solve_csr_minner(Op, M, 4, 8, 48, X0, tol=1e-10)
    assert r["converged"]
    lam = sl.eigh(Kd, Md, eigvals_only=True)[::-1][:8]
    assert np.max(np.abs(r["evals"][:8] - lam) / lam) < 1e-10
    X = r["ritz"]
    assert np.abs(X.T @ Md @ X - np.eye(8)).max() < 1e-10
