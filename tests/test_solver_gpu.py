"""End-to-end parity of the CUDA backend driven by the reference's unchanged BlockLanczos.

* The reference's own test bodies (tests/test_lanczos_{convergence,extend}.hh) run on the
  CUDA backend (trl_b200/lib/trl_cuda_ref_tests) with the reference's cases and tolerances.
* The small benchmark workload (2-D 5-point Laplacian 128x128, bs 4, nev 10, ncv 160) is
  solved by the oracle (reference OpenMP backend) and by the CUDA backend from the same
  start block: eigenvalues agree to 1e-10 relative, eigenvector subspaces by principal
  angles per eigenvalue cluster, residuals ||Ax - lambda x|| / ||A||_1 below the tolerance.
"""
import json
import os
import pathlib
import subprocess

import numpy as np
import pytest
import torch

from trl_b200 import native
from trl_b200 import problems as P

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).parent / "golden"


def _run(args):
    return subprocess.run(args, capture_output=True, text=True, timeout=600)


def test_reference_test_bodies_fp64():
    r = _run([native.REF_TESTS_BIN])
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "ALL PASSED" in r.stdout
    assert r.stdout.count(" passed.") == 8 and r.stdout.count("Passed.") == 4


def test_reference_test_bodies_fp32():
    r = _run([native.REF_TESTS_BIN, "fp32"])
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "ALL PASSED" in r.stdout


def clusters(evals, rel=1e-8):
    groups, cur = [], [0]
    for i in range(1, len(evals)):
        if abs(evals[i] - evals[i - 1]) <= rel * abs(evals[0]):
            cur.append(i)
        else:
            groups.append(cur)
            cur = [i]
    groups.append(cur)
    return groups


def max_principal_sine(Xa, Xb, evals):
    """max over eigenvalue clusters of sin(largest principal angle) between the two spans."""
    worst = 0.0
    for g in clusters(evals):
        Qa, _ = np.linalg.qr(Xa[:, g])
        Qb, _ = np.linalg.qr(Xb[:, g])
        s = np.linalg.norm(Qb - Qa @ (Qa.T @ Qb), 2)
        worst = max(worst, s)
    return worst


@pytest.fixture(scope="module")
def laplace128_oracle(oracle):
    A = P.laplace2d(128)
    X0 = P.initial_block(A.n, 4, seed=42)
    r = oracle.solve_csr(A, 4, 10, 160, X0, tol=1e-8, ritz=True)
    assert r["converged"]
    return A, X0, r


@pytest.mark.parametrize("reorth", [native.TRL_REORTH_CGS2, native.TRL_REORTH_CGS_IFNEEDED, native.TRL_REORTH_MGS, native.TRL_REORTH_PARTIAL])
@pytest.mark.parametrize("passes", [1, 2])
def test_laplace128_fp64_matches_oracle(laplace128_oracle, reorth, passes):
    A, X0, ref = laplace128_oracle
    out = native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-8, reorth=reorth, cholqr_passes=passes)
    assert out["converged"]
    exact = P.laplace2d_eigenvalues(128)[:10]
    assert np.max(np.abs(out["evals"] - ref["evals"][:10]) / np.abs(ref["evals"][:10])) < 1e-10
    assert np.max(np.abs(out["evals"] - exact) / exact) < 1e-10
    # the Ritz estimate test is ||beta y|| / |theta| < tol; true residuals sit at that level
    assert out["max_theta_residual"] < 5e-8
    assert np.max(out["resid"]) < 5e-8
    assert max_principal_sine(out["evecs"], ref["ritz"], out["evals"]) < 1e-5
    # same number of restarts as the reference up to small drift from rounding
    assert abs(out["restarts"] - ref["iterations"]) <= max(3, ref["iterations"] // 5)


@pytest.mark.parametrize("pairs", [0, 1])
def test_partial_reorthogonalisation_with_and_without_pairs(laplace128_oracle, pairs):
    """partial_pairs = 1 (default) also projects the step after each fired sketch test; both
    settings give the reference's eigenpairs with orthonormal Ritz vectors."""
    A, X0, ref = laplace128_oracle
    out = native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-8, reorth=native.TRL_REORTH_PARTIAL, partial_pairs=pairs)
    assert out["converged"]
    assert np.max(np.abs(out["evals"] - ref["evals"][:10]) / np.abs(ref["evals"][:10])) < 1e-10
    assert np.max(out["resid"]) < 5e-8
    X = out["evecs"]
    assert np.abs(X.T @ X - np.eye(10)).max() < 1e-10
    assert abs(out["restarts"] - ref["iterations"]) <= max(3, ref["iterations"] // 5)


def test_eigenvectors_into_the_callers_buffer(laplace128_oracle):
    """evecs_out (here page-locked, as a repeated caller keeps it) receives exactly what the
    allocating call returns, and is returned itself."""
    import torch

    A, X0, ref = laplace128_oracle
    kw = dict(bs=4, nev=10, ncv=160, tol=1e-8)
    buf = torch.full((A.n, 10), float("nan"), dtype=torch.float64).pin_memory().numpy()
    mine = native.solve_csr_host(A, X0, evecs_out=buf, **kw)
    fresh = native.solve_csr_host(A, X0, **kw)
    assert mine["evecs"] is buf
    assert np.array_equal(buf, fresh["evecs"])
    assert np.array_equal(mine["evals"], fresh["evals"])


@pytest.mark.parametrize("reorth", [native.TRL_REORTH_CGS_IFNEEDED, native.TRL_REORTH_MGS])
def test_fused_and_call_by_call_execution_agree(laplace128_oracle, reorth):
    """batching = 1 fuses the three-term step's product/subtract pairs (deferring the
    temporary) and the restart rotation; batching = 0 issues every driver call as its own
    kernel. Both must give the reference's eigenpairs."""
    A, X0, ref = laplace128_oracle
    outs = [native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-8, reorth=reorth, batching=b) for b in (0, 1)]
    for out in outs:
        assert out["converged"]
        assert np.max(np.abs(out["evals"] - ref["evals"][:10]) / np.abs(ref["evals"][:10])) < 1e-10
        assert np.max(out["resid"]) < 5e-8
    assert max_principal_sine(outs[0]["evecs"], outs[1]["evecs"], outs[0]["evals"]) < 1e-5
    assert abs(outs[0]["restarts"] - outs[1]["restarts"]) <= 2
    if reorth == native.TRL_REORTH_CGS_IFNEEDED:
        assert outs[1]["kernel_launches"] < outs[0]["kernel_launches"]


def test_laplace128_mixed_reaches_fp64_accuracy(laplace128_oracle):
    A, X0, ref = laplace128_oracle
    out = native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-10, mode=native.TRL_MODE_MIXED, fp32_tol=1e-5)
    assert out["converged"]
    exact = P.laplace2d_eigenvalues(128)[:10]
    assert np.max(np.abs(out["evals"] - exact) / exact) < 1e-11
    assert out["max_rel_residual"] < 1e-9
    assert out["restarts_fp32"] > 0


@pytest.mark.parametrize("refine,refine_fp32", [(native.TRL_REFINE_CHEBYSHEV, 1), (native.TRL_REFINE_CHEBYSHEV, 0), (native.TRL_REFINE_LANCZOS, 1)])
def test_mixed_refinements_reach_fp64_accuracy(laplace128_oracle, refine, refine_fp32):
    """Both FP64 refinements of the mixed mode from the FP32 phase's kept Ritz vectors: the
    Chebyshev-filtered subspace iteration with Rayleigh-Ritz (with and without its FP32
    filter rounds), and a BlockLanczos restart."""
    A, X0, ref = laplace128_oracle
    out = native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-10, mode=native.TRL_MODE_MIXED, fp32_tol=1e-4, refine=refine,
                                refine_fp32=refine_fp32)
    assert out["converged"]
    exact = P.laplace2d_eigenvalues(128)[:10]
    assert np.max(np.abs(out["evals"] - exact) / exact) < 1e-11
    assert np.max(np.abs(out["evals"] - ref["evals"][:10]) / ref["evals"][:10]) < 1e-11
    assert out["max_theta_residual"] < 1e-10
    assert max_principal_sine(out["evecs"], ref["ritz"], out["evals"]) < 1e-5
    if refine == native.TRL_REFINE_CHEBYSHEV:
        assert out["refine_rounds"] >= 1 and out["refine_degree"] > 0 and out["restarts"] == 0
        if not refine_fp32:
            assert out["refine_degree_fp32"] == 0
    else:
        assert out["refine_rounds"] == 0 and out["restarts"] > 0


@pytest.mark.parametrize("mode", [native.TRL_MODE_FP64, native.TRL_MODE_MIXED])
def test_partial_and_full_projected_eigensolvers_agree(laplace128_oracle, mode):
    """The restart's projected eigenproblem solved for the kept eigenvectors only (cluster
    tridiagonalisation + inverse iteration, the default) and for all of them (cuSOLVER
    syevd): same eigenpairs, same number of restarts."""
    A, X0, ref = laplace128_oracle
    kw = dict(bs=4, nev=10, ncv=160, tol=1e-10, mode=mode, fp32_tol=1e-4)
    part = native.solve_csr_host(A, X0, small_eigen_full=0, **kw)
    full = native.solve_csr_host(A, X0, small_eigen_full=1, **kw)
    assert part["converged"] and full["converged"]
    assert np.max(np.abs(part["evals"] - full["evals"]) / np.abs(full["evals"])) < 1e-12
    assert abs(part["restarts"] - full["restarts"]) <= 1 and abs(part["restarts_fp32"] - full["restarts_fp32"]) <= 1
    assert part["max_theta_residual"] < 1e-10
    assert max_principal_sine(part["evecs"], ref["ritz"], part["evals"]) < 1e-5


@pytest.mark.parametrize("fp32_ncv", [0, 96])
def test_mixed_loose_fp32_phase_filters_in_fp32(laplace128_oracle, fp32_ncv):
    """A loose FP32 phase (fp32_tol 1e-2, optionally on a smaller FP32 basis) leaves most of
    the work to the filter: its FP32 rounds run first and the FP64 rounds finish at 1e-10."""
    A, X0, ref = laplace128_oracle
    out = native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-10, mode=native.TRL_MODE_MIXED, fp32_tol=1e-2, fp32_ncv=fp32_ncv)
    assert out["converged"]
    assert 0 < out["refine_degree_fp32"] < out["refine_degree"]
    exact = P.laplace2d_eigenvalues(128)[:10]
    assert np.max(np.abs(out["evals"] - exact) / exact) < 1e-11
    assert out["max_theta_residual"] < 1e-10
    assert max_principal_sine(out["evecs"], ref["ritz"], out["evals"]) < 1e-5


def test_fp32_ncv_must_be_a_multiple_of_the_block_size(laplace128_oracle):
    A, X0, _ = laplace128_oracle
    with pytest.raises(native.TrlError):
        native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-10, mode=native.TRL_MODE_MIXED, fp32_ncv=98)


@pytest.mark.parametrize("refine", ["chebyshev", "lanczos"])
def test_mixed_with_kept_values_on_both_sides_of_zero(oracle, refine):
    """Largest-magnitude eigenvalues of an indefinite matrix (the bandwidth-stress pattern):
    the kept Ritz values straddle zero. The Chebyshev refinement then filters on [-b, b]
    centred at zero (b the smallest kept |theta|), amplifying both ends; the Lanczos
    refinement restarts BlockLanczos. Both agree with the oracle to 1e-10."""
    A = P.zipf_symmetric(20_000, seed=7)
    X0 = P.initial_block(A.n, 8, seed=11)
    ref = oracle.solve_csr(A, 8, 16, 128, X0, tol=1e-10)
    kind = native.TRL_REFINE_CHEBYSHEV if refine == "chebyshev" else native.TRL_REFINE_LANCZOS
    out = native.solve_csr_host(A, X0, bs=8, nev=16, ncv=128, tol=1e-10, mode=native.TRL_MODE_MIXED, fp32_tol=1e-4, refine=kind)
    assert out["converged"]
    assert np.min(out["evals"]) < 0 < np.max(out["evals"])  # both ends are wanted
    if refine == "chebyshev":
        assert out["refine_rounds"] > 0 and out["restarts"] == 0
    else:
        assert out["refine_rounds"] == 0 and out["restarts"] > 0
    assert np.max(np.abs(out["evals"] - ref["evals"][:16]) / np.abs(ref["evals"][:16])) < 1e-10
    assert out["max_theta_residual"] < 1e-10


def test_fp32_mode_accuracy_is_stated(laplace128_oracle):
    A, X0, ref = laplace128_oracle
    out = native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-5, mode=native.TRL_MODE_FP32)
    assert out["converged"]
    exact = P.laplace2d_eigenvalues(128)[:10]
    assert np.max(np.abs(out["evals"] - exact) / exact) < 1e-5


def test_device_entry_point_matches_host_entry_point(laplace128_oracle):
    A, X0, ref = laplace128_oracle
    h = native.Handle(0)
    A64 = native.DeviceCSRTensors.from_host(A)
    X0d = torch.from_numpy(X0).cuda()
    ev = torch.zeros((A.n, 10), dtype=torch.float64, device="cuda")
    out = native.solve_csr_device(h, A64, None, X0d, evecs=ev, bs=4, nev=10, ncv=160, tol=1e-8)
    host = native.solve_csr_host(A, X0, bs=4, nev=10, ncv=160, tol=1e-8)
    assert out["converged"] and host["converged"]
    assert np.allclose(out["evals"], host["evals"], rtol=1e-13)
    assert out["kernel_launches"] > 0
    h.close()


def test_smallest_via_shift(oracle):
    """Smallest eigenvalues through sigma*I - A (the |theta|-descending order keeps largest)."""
    A = P.anisotropic3d(12, coef=(1.0, 2.0, 3.0))
    sigma = A.gershgorin_bound()
    X0 = P.initial_block(A.n, 4, seed=1)
    out = native.solve_csr_host(A, X0, bs=4, nev=8, ncv=64, tol=1e-10, alpha=-1.0, beta=sigma)
    lam = sigma - out["evals"]
    exact = np.sort(np.linalg.eigvalsh(A.to_dense()))[:8]
    assert np.max(np.abs(lam - exact) / np.abs(exact)) < 1e-9
    ref = oracle.solve_csr(A, 4, 8, 64, X0, tol=1e-10, alpha=-1.0, beta=sigma)
    assert np.max(np.abs(out["evals"] - ref["evals"][:8]) / ref["evals"][:8]) < 1e-10


@pytest.mark.parametrize("reorth", [native.TRL_REORTH_CGS1, native.TRL_REORTH_CGS_IFNEEDED, native.TRL_REORTH_CGS2, native.TRL_REORTH_MGS, native.TRL_REORTH_PARTIAL])
@pytest.mark.parametrize("batching", [0, 1])
def test_shifted_small_problem_to_tight_tolerance(reorth, batching):
    """sigma*I - A with a wide spectrum, 12 restart cycles to 1e-12: every block step carries a
    large T_ii component, so any reorganisation of the three-term step that weakens the
    reorthogonalisation shows up as lost orthogonality after the first restart."""
    A = P.anisotropic3d(9, coef=(1.0, 3.0, 7.0))
    sigma = A.gershgorin_bound()
    X0 = P.initial_block(A.n, 4, seed=3)
    out = native.solve_csr_host(A, X0, bs=4, nev=4, ncv=64, tol=1e-12, alpha=-1.0, beta=sigma, reorth=reorth, batching=batching)
    assert out["converged"]
    exact = np.sort(np.linalg.eigvalsh(A.to_dense()))[:4]
    assert np.max(np.abs(sigma - out["evals"] - exact) / np.abs(exact)) < 1e-9
    assert np.max(out["resid"]) < 1e-11


def test_elasticity_smallest_fp64_and_mixed(oracle):
    """The mixed-precision workload's matrix family at small size (8^3 nodes x 3 dofs,
    27-point coupling, diagonal dominance 1.05): 16 smallest eigenpairs through sigma*I - A,
    FP64 and mixed, against the reference's OpenMP backend and a dense eigensolve."""
    A = P.elasticity27(8, seed=42)
    sigma = A.gershgorin_bound()
    X0 = P.initial_block(A.n, 8, seed=42)
    ref = oracle.solve_csr(A, 8, 16, 128, X0, tol=1e-10, alpha=-1.0, beta=sigma)
    assert ref["converged"]
    exact = np.sort(np.linalg.eigvalsh(A.to_dense()))[:16]
    for mode in (native.TRL_MODE_FP64, native.TRL_MODE_MIXED):
        out = native.solve_csr_host(A, X0, bs=8, nev=16, ncv=128, tol=1e-10, alpha=-1.0, beta=sigma, mode=mode, fp32_tol=1e-5)
        assert out["converged"], mode
        assert np.max(np.abs(out["evals"] - ref["evals"][:16]) / np.abs(ref["evals"][:16])) < 1e-10, mode
        assert np.max(np.abs((sigma - out["evals"]) - exact)) < 1e-9 * sigma, mode
        assert out["max_rel_residual"] < 1e-9, mode


@pytest.mark.parametrize("bs", [4, 8, 16])
def test_zipf_largest_against_reference(oracle, bs):
    """The bandwidth-stress workload's matrix family at small size (n = 20,000, Zipf(1.5)
    degrees capped at 512, mirrored N(0,1) values): 16 largest-magnitude eigenpairs for
    block sizes 4, 8, 16 against the reference's OpenMP backend."""
    A = P.zipf_symmetric(20_000, seed=7)
    X0 = P.initial_block(A.n, bs, seed=11)
    ncv = 16 * bs
    ref = oracle.solve_csr(A, bs, 16, ncv, X0, tol=1e-10)
    assert ref["converged"]
    out = native.solve_csr_host(A, X0, bs=bs, nev=16, ncv=ncv, tol=1e-10)
    assert out["converged"]
    assert np.max(np.abs(out["evals"] - ref["evals"][:16]) / np.abs(ref["evals"][:16])) < 1e-10
    assert out["max_rel_residual"] < 1e-9


def test_invalid_parameters_raise():
    A = P.laplace1d(64)
    X0 = P.initial_block(64, 4)
    with pytest.raises(native.TrlError) as e:
        native.solve_csr_host(A, X0, bs=4, nev=16, ncv=16)  # nev >= ncv (lanczos.hh:50)
    assert e.value.status == native.TRL_EINVAL
    with pytest.raises(native.TrlError):
        native.solve_csr_host(A, X0, bs=4, nev=4, ncv=62)  # ncv not a multiple of bs


@pytest.mark.slow
def test_aniso96_fp64_and_mixed_to_analytic():
    """The 96^3 anisotropic Laplacian (1,10,100): 32 largest to 1e-10, both modes, against the
    analytic spectrum and against the eigenvalues and restart count of the reference's own
    OpenMP BlockLanczos on the same matrix and start block (tests/golden/aniso96_reference.json,
    written by tests/golden/make_aniso96_reference.py)."""
    A = P.anisotropic3d(96)
    exact = P.anisotropic3d_eigenvalues(96, k=32)
    with open(GOLDEN / "aniso96_reference.json") as f:
        ref = json.load(f)
    ref_evals = np.asarray(ref["evals"])
    X0 = P.initial_block(A.n, 8, seed=42)
    for mode in (native.TRL_MODE_FP64, native.TRL_MODE_MIXED):
        out = native.solve_csr_host(A, X0, vectors=False, bs=8, nev=32, ncv=384, tol=1e-10, mode=mode, fp32_tol=1e-5)
        assert out["converged"], mode
        assert np.max(np.abs(out["evals"] - exact) / exact) < 1e-10, mode
        assert np.max(np.abs(out["evals"] - ref_evals) / np.abs(ref_evals)) < 1e-10, mode
        assert out["max_rel_residual"] < 1e-9, mode
        if mode == native.TRL_MODE_FP64:
            assert abs(out["restarts"] - ref["restarts"]) <= max(3, ref["restarts"] // 5)


def test_solve_from_matrix_market_file(tmp_path):
    """A symmetric Matrix Market file (lower triangle, as the reference's examples read
    them) loaded with trl_csr_read_mtx and solved on the GPU: the 2-D Laplacian's largest
    eigenvalues to 1e-10."""
    A = P.laplace2d(40)
    rows = A.row_indices()
    low = [(int(r) + 1, int(c) + 1, v) for r, c, v in zip(rows, A.colind, A.values) if c <= r]
    path = tmp_path / "laplace40.mtx"
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{A.n} {A.n} {len(low)}\n")
        for r, c, v in low:
            f.write(f"{r} {c} {v:.17g}\n")
    B = native.read_mtx(str(path))
    X0 = P.initial_block(B.n, 4, seed=42)
    out = native.solve_csr_host(B, X0, bs=4, nev=8, ncv=96, tol=1e-10)
    assert out["converged"]
    exact = P.laplace2d_eigenvalues(40)[:8]
    assert np.max(np.abs(out["evals"] - exact) / exact) < 1e-10


def test_zipf_fp64_matches_the_reference_on_an_indefinite_spectrum():
    """The bandwidth-stress pattern at 524,288 rows, block size 8, the 100 largest-magnitude
    eigenpairs (both ends of an indefinite spectrum): the reference's own driver and OpenMP
    backend (tests/golden/zipf524k_b8_reference.json, made by make_zipf_reference.py) and the
    CUDA backend agree to 1e-10. Converged Ritz pairs put couplings of ~1e-160 into the
    projected matrix; before negligible entries were flushed, their underflowing squares made
    the Householder reduction non-orthogonal and the solve stopped with a spurious eigenvalue."""
    import json
    import os

    with open(os.path.join(os.path.dirname(__file__), "golden", "zipf524k_b8_reference.json")) as f:
        ref = json.load(f)
    A = P.zipf_symmetric(524288, seed=42)
    X0 = P.initial_block(A.n, 8, seed=42)
    out = native.solve_csr_host(A, X0, bs=8, nev=100, ncv=256, tol=1e-10, max_restarts=3000)
    assert out["converged"]
    r = np.asarray(ref["evals"])
    assert np.max(np.abs(out["evals"] - r) / np.abs(r)) < 1e-10
    assert out["max_theta_residual"] < 1e-9
    assert abs(out["restarts"] - ref["restarts"]) <= max(3, ref["restarts"] // 5)


@pytest.mark.parametrize("case", ["laplace2d", "zipf"])
def test_mixed_auto_refinement_chooses_and_converges(oracle, case):
    """TRL_REFINE_AUTO (the default) predicts the Chebyshev refinement's time after its first
    Rayleigh-Ritz step and hands over to the Lanczos refinement when that is estimated
    cheaper; either way the eigenpairs reach the FP64 tolerance and agree with the oracle."""
    if case == "laplace2d":
        A, bs, nev, ncv = P.laplace2d(128), 4, 10, 160
    else:
        A, bs, nev, ncv = P.zipf_symmetric(20_000, seed=7), 8, 16, 128
    X0 = P.initial_block(A.n, bs, seed=11)
    ref = oracle.solve_csr(A, bs, nev, ncv, X0, tol=1e-10)
    out = native.solve_csr_host(A, X0, bs=bs, nev=nev, ncv=ncv, tol=1e-10, mode=native.TRL_MODE_MIXED, fp32_tol=1e-4)
    assert out["converged"]
    assert out["refine_used"] in (native.TRL_REFINE_CHEBYSHEV, native.TRL_REFINE_LANCZOS)
    assert out["refine_predicted_s"] > 0 and out["refine_lanczos_estimate_s"] > 0
    if out["refine_used"] == native.TRL_REFINE_LANCZOS:
        # handed over after the first Rayleigh-Ritz step, on the prediction
        assert out["restarts"] > 0 and out["refine_rounds"] == 1
        assert out["refine_predicted_s"] > out["refine_lanczos_estimate_s"]
    else:
        assert out["refine_rounds"] >= 1
    assert np.max(np.abs(out["evals"] - ref["evals"][:nev]) / np.abs(ref["evals"][:nev])) < 1e-10
    assert out["max_theta_residual"] < 1e-10


@pytest.mark.parametrize("bs,reorth", [(4, native.TRL_REORTH_CGS_IFNEEDED), (4, native.TRL_REORTH_MGS), (2, native.TRL_REORTH_PARTIAL), (8, native.TRL_REORTH_CGS2)])
def test_m_inner_product_matches_the_oracle(oracle, bs, reorth):
    """K x = lambda M x with a non-diagonal SPD M through op = M^{-1} K (self-adjoint in the M
    inner product): dot = V^T (M W) and CholQR in that inner product on the device, against
    the reference driver with the same inner product (the oracle) and a dense generalised
    eigensolver; Ritz vectors M-orthonormal."""
    import scipy.linalg as sl

    K, M = P.diffusion2d_consistent_mass(12, seed=3)
    Kd, Md = K.to_dense(), M.to_dense()
    Op = P.dense_csr(np.linalg.solve(Md, Kd))
    nev, ncv = 8, 12 * bs
    X0 = P.initial_block(K.n, bs, seed=5)
    ref = oracle.solve_csr_minner(Op, M, bs, nev, ncv, X0, tol=1e-10)
    h = native.Handle(0)
    ev = torch.zeros((K.n, nev), dtype=torch.float64, device="cuda")
    out = native.solve_csr_minner_device(h, native.DeviceCSRTensors.from_host(Op), native.DeviceCSRTensors.from_host(M), torch.from_numpy(X0).cuda(), evecs=ev,
                                         bs=bs, nev=nev, ncv=ncv, tol=1e-10, reorth=reorth)
    assert out["converged"] and ref["converged"]
    lam = sl.eigh(Kd, Md, eigvals_only=True)[::-1][:nev]
    assert np.max(np.abs(out["evals"] - ref["evals"][:nev]) / lam) < 1e-10
    assert np.max(np.abs(out["evals"] - lam) / lam) < 1e-10
    X = ev.cpu().numpy()
    assert np.abs(X.T @ Md @ X - np.eye(nev)).max() < 1e-9
    assert out["max_theta_residual"] < 1e-9
    h.close()
