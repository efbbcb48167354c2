"""The prepared operator (trl_cuda_op_*: sliced-ELL copy with rows sorted by length inside
windows of 4096 rows) against the oracle's CSR apply (examples/sycl/csrevp.hh:159-187
semantics) and against the CSR kernel's per-row walk (trl_cuda_spmm_blocks), bit for bit:
every row still sums its entries in CSR order.

Tolerances as in test_kernels_gpu.py: FP64 1e-12 and FP32 2e-6 relative to the summed
magnitudes sum_j |a_ij| max|x_j|.
"""
import numpy as np
import pytest
import torch

from trl_b200 import native
from trl_b200 import problems as P

from test_kernels_gpu import BS, DT, _long_row_csr, _random_csr, as_dt, close, dev, host

pytestmark = pytest.mark.gpu


def _patterns():
    rng = np.random.default_rng(77)
    return [
        ("laplace2d", P.laplace2d(64)),
        ("aniso3d", P.anisotropic3d(9, coef=(1.0, 10.0, 100.0))),
        ("elasticity", P.elasticity27(7, seed=3)),
        # three windows, heavy-tailed rows (slices taken window-major)
        ("zipf", P.zipf_symmetric(9001, cap=512, seed=4)),
        ("long_rows", _long_row_csr(rng)),
        ("random_empty_rows", _random_csr(5003, rng)),
        ("tiny", P.diagonal(3)),
    ]


PATTERNS = _patterns()


def _mag(A, vals, X):
    rows = A.row_indices()
    mag = np.zeros(A.n)
    np.add.at(mag, rows, np.abs(vals) * np.abs(X).reshape(-1, A.n, X.shape[-1]).max(axis=(0, 2))[A.colind])
    return mag.max() if A.n else 1.0


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("case", PATTERNS, ids=lambda c: c[0])
def test_prepared_spmm_matches_oracle(cuda_handle, oracle, bs, dtype, case):
    name, A = case
    rng = np.random.default_rng(bs)
    vals = A.values.astype(np.float32).astype(np.float64) if dtype == torch.float32 else A.values
    Ah = P.CSRMatrix(A.n, A.rowptr, A.colind, vals)
    Ad = native.DeviceCSRTensors.from_host(Ah, dtype)
    op = cuda_handle.prepare(Ad, bs)
    info = op.info()
    assert info["stored"] >= A.nnz
    assert info["longest_row"] == int(np.diff(A.rowptr).max())
    tol = 1e-12 if dtype == torch.float64 else 2e-6
    X = as_dt(rng.standard_normal((A.n, bs)), dtype)
    for alpha, beta in ((1.0, 0.0), (-1.0, 3.5)):
        Yd = torch.full((A.n, bs), float("nan"), dtype=dtype, device="cuda")
        op.spmm(dev(X, dtype), Yd, alpha, beta)
        close(host(Yd), oracle.spmm(Ah, X, alpha, beta), _mag(A, vals, X) + abs(beta) * np.abs(X).max(), tol)
    op.close()


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("nb", [1, 2, 5, 8])
@pytest.mark.parametrize("case", [PATTERNS[1], PATTERNS[3], PATTERNS[4]], ids=lambda c: c[0])
def test_prepared_spmm_blocks_three_term(cuda_handle, oracle, bs, dtype, nb, case):
    """Y_j = alpha A X_j + beta X_j + gamma W_j on nb blocks (groups of four blocks per pass
    and a remainder group) with W separate, W = Y in place, and no W; the no-W result equals
    the CSR kernel's multi-block walk bit for bit."""
    name, A = case
    rng = np.random.default_rng(31 * bs + nb)
    tol = 1e-12 if dtype == torch.float64 else 2e-6
    vals = A.values.astype(np.float32).astype(np.float64) if dtype == torch.float32 else A.values
    Ah = P.CSRMatrix(A.n, A.rowptr, A.colind, vals)
    Ad = native.DeviceCSRTensors.from_host(Ah, dtype)
    op = cuda_handle.prepare(Ad, bs)
    X = as_dt(rng.standard_normal((nb, A.n, bs)), dtype)
    W = as_dt(rng.standard_normal((nb, A.n, bs)), dtype)
    alpha, beta, gamma = 0.75, -1.25, 0.5
    ref = np.stack([oracle.spmm(Ah, X[j], alpha, beta) for j in range(nb)])
    scale = abs(alpha) * _mag(A, vals, X) + abs(beta) * np.abs(X).max() + abs(gamma) * np.abs(W).max()
    Xd = dev(X, dtype)
    Yd = torch.full((nb, A.n, bs), float("nan"), dtype=dtype, device="cuda")
    op.spmm(Xd, Yd, alpha, beta, gamma, dev(W, dtype))
    close(host(Yd), ref + gamma * W, scale, tol)
    Yd = dev(W, dtype)
    op.spmm(Xd, Yd, alpha, beta, gamma, Yd)
    close(host(Yd), ref + gamma * W, scale, tol)
    Yd = torch.full((nb, A.n, bs), float("nan"), dtype=dtype, device="cuda")
    op.spmm(Xd, Yd, alpha, beta)
    close(host(Yd), ref, scale, tol)
    if nb > 1:
        Yc = torch.full((nb, A.n, bs), float("nan"), dtype=dtype, device="cuda")
        cuda_handle.spmm_blocks(Ad, Xd, Yc, alpha, beta, 0.0, None)
        assert torch.equal(Yd, Yc)
    op.close()


def test_prepared_spmm_rejects_bad_arguments(cuda_handle):
    A = native.DeviceCSRTensors.from_host(P.laplace1d(16))
    with pytest.raises(native.TrlError) as e:
        cuda_handle.prepare(A, 3)
    assert e.value.status == native.TRL_ENOTSUP
    op = cuda_handle.prepare(A, 4)
    X = torch.zeros((16, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(native.TrlError) as e:
        op.spmm(X, X)
    assert e.value.status == native.TRL_EINVAL
    Xs = torch.zeros(16 * 4 + 1, dtype=torch.float64, device="cuda")[1:].view(16, 4)  # 8-byte aligned only
    with pytest.raises(native.TrlError) as e:
        op.spmm(Xs, torch.zeros_like(X))
    assert e.value.status == native.TRL_EINVAL
    op.close()
