"""Parity of every C-ABI kernel (include/trl_cuda.h) with the reference's own OpenMP kernels
(the oracle: impl/openmp/blockview.hh, the restated evp_base.hh) on the same seeded inputs.

Tolerances: FP64 results agree with the reference to 1e-12 relative to the magnitude of the
summed terms (sum |x_i y_i|); only the summation order differs. FP32 storage is widened to
FP64 before every product, so contractions of FP32 data agree with an FP64 evaluation of
the same FP32 inputs to the same 1e-12. FP32 SpMM accumulates in FP32 (as specified for the
mixed mode) and is held to 1e-5 relative.
"""
import numpy as np
import pytest
import torch

from trl_b200 import native
from trl_b200 import problems as P

pytestmark = pytest.mark.gpu

BS = [1, 2, 4, 8, 16]
DT = [torch.float64, torch.float32]


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def host(t):
    torch.cuda.synchronize()
    return t.double().cpu().numpy()


def as_dt(a, dtype):
    return a.astype(np.float32).astype(np.float64) if dtype == torch.float32 else a


def close(a, b, scale, tol=1e-12):
    err = np.max(np.abs(a - b)) if a.size else 0.0
    assert err <= tol * max(scale, 1e-300), (err, scale)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("n", [0, 1, 37, 1029, 200_003])
def test_dot_matches_reference(cuda_handle, oracle, bs, dtype, n):
    rng = np.random.default_rng(n * 31 + bs)
    X = as_dt(rng.standard_normal((n, bs)), dtype)
    Y = as_dt(rng.standard_normal((n, bs)), dtype)
    R = np.zeros((bs, bs))
    oracle.block_view_op(bs, oracle.OP_DOT, X.copy(), Y.copy(), R)  # blockview.hh:152-182
    Rd = torch.zeros((1, bs, bs), dtype=torch.float64, device="cuda")
    cuda_handle.block_dot(dev(X, dtype)[None], dev(Y, dtype), Rd)
    close(host(Rd)[0], R, (np.abs(X).T @ np.abs(Y)).max() if n else 1.0)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("nblk", [1, 3, 9, 17, 49])
def test_multiblock_dot_and_update(cuda_handle, oracle, bs, dtype, nblk):
    """One classical Gram-Schmidt pass against nblk blocks, C_j = V_j^T w then
    w -= sum_j V_j C_j, against the reference's BlockView::dot and subtract_product applied
    block by block (blockview.hh:152-182, 189-201), the loop of the reference's
    orthogonalisation strategies."""
    rng = np.random.default_rng(nblk * 7 + bs)
    n = 4099
    V = as_dt(rng.standard_normal((nblk, n, bs)), dtype)
    w = as_dt(rng.standard_normal((n, bs)), dtype)
    Cd = torch.zeros((nblk, bs, bs), dtype=torch.float64, device="cuda")
    Vd, wd = dev(V, dtype), dev(w, dtype)
    cuda_handle.block_dot(Vd, wd, Cd)
    Cref = np.zeros((nblk, bs, bs))
    for j in range(nblk):
        oracle.block_view_op(bs, oracle.OP_DOT, V[j].copy(), w.copy(), Cref[j])
    close(host(Cd), Cref, np.einsum("jnb,nc->jbc", np.abs(V), np.abs(w)).max())
    cuda_handle.block_update(wd, Vd, Cd)
    C = host(Cd)
    ref = w.copy()
    for j in range(nblk):
        oracle.block_view_op(bs, oracle.OP_SUB_PROD, ref, V[j].copy(), C[j].copy())
    got = host(wd)
    tol = 1e-12 if dtype == torch.float64 else 2e-7
    close(got, ref, np.abs(ref).max() + np.abs(w).max(), tol)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("n", [1, 13, 5003])
def test_block_view_ops_match_reference(cuda_handle, oracle, bs, dtype, n):
    rng = np.random.default_rng(1000 + n + bs)
    X = as_dt(rng.standard_normal((n, bs)), dtype)
    Y = as_dt(rng.standard_normal((n, bs)), dtype)
    W = rng.standard_normal((bs, bs))
    tol = 1e-12 if dtype == torch.float64 else 2e-7  # FP32 results are rounded to FP32 storage
    scale = np.abs(X).max() * np.abs(W).sum(axis=0).max() + np.abs(Y).max()
    Wd = dev(W)
    # mult: Y = X W  (blockview.hh:104-119)
    Z = np.zeros_like(X)
    oracle.block_view_op(bs, oracle.OP_MULT, X.copy(), Z, W.copy())
    Zd = torch.zeros((n, bs), dtype=dtype, device="cuda")
    cuda_handle.bv_mult(native.TRL_MULT, dev(X, dtype), Wd, Zd)
    close(host(Zd), Z, scale, tol)
    # mult_transpose: Y = X W^T  (blockview.hh:126-141)
    Z = np.zeros_like(X)
    oracle.block_view_op(bs, oracle.OP_MULT_T, X.copy(), Z, W.copy())
    cuda_handle.bv_mult(native.TRL_MULT_TRANSPOSE, dev(X, dtype), Wd, Zd)
    close(host(Zd), Z, scale, tol)
    # mult_add: Y += X W  (blockview.hh:81-97)
    Z = Y.copy()
    oracle.block_view_op(bs, oracle.OP_MULT_ADD, X.copy(), Z, W.copy())
    Zd = dev(Y, dtype)
    cuda_handle.bv_mult(native.TRL_MULT_ADD, dev(X, dtype), Wd, Zd)
    close(host(Zd), Z, scale, tol)
    # subtract_product: X -= Y W  (blockview.hh:189-201)
    Z = X.copy()
    oracle.block_view_op(bs, oracle.OP_SUB_PROD, Z, Y.copy(), W.copy())
    Zd = dev(X, dtype)
    cuda_handle.bv_mult(native.TRL_SUBTRACT, dev(Y, dtype), Wd, Zd)
    close(host(Zd), Z, scale, tol)
    # Y -= X W^T: mult_transpose followed by -= (lanczos.hh:243-245) in one pass
    Zd = dev(X, dtype)
    cuda_handle.bv_mult(native.TRL_SUBTRACT_TRANSPOSE, dev(Y, dtype), Wd, Zd)
    close(host(Zd), X - Y @ W.T, scale, tol)
    # operator-=  (blockview.hh:69-74)
    Z = X.copy()
    oracle.block_view_op(bs, oracle.OP_SUB, Z, Y.copy(), W.copy())
    Zd = dev(X, dtype)
    cuda_handle.bv_sub(Zd, dev(Y, dtype))
    close(host(Zd), Z, scale, tol)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("m,k", [(1, 1), (5, 2), (48, 5), (40, 11), (9, 9)])
def test_rotation_matches_mult_add_loop(cuda_handle, oracle, bs, dtype, m, k):
    """W_j = sum_i V_i Y_ij in one pass == the k*m mult_add calls of lanczos.hh:105-114."""
    rng = np.random.default_rng(m * 100 + k + bs)
    n = 2311
    V = as_dt(rng.standard_normal((m, n, bs)), dtype)
    Y = rng.standard_normal((m, m + 1, bs, bs))  # ldy = m + 1 block columns
    ref = np.zeros((k, n, bs))
    for j in range(k):
        for i in range(m):
            oracle.block_view_op(bs, oracle.OP_MULT_ADD, V[i].copy(), ref[j], Y[i, j].copy())
    Wd = torch.zeros((k, n, bs), dtype=dtype, device="cuda")
    cuda_handle.block_rotate(dev(V, dtype), dev(Y), k, Wd)
    tol = 1e-12 if dtype == torch.float64 else 2e-7
    close(host(Wd), ref, np.einsum("inb,ijbc->jnc", np.abs(V), np.abs(Y[:, :k])).max(), tol)


@pytest.mark.parametrize("bs", BS)
def test_cholqr_single_pass_matches_reference(cuda_handle, oracle, bs):
    rng = np.random.default_rng(bs)
    n = 3001
    X = rng.standard_normal((n, bs))
    V = X.copy()
    R = oracle.orthonormalize(V)  # evp_base.hh:39-71
    Xd = dev(X)
    Rd = torch.zeros((bs, bs), dtype=torch.float64, device="cuda")
    cuda_handle.cholqr(Xd, 1, Rd)
    cuda_handle.sync()
    close(host(Rd), R, np.abs(R).max(), 1e-11)
    close(host(Xd), V, 1.0, 1e-10)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
def test_cholqr2_orthonormal_and_factor(cuda_handle, bs, dtype):
    rng = np.random.default_rng(bs + 99)
    n = 50_000
    # ill-conditioned block (cond ~ 1e5): CholQR2 restores orthogonality
    X = rng.standard_normal((n, bs)) @ np.diag(np.logspace(0, -5 if bs > 1 else 0, bs))
    X = as_dt(X, dtype)
    Xd = dev(X, dtype)
    Rd = torch.zeros((bs, bs), dtype=torch.float64, device="cuda")
    cuda_handle.cholqr(Xd, 2, Rd)
    cuda_handle.sync()
    Q = host(Xd)
    R = host(Rd)
    eps = 1e-13 if dtype == torch.float64 else 1e-6
    assert np.abs(Q.T @ Q - np.eye(bs)).max() < eps * 10
    assert np.allclose(np.tril(R, -1), 0)
    rel = np.abs(Q @ R - X).max() / np.abs(X).max()
    assert rel < (1e-12 if dtype == torch.float64 else 1e-6)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("contiguous", [True, False])
def test_project_out_modes(cuda_handle, bs, dtype, contiguous):
    """trl_cuda_project_out against numpy classical Gram-Schmidt (one / two passes), its
    returned Gram matrix, and the DGKS decision of the if-needed mode."""
    rng = np.random.default_rng(7 * bs + contiguous)
    n, nblk = 3001, 6
    Q, _ = np.linalg.qr(rng.standard_normal((n, nblk * bs)))
    V = as_dt(Q.reshape(n, nblk, bs).transpose(1, 0, 2).copy(), dtype)
    eps = 1e-12 if dtype == torch.float64 else 2e-6

    def run(w0, mode):
        store = torch.zeros((nblk + 1, n, bs), dtype=dtype, device="cuda")
        store[:nblk] = dev(V, dtype)
        if contiguous:
            Vd, Wd = store[:nblk], store[nblk]
            Wd.copy_(dev(w0, dtype))
        else:
            Vd, Wd = dev(V, dtype), dev(w0, dtype)
        G = torch.zeros((bs, bs), dtype=torch.float64, device="cuda")
        cuda_handle.project_out(Vd, Wd, mode, G)
        return host(Wd), host(G)

    Vf = V.transpose(1, 0, 2).reshape(n, nblk * bs)
    # a vector with a large component in span(V): one pass loses orthogonality, two restore it
    w = as_dt(Vf @ rng.standard_normal((nblk * bs, bs)) * 100 + rng.standard_normal((n, bs)), dtype)
    w1 = w - Vf @ (Vf.T @ w)
    w2 = w1 - Vf @ (Vf.T @ w1)
    got1, G1 = run(w, native.TRL_CGS_ONE)
    got2, G2 = run(w, native.TRL_CGS_TWO)
    got3, G3 = run(w, native.TRL_CGS_IFNEEDED)
    scale = np.abs(w).max()
    close(got1, w1, scale, eps)
    close(got2, w2, scale, eps)
    close(got3, got2, scale, eps)  # large cancellation: the criterion asks for the second pass
    close(G1, got1.T @ got1, np.abs(G1).max(), 1e-10)
    close(G2, got2.T @ got2, np.abs(G2).max(), 1e-10)
    assert np.abs(Vf.T @ got2).max() < 1e4 * eps * np.abs(got2).max()
    # an almost orthogonal vector: the if-needed mode keeps one pass
    w = as_dt(rng.standard_normal((n, bs)) + Vf @ rng.standard_normal((nblk * bs, bs)) * 1e-3, dtype)
    got1, _ = run(w, native.TRL_CGS_ONE)
    got3, G3 = run(w, native.TRL_CGS_IFNEEDED)
    assert np.array_equal(got1, got3)
    close(G3, got3.T @ got3, np.abs(G3).max(), 1e-10)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
def test_cholqr_with_given_gram_matches_cholqr(cuda_handle, bs, dtype):
    rng = np.random.default_rng(bs + 5)
    X = as_dt(rng.standard_normal((20_011, bs)), dtype)
    X1, X2 = dev(X, dtype), dev(X, dtype)
    R1 = torch.zeros((bs, bs), dtype=torch.float64, device="cuda")
    R2 = torch.zeros_like(R1)
    G0 = torch.zeros_like(R1)
    cuda_handle.block_dot(X2[None], X2, G0[None])
    cuda_handle.cholqr(X1, 2, R1)
    cuda_handle.cholqr_gram(X2, 2, R2, G0)
    cuda_handle.sync()
    tol = 1e-12 if dtype == torch.float64 else 1e-6
    close(host(X2), host(X1), 1.0, tol)
    close(host(R2), host(R1), np.abs(host(R1)).max(), tol)


def test_cholqr_breakdown_is_reported(cuda_handle):
    Xd = torch.zeros((100, 4), dtype=torch.float64, device="cuda")
    Rd = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    cuda_handle.cholqr(Xd, 1, Rd)
    with pytest.raises(native.TrlError) as e:
        cuda_handle.sync()
    assert e.value.status == native.TRL_ECHOLESKY
    cuda_handle.sync()  # the status word is cleared by the report; the context stays usable


@pytest.mark.parametrize("bs", [4, 8, 16])
@pytest.mark.parametrize("dtype", DT)
def test_project_out_sketch_decides_on_the_device(cuda_handle, bs, dtype):
    """trl_cuda_project_out_sketch: with a threshold far below the block's orthogonality loss
    it projects exactly as the if-needed mode; far above, it leaves the block untouched and
    returns its Gram matrix; the decision follows ||S^T W||_F / ||W||_F."""
    rng = np.random.default_rng(11 * bs)
    n, nblk = 2003, 5
    Q, _ = np.linalg.qr(rng.standard_normal((n, nblk * bs)))
    V = as_dt(Q.reshape(n, nblk, bs).transpose(1, 0, 2).copy(), dtype)
    Vf = V.transpose(1, 0, 2).reshape(n, nblk * bs)
    Gc = rng.standard_normal((nblk, bs, bs)) / np.sqrt(bs)
    S = as_dt(sum(V[j] @ Gc[j] for j in range(nblk)), dtype)
    w = as_dt(Vf @ rng.standard_normal((nblk * bs, bs)) * 1e-3 + rng.standard_normal((n, bs)), dtype)
    eps = 1e-12 if dtype == torch.float64 else 2e-6
    est = np.linalg.norm(S.T @ w) / np.linalg.norm(w)
    for thr, projected in ((est / 100, True), (est * 100, False)):
        Wd = dev(w, dtype)
        G = torch.zeros((bs, bs), dtype=torch.float64, device="cuda")
        cuda_handle.project_out_sketch(dev(V, dtype), Wd, dev(S, dtype), thr, G)
        got = host(Wd)
        if projected:
            Wr = dev(w, dtype)
            Gr = torch.zeros((bs, bs), dtype=torch.float64, device="cuda")
            cuda_handle.project_out(dev(V, dtype), Wr, native.TRL_CGS_IFNEEDED, Gr)
            close(got, host(Wr), np.abs(w).max(), eps)
            close(host(G), host(Gr), np.abs(host(Gr)).max(), 1e-12)
            assert np.abs(Vf.T @ got).max() < 1e3 * eps * np.abs(got).max()
        else:
            assert np.array_equal(got, w)
            close(host(G), w.T @ w, np.abs(w.T @ w).max(), 1e-12 if dtype == torch.float64 else 1e-6)


@pytest.mark.parametrize("dtype", DT)
def test_project_out_sketch_pairs(cuda_handle, dtype):
    """With a pair state, a step whose sketch test fired also projects the next step (one
    step only: a forced projection forces nothing). 'loud' blocks exceed the threshold 100x;
    'quiet' ones carry a component along V 10x below it, which a projection removes and
    which otherwise stays bit for bit."""
    bs, n, nblk = 8, 2003, 5
    rng = np.random.default_rng(5)
    Q, _ = np.linalg.qr(rng.standard_normal((n, nblk * bs)))
    V = as_dt(Q.reshape(n, nblk, bs).transpose(1, 0, 2).copy(), dtype)
    Vf = V.transpose(1, 0, 2).reshape(n, nblk * bs)
    Gc = rng.standard_normal((nblk, bs, bs)) / np.sqrt(bs)
    S = as_dt(sum(V[j] @ Gc[j] for j in range(nblk)), dtype)

    def block(scale):
        r = rng.standard_normal((n, bs))
        r -= Vf @ (Vf.T @ r)
        return as_dt(r + scale * (Vf @ rng.standard_normal((nblk * bs, bs))), dtype)

    def est(x):
        return np.linalg.norm(S.T @ x) / np.linalg.norm(x)

    loud = block(0.3)
    thr = est(loud) / 100
    quiet = block(0.3 / 1000)
    assert est(quiet) < thr / 3
    seq = [quiet, loud, quiet, quiet, loud, loud, quiet, quiet]
    eps = 1e-12 if dtype == torch.float64 else 2e-6
    for pairs, expect in ((True, [0, 1, 1, 0, 1, 1, 1, 0]), (False, [0, 1, 0, 0, 1, 1, 0, 0])):
        state = torch.zeros(1, dtype=torch.int32, device="cuda") if pairs else None
        got = []
        for x in seq:
            Wd = dev(x, dtype)
            G = torch.zeros((bs, bs), dtype=torch.float64, device="cuda")
            cuda_handle.project_out_sketch(dev(V, dtype), Wd, dev(S, dtype), thr, G, pair_state=state)
            out = host(Wd)
            if np.array_equal(out, x):
                got.append(0)
            else:
                assert np.abs(Vf.T @ out).max() < 1e3 * eps * np.abs(out).max()
                got.append(1)
        assert got == expect, (pairs, got)
        if pairs:
            assert int(state.item()) == 0  # the last step's test did not fire


def _random_csr(n, rng, max_deg=40, empty_frac=0.1):
    deg = rng.integers(0, max_deg, size=n)
    deg[rng.random(n) < empty_frac] = 0
    rows = np.repeat(np.arange(n), deg)
    cols = rng.integers(0, n, size=rows.size)
    vals = rng.standard_normal(rows.size)
    key = np.unique(rows.astype(np.int64) * n + cols)
    rows, cols = key // n, key % n
    vals = rng.standard_normal(rows.size)
    return P._from_coo(n, rows, cols, vals)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 3.5)])
def test_spmm_matches_reference(cuda_handle, oracle, bs, alpha, beta):
    rng = np.random.default_rng(bs)
    for A in (P.laplace2d(64), _random_csr(7919, rng), P.diagonal(5)):
        X = rng.standard_normal((A.n, bs))
        ref = oracle.spmm(A, X, alpha, beta)  # examples/sycl/csrevp.hh:159-187 semantics
        Ad = native.DeviceCSRTensors.from_host(A)
        Yd = torch.zeros((A.n, bs), dtype=torch.float64, device="cuda")
        cuda_handle.spmm(Ad, dev(X), Yd, alpha, beta)
        rows = A.row_indices()
        mag = np.zeros(A.n)
        np.add.at(mag, rows, np.abs(A.values) * np.abs(X[A.colind]).max(axis=1))
        close(host(Yd), ref, mag.max() + abs(beta) * np.abs(X).max())


@pytest.mark.parametrize("bs", [4, 8, 16])
def test_spmm_fp32(cuda_handle, oracle, bs):
    rng = np.random.default_rng(5)
    A = _random_csr(10007, rng, max_deg=100)
    X = rng.standard_normal((A.n, bs)).astype(np.float32).astype(np.float64)
    ref = oracle.spmm(A, X)
    Ad = native.DeviceCSRTensors.from_host(A, torch.float32)
    Yd = torch.zeros((A.n, bs), dtype=torch.float32, device="cuda")
    cuda_handle.spmm(Ad, dev(X, torch.float32), Yd)
    scale = np.abs(ref).max()
    close(host(Yd), ref, scale, 1e-5)


def test_spmm_rejects_bad_arguments(cuda_handle):
    A = native.DeviceCSRTensors.from_host(P.laplace1d(16))
    X = torch.zeros((16, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(native.TrlError) as e:
        cuda_handle.spmm(A, X, torch.zeros_like(X))
    assert e.value.status == native.TRL_ENOTSUP
    X = torch.zeros((16, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(native.TrlError) as e:
        cuda_handle.spmm(A, X, X)
    assert e.value.status == native.TRL_EINVAL


@pytest.mark.parametrize("bs,nblk", [(1, 7), (4, 10), (8, 12), (16, 4)])
def test_small_eigen_matches_reference(cuda_handle, oracle, bs, nblk):
    rng = np.random.default_rng(bs * nblk)
    N = bs * nblk
    M = rng.standard_normal((N, N))
    D = M + M.T
    # block layout with a garbage upper triangle: both implementations read the lower one
    T = D.reshape(nblk, bs, nblk, bs).transpose(0, 2, 1, 3).copy()
    beta = np.triu(rng.standard_normal((bs, bs))) * 1e-7
    nev = min(N, 2 * bs + 1)
    ev_ref, Y_ref, nc_ref = oracle.solve_small_dense(T, beta, bs, nev, tol=1e-7)
    evals, evecs, ev_host, nconv = cuda_handle.small_eigen(dev(T), dev(beta), nev, 1e-7)
    assert np.allclose(ev_host, ev_ref, rtol=0, atol=1e-12 * np.abs(ev_ref).max())
    assert np.allclose(host(evals), ev_host)
    Yg = host(evecs).transpose(0, 2, 1, 3).reshape(N, N)
    Yr = Y_ref.transpose(0, 2, 1, 3).reshape(N, N)
    signs = np.sign(np.sum(Yg * Yr, axis=0))
    assert np.allclose(Yg * signs, Yr, atol=1e-10)
    assert nconv == nc_ref


def _block_layout(D, bs, rng=None):
    """Dense symmetric D as a block matrix; the upper triangle is overwritten with garbage
    (both eigensolvers read the lower one)."""
    N = D.shape[0]
    nblk = N // bs
    M = D.copy()
    if rng is not None:
        iu = np.triu_indices(N, 1)
        M[iu] = rng.standard_normal(iu[0].size)
    return M.reshape(nblk, bs, nblk, bs).transpose(0, 2, 1, 3).copy()


def _spectrum_matrix(lam, rng):
    N = lam.size
    Q, _ = np.linalg.qr(rng.standard_normal((N, N)))
    return (Q * lam) @ Q.T


def _partial_cases():
    rng = np.random.default_rng(2024)
    cases = []
    # 448: the 8-CTA cluster with shared-memory rows; 512, 640: 16 CTAs, shared-memory rows;
    # 768, 1024: 16 CTAs, rows in global memory
    for N, bs in ((40, 8), (160, 4), (384, 8), (448, 16), (512, 16), (640, 16), (768, 16), (1024, 16)):
        M = rng.standard_normal((N, N))
        cases.append((f"random{N}", M + M.T, bs))
    # exact degenerate pairs and a tight cluster at the wanted end (relative gaps 1e-9)
    lam = np.linspace(-3.0, 1.0, 384)
    lam[-1] = lam[-2] = 5.0
    lam[-10:-2] = 4.0 + 1e-9 * np.arange(8)
    cases.append(("clustered384", _spectrum_matrix(lam, rng), 8))
    # thick-restart projected matrices: kept Ritz values on the diagonal, coupling to the
    # next block, block-tridiagonal below (the structure lanczos.hh:119-150 builds); the
    # second has the shape of the 4M-row bandwidth-stress solve at block size 16 (N = 512,
    # 100 wanted, 112 kept vectors: the Gram-Schmidt of the kept vectors in global memory)
    for bs, nblk, kr, nev in ((8, 48, 5, None), (16, 32, 7, 100)):
        N = nblk * bs
        T = np.zeros((N, N))
        T[: kr * bs, : kr * bs] = np.diag(np.sort(rng.uniform(440, 444, kr * bs))[::-1])
        for b in range(kr, nblk):
            D = rng.standard_normal((bs, bs)) * 50 + np.eye(bs) * 200
            T[b * bs:(b + 1) * bs, b * bs:(b + 1) * bs] = D + D.T
            if b + 1 < nblk:
                Bt = np.triu(rng.standard_normal((bs, bs))) * 20
                T[(b + 1) * bs:(b + 2) * bs, b * bs:(b + 1) * bs] = Bt
                T[b * bs:(b + 1) * bs, (b + 1) * bs:(b + 2) * bs] = Bt.T
        C = rng.standard_normal((bs, kr * bs)) * 1e-3
        T[kr * bs:(kr + 1) * bs, : kr * bs] = C
        T[: kr * bs, kr * bs:(kr + 1) * bs] = C.T
        cases.append((f"restart{N}", T, bs) + ((nev,) if nev else ()))
    # kept Ritz values on both sides of zero whose couplings to the next block are ~1e-160
    # (fully converged pairs): the squares of those entries underflow, and a Householder
    # reflector built from their norm is not orthogonal unless they are treated as zero (the
    # shape of the 524,288-row Zipf solve at block size 8)
    bs, nblk, kr = 8, 32, 13
    N = nblk * bs
    T = np.zeros((N, N))
    kept = np.concatenate([rng.uniform(26.0, 27.0, kr * bs // 2), -rng.uniform(26.0, 27.0, kr * bs - kr * bs // 2)])
    T[: kr * bs, : kr * bs] = np.diag(kept[np.argsort(-np.abs(kept))])
    for b in range(kr, nblk):
        D = rng.standard_normal((bs, bs)) * 5
        T[b * bs:(b + 1) * bs, b * bs:(b + 1) * bs] = D + D.T
        if b + 1 < nblk:
            Bt = np.triu(rng.standard_normal((bs, bs))) * 8
            T[(b + 1) * bs:(b + 2) * bs, b * bs:(b + 1) * bs] = Bt
            T[b * bs:(b + 1) * bs, (b + 1) * bs:(b + 2) * bs] = Bt.T
    C = rng.standard_normal((bs, kr * bs)) * 1e-4
    C[:, :4] *= 1e-156
    T[kr * bs:(kr + 1) * bs, : kr * bs] = C
    T[: kr * bs, kr * bs:(kr + 1) * bs] = C.T
    cases.append(("restart_tiny_coupling256", T, bs, 100))
    return cases


@pytest.mark.parametrize("case", _partial_cases(), ids=lambda c: c[0])
def test_small_eigen_partial_matches_full(cuda_handle, oracle, case):
    """The kept-vectors eigensolver (cluster tridiagonalisation, bisection, inverse iteration)
    against cuSOLVER's full syevd path and the oracle: all eigenvalues, the first kvec
    eigenvectors (residual, orthogonality, and the spanned subspace of each cluster), the
    zeroed remaining columns, and the convergence count."""
    name, D, bs = case[:3]
    rng = np.random.default_rng(7)
    N = D.shape[0]
    T = _block_layout(D, bs, rng)
    beta = np.triu(rng.standard_normal((bs, bs))) * 1e-9
    nev = case[3] if len(case) > 3 else 2 * bs
    kvec = min(N, (nev // bs + 1) * bs)
    ev_ref, Y_ref, nc_ref = oracle.solve_small_dense(T, beta, bs, nev, tol=1e-7)
    for rep in range(2):  # the second call runs on the workspace the first one left
        evals, evecs, hev, nconv = cuda_handle.small_eigen_partial(dev(T), dev(beta), nev, 1e-7, kvec)
        nrm = np.abs(ev_ref).max()
        assert np.allclose(hev, ev_ref, rtol=0, atol=1e-12 * nrm)
        assert np.array_equal(host(evals), hev)
        Yg = host(evecs).transpose(0, 2, 1, 3).reshape(N, N)
        X = Yg[:, :kvec]
        assert np.all(Yg[:, kvec:] == 0.0)
        # residual and orthogonality of the returned vectors
        R = D @ X - X * hev[:kvec]
        assert np.abs(R).max() < 1e-11 * nrm, np.abs(R).max() / nrm
        assert np.abs(X.T @ X - np.eye(kvec)).max() < 1e-11
        # same invariant subspaces as the reference: clusters of eigenvalues closer than
        # 1e-6 ||T|| compared as subspaces
        Xr = Y_ref.transpose(0, 2, 1, 3).reshape(N, N)[:, :kvec]
        c0 = 0
        while c0 < kvec:
            c1 = c0 + 1
            while c1 < kvec and abs(ev_ref[c1] - ev_ref[c1 - 1]) < 1e-6 * nrm:
                c1 += 1
            if c1 == kvec and c1 < N and abs(ev_ref[c1] - ev_ref[c1 - 1]) < 1e-6 * nrm:
                break  # the last cluster continues past kvec: its span is not determined by kvec columns
            s = np.linalg.svd(Xr[:, c0:c1].T @ X[:, c0:c1], compute_uv=False)
            assert s.min() > 1 - 1e-9, (name, c0, c1, s.min())
            c0 = c1
        assert nconv == nc_ref
        full = cuda_handle.small_eigen(dev(T), dev(beta), nev, 1e-7)
        assert np.allclose(hev, full[2], rtol=0, atol=1e-12 * nrm)


def test_small_eigen_partial_rejects_bad_kvec(cuda_handle):
    T = torch.zeros((4, 4, 4, 4), dtype=torch.float64, device="cuda")
    beta = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(native.TrlError) as e:
        cuda_handle.small_eigen_partial(T, beta, 4, 1e-8, 17)
    assert e.value.status == native.TRL_EINVAL


def test_sddmm_matches_dense(cuda_handle):
    rng = np.random.default_rng(11)
    A = _random_csr(3001, rng)
    k = 5
    X = rng.standard_normal((A.n, k))
    w = rng.uniform(size=k)
    out = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    cuda_handle.sddmm(native.DeviceCSRTensors.from_host(A), dev(X), dev(w), out)
    rows = A.row_indices()
    ref = np.sum(w * X[rows] * X[A.colind], axis=1)
    close(host(out), ref, np.abs(ref).max() + 1e-300)


def test_convert_and_norm1(cuda_handle):
    A = P.anisotropic3d(8)
    Ad = native.DeviceCSRTensors.from_host(A)
    assert cuda_handle.csr_norm1(Ad) == pytest.approx(A.gershgorin_bound(), rel=1e-15)
    sig = 500.0
    assert cuda_handle.csr_norm1(Ad, -1.0, sig) == pytest.approx(
        np.max(np.abs(sig - np.diag(A.to_dense())) + np.abs(A.to_dense() - np.diag(np.diag(A.to_dense()))).sum(1)), rel=1e-14)
    x = torch.randn(1000, dtype=torch.float64, device="cuda")
    y = torch.empty(1000, dtype=torch.float32, device="cuda")
    cuda_handle.convert(y, x)
    torch.cuda.synchronize()
    assert torch.equal(y, x.float())


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
def test_spmm_on_elasticity_and_zipf_patterns(cuda_handle, oracle, bs, dtype):
    """The structures of the mixed-precision and bandwidth-stress workloads at small size:
    81 entries per row in 3x3 node blocks (elasticity, 27-point coupling) and heavy-tailed
    row lengths up to the cap (Zipf(1.5) degrees, mirrored)."""
    rng = np.random.default_rng(17 * bs)
    for A in (P.elasticity27(7, seed=3), P.zipf_symmetric(6000, cap=512, seed=4)):
        X = as_dt(rng.standard_normal((A.n, bs)), dtype)
        vals = A.values.astype(np.float32).astype(np.float64) if dtype == torch.float32 else A.values
        Ah = P.CSRMatrix(A.n, A.rowptr, A.colind, vals)
        ref = oracle.spmm(Ah, X)
        Ad = native.DeviceCSRTensors.from_host(Ah, dtype)
        Yd = torch.zeros((A.n, bs), dtype=dtype, device="cuda")
        cuda_handle.spmm(Ad, dev(X, dtype), Yd)
        rows = A.row_indices()
        mag = np.zeros(A.n)
        np.add.at(mag, rows, np.abs(vals) * np.abs(X[A.colind]).max(axis=1))
        # FP64 to rounding; FP32 accumulates in FP32 (relative to the summed magnitudes)
        close(host(Yd), ref, mag.max(), 1e-12 if dtype == torch.float64 else 2e-6)


def _long_row_csr(rng, n=4099):
    """Short rows (0-5 entries) around long ones placed where the warp-wide sweep of long
    rows has its edge cases: every 37th row 33-699 entries (longer than a stage chunk), the
    last row of a 4/8/16/32-row warp iteration, an iteration of mixed long rows (64-71),
    rows of exactly 32 (not swept) and 33 entries alone in an iteration, and a long last
    row with n a multiple of no iteration width."""
    deg = rng.integers(0, 6, size=n)
    every = np.arange(n) % 37 == 5
    deg[every] = rng.integers(33, 700, size=every.sum())
    deg[[7, 15, 31, 63]] = 400
    deg[64:72] = [33, 40, 50, 300, 500, 33, 64, 129]
    deg[128:136] = [32, 0, 0, 0, 0, 0, 0, 0]
    deg[136:144] = [33, 0, 0, 0, 0, 0, 0, 0]
    deg[n - 1] = 600
    rows = np.repeat(np.arange(n), deg)
    cols = np.concatenate([rng.choice(n, size=d, replace=False) for d in deg])
    return P._from_coo(n, rows, cols, rng.standard_normal(rows.size))


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
def test_spmm_long_rows_swept_by_the_warp(cuda_handle, oracle, bs, dtype):
    """Rows much longer than their warp iteration's mean are summed by all row groups of
    the warp; the one-block entry points (plain and three-term) and the multi-block one
    (which walks them per row) all match the oracle."""
    rng = np.random.default_rng(23)
    A = _long_row_csr(rng)
    vals = A.values.astype(np.float32).astype(np.float64) if dtype == torch.float32 else A.values
    Ah = P.CSRMatrix(A.n, A.rowptr, A.colind, vals)
    Ad = native.DeviceCSRTensors.from_host(Ah, dtype)
    X = as_dt(rng.standard_normal((2, A.n, bs)), dtype)
    W = as_dt(rng.standard_normal((A.n, bs)), dtype)
    rows = A.row_indices()
    mag = np.zeros(A.n)
    np.add.at(mag, rows, np.abs(vals) * np.abs(X).max(axis=(0, 2))[A.colind])
    tol = 1e-12 if dtype == torch.float64 else 2e-6
    Yd = torch.full((A.n, bs), float("nan"), dtype=dtype, device="cuda")
    cuda_handle.spmm(Ad, dev(X[0], dtype), Yd)
    close(host(Yd), oracle.spmm(Ah, X[0]), mag.max(), tol)
    alpha, beta, gamma = -0.5, 2.0, 0.25
    ref = np.stack([oracle.spmm(Ah, X[j], alpha, beta) for j in range(2)])
    scale = abs(alpha) * mag.max() + abs(beta) * np.abs(X).max() + abs(gamma) * np.abs(W).max()
    Yd = dev(W, dtype)
    cuda_handle.spmm3(Ad, dev(X[0], dtype), Yd, alpha, beta, gamma, Yd)
    close(host(Yd), ref[0] + gamma * W, scale, tol)
    Yd = torch.full((2, A.n, bs), float("nan"), dtype=dtype, device="cuda")
    cuda_handle.spmm_blocks(Ad, dev(X, dtype), Yd, alpha, beta, 0.0, None)
    close(host(Yd), ref, scale, tol)


@pytest.mark.parametrize("bs", BS)
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("nb", [1, 3, 5])
def test_spmm_blocks_three_term(cuda_handle, oracle, bs, dtype, nb):
    """Y_j = alpha A X_j + beta X_j + gamma W_j on nb blocks in one call, with W = Y (the
    Chebyshev filter's in-place recurrence), W separate and W absent. Short rows stage each
    warp's CSR range once for all blocks; long rows (Zipf degrees) take the chunked path."""
    rng = np.random.default_rng(31 * bs + nb)
    tol = 1e-12 if dtype == torch.float64 else 2e-6
    for A in (P.anisotropic3d(9), P.zipf_symmetric(4000, cap=400, seed=9)):
        vals = A.values.astype(np.float32).astype(np.float64) if dtype == torch.float32 else A.values
        Ah = P.CSRMatrix(A.n, A.rowptr, A.colind, vals)
        Ad = native.DeviceCSRTensors.from_host(Ah, dtype)
        X = as_dt(rng.standard_normal((nb, A.n, bs)), dtype)
        W = as_dt(rng.standard_normal((nb, A.n, bs)), dtype)
        alpha, beta, gamma = 0.75, -1.25, 0.5
        ref = np.stack([oracle.spmm(Ah, X[j], alpha, beta) for j in range(nb)])
        rows = A.row_indices()
        mag = np.zeros(A.n)
        np.add.at(mag, rows, np.abs(vals) * np.abs(X).max(axis=(0, 2))[A.colind])
        scale = abs(alpha) * mag.max() + abs(beta) * np.abs(X).max() + abs(gamma) * np.abs(W).max()
        Xd = dev(X, dtype)
        # W separate
        Yd = torch.full((nb, A.n, bs), float("nan"), dtype=dtype, device="cuda")
        cuda_handle.spmm_blocks(Ad, Xd, Yd, alpha, beta, gamma, dev(W, dtype))
        close(host(Yd), ref + gamma * W, scale, tol)
        # W = Y, updated in place
        Yd = dev(W, dtype)
        cuda_handle.spmm_blocks(Ad, Xd, Yd, alpha, beta, gamma, Yd)
        close(host(Yd), ref + gamma * W, scale, tol)
        # no W: matches the one-block entry point block by block - bit for bit where no row
        # is swept by the whole warp (the stencil); the multi-block walk takes Zipf's long
        # rows per row, in another summation order
        Yd = torch.full((nb, A.n, bs), float("nan"), dtype=dtype, device="cuda")
        cuda_handle.spmm_blocks(Ad, Xd, Yd, alpha, beta, 0.0, None)
        for j in range(nb):
            Y1 = torch.empty((A.n, bs), dtype=dtype, device="cuda")
            cuda_handle.spmm3(Ad, Xd[j], Y1, alpha, beta, 0.0, None)
            if np.diff(A.rowptr).max() > 32:
                close(host(Yd[j]), host(Y1), scale, tol)
            else:
                assert torch.equal(Yd[j], Y1)
        close(host(Yd), ref, scale, tol)


def test_spmm_blocks_rejects_bad_block_count(cuda_handle):
    A = native.DeviceCSRTensors.from_host(P.laplace1d(16))
    X = torch.zeros((0, 16, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(native.TrlError) as e:
        cuda_handle.spmm_blocks(A, X, X, 1.0, 0.0, 0.0, None)
    assert e.value.status == native.TRL_EINVAL


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.0, 40.0), (2.5, -3.0)])
def test_csr_gershgorin_interval(cuda_handle, alpha, beta):
    rng = np.random.default_rng(3)
    for A in (P.anisotropic3d(6), _random_csr(2003, rng)):
        D = alpha * A.to_dense() + beta * np.eye(A.n)
        c = np.diag(D)
        r = np.abs(D).sum(axis=1) - np.abs(c)
        for dtype in DT:
            vals = A.values.astype(np.float32).astype(np.float64) if dtype == torch.float32 else A.values
            Ad = native.DeviceCSRTensors.from_host(P.CSRMatrix(A.n, A.rowptr, A.colind, vals), dtype)
            lo, hi = cuda_handle.csr_gershgorin(Ad, alpha, beta)
            if dtype == torch.float64:
                assert lo == pytest.approx((c - r).min(), rel=1e-13, abs=1e-13)
                assert hi == pytest.approx((c + r).max(), rel=1e-13, abs=1e-13)
            ev = np.linalg.eigvalsh(alpha * P.CSRMatrix(A.n, A.rowptr, A.colind, vals).to_dense() + beta * np.eye(A.n)) if A.n < 600 else None
            if ev is not None:
                assert lo <= ev.min() + 1e-9 and hi >= ev.max() - 1e-9
