"""Adjoint of weighted eigenvalue sums (trl_cuda_eigen_adjoint, an SDDMM over the CSR pattern).

Problem: K x = lambda M x on an m x m grid, K a 5-point diffusion operator with log-normal
edge conductivities (Dirichlet boundary edges), M a lumped mass U[0.5, 1.5]; f = sum_c w_c
lambda_c over the smallest k eigenvalues, w_c ~ U(0, 1). Checks:
  * the SDDMM gradient equals the dense FP64 formula evaluated from the same eigenvectors;
  * central finite differences of f on 50 random entries (edges and masses) of the 64 x 64
    variant, eigenvalues from a shift-invert Lanczos (scipy ARPACK, relative accuracy),
    agree with the adjoint to 1e-6 relative;
  * near-degenerate clusters: with cluster-averaged weights the gradient of f is that of the
    cluster sums and does not depend on the basis chosen inside a degenerate eigenspace;
  * the full GPU path (block Lanczos on the shifted operator -> eigenvectors -> adjoint) on a
    small grid, wrapped in a torch.autograd.Function (test harness only).
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from trl_b200 import generalized as G
from trl_b200 import native
from trl_b200 import problems as P

pytestmark = pytest.mark.gpu


def scipy_csr(A):
    return sp.csr_matrix((A.values, A.colind, A.rowptr), shape=(A.n, A.n))


def smallest_pairs(K, mass, k):
    """Reference eigenpairs of K x = lambda M x by shift-invert Lanczos (ARPACK) around 0:
    relative accuracy for the small eigenvalues. x is M-normalised."""
    Ks = scipy_csr(K)
    Ms = sp.diags(mass)
    lam, X = spla.eigsh(Ks, k=k, M=Ms, sigma=0.0, which="LM", tol=0)
    order = np.argsort(lam)
    lam, X = lam[order], X[:, order]
    X = X / np.sqrt(np.einsum("ic,i,ic->c", X, mass, X))
    return lam, X


def f_value(K, mass, w, k):
    lam, _ = smallest_pairs(K, mass, k)
    return float(np.dot(w, lam))


def grad_from_vectors(h, K, mass, edges, X, lam, w, cluster_rtol=1e-8):
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    return G.eigen_sum_gradient(h, K, K.n, edges, Xd, lam, w, cluster_rtol=cluster_rtol)


@pytest.fixture(scope="module")
def grid64():
    K, mass, edges = P.diffusion2d_mass(64, sigma=1.0, seed=3)
    k = 16
    w = np.random.default_rng(4).uniform(size=k)
    lam, X = smallest_pairs(K, mass, k)
    return K, mass, edges, w, lam, X


def test_sddmm_matches_dense_formula(cuda_handle, grid64):
    K, mass, edges, w, lam, X = grid64
    dk, dm = grad_from_vectors(cuda_handle, K, mass, edges, X, lam, w, cluster_rtol=0.0)
    a, b = edges["a"], edges["b"]
    xb = np.where((b >= 0)[:, None], X[np.maximum(b, 0)], 0.0)
    dk_ref = np.einsum("c,ec->e", w, (X[a] - xb) ** 2)
    dm_ref = -np.einsum("c,c,ic->i", w, lam, X ** 2)
    assert np.max(np.abs(dk - dk_ref)) <= 1e-12 * np.abs(dk_ref).max()
    assert np.max(np.abs(dm - dm_ref)) <= 1e-12 * np.abs(dm_ref).max()


def _fd4(f, x0, h):
    """Fourth-order central difference (truncation O(h^4))."""
    return (-f(x0 + 2 * h) + 8 * f(x0 + h) - 8 * f(x0 - h) + f(x0 - 2 * h)) / (12 * h)


def test_gradient_matches_central_differences_50_entries(cuda_handle, grid64):
    """50 random entries (35 edge conductivities, 15 masses). The error of each entry is taken
    relative to the largest gradient entry of its kind: entries whose own gradient is tiny
    are limited by the eigenvalue accuracy of the finite differences, not by the adjoint."""
    K, mass, edges, w, lam, X = grid64
    dk, dm = grad_from_vectors(cuda_handle, K, mass, edges, X, lam, w)
    rng = np.random.default_rng(11)
    e_idx = rng.choice(edges["a"].size, size=35, replace=False)
    m_idx = rng.choice(mass.size, size=15, replace=False)
    errs = []
    for e in e_idx:
        def fk(v, e=e):
            kap = edges["kappa"].copy()
            kap[e] = v
            return f_value(P.assemble_diffusion(K.n, edges["a"], edges["b"], kap), mass, w, lam.size)
        fd = _fd4(fk, edges["kappa"][e], 1e-3 * edges["kappa"][e])
        errs.append(abs(fd - dk[e]) / np.abs(dk).max())
    for i in m_idx:
        def fmass(v, i=i):
            ms = mass.copy()
            ms[i] = v
            return f_value(K, ms, w, lam.size)
        fd = _fd4(fmass, mass[i], 1e-3 * mass[i])
        errs.append(abs(fd - dm[i]) / np.abs(dm).max())
    assert max(errs) < 1e-6, sorted(errs)[-5:]


def test_degenerate_clusters_give_basis_independent_gradient(cuda_handle):
    m = 16
    n = m * m
    idx = np.arange(n).reshape(m, m)
    a = np.concatenate([idx[:, :-1].ravel(), idx[:-1, :].ravel(), idx[:, 0], idx[:, -1], idx[0, :], idx[-1, :]])
    b = np.concatenate([idx[:, 1:].ravel(), idx[1:, :].ravel()] + [np.full(m, -1)] * 4)
    edges = {"a": a, "b": b, "kappa": np.ones(a.size)}
    K = P.assemble_diffusion(n, a, b, edges["kappa"])
    mass = np.ones(n)
    k = 8  # (1,1), (1,2)+(2,1), (2,2), (1,3)+(3,1), (2,3)+(3,2): ends on a complete cluster
    lam, X = np.linalg.eigh(K.to_dense())
    lam, X = lam[:k], X[:, :k]
    rng = np.random.default_rng(5)
    w = rng.uniform(size=k)
    # rotate each exactly degenerate pair by a random angle: individual eigenvectors change
    Xr = X.copy()
    for s in range(k - 1):
        if abs(lam[s + 1] - lam[s]) < 1e-10:
            t = rng.uniform(0, np.pi)
            c, si = np.cos(t), np.sin(t)
            Xr[:, [s, s + 1]] = X[:, [s, s + 1]] @ np.array([[c, -si], [si, c]])
    g1, m1 = grad_from_vectors(cuda_handle, K, mass, edges, X, lam, w)
    g2, m2 = grad_from_vectors(cuda_handle, K, mass, edges, Xr, lam, w)
    assert np.max(np.abs(g1 - g2)) < 1e-12 * np.abs(g1).max()
    assert np.max(np.abs(m1 - m2)) < 1e-12 * np.abs(m1).max()
    # without the cluster averaging the two bases disagree
    h1, _ = grad_from_vectors(cuda_handle, K, mass, edges, X, lam, w, cluster_rtol=0.0)
    h2, _ = grad_from_vectors(cuda_handle, K, mass, edges, Xr, lam, w, cluster_rtol=0.0)
    assert np.max(np.abs(h1 - h2)) > 1e-6 * np.abs(h1).max()
    # and the averaged gradient is the derivative of the cluster sums (central differences)
    wbar = w.copy()
    s = 0
    while s < k:
        e = s + 1
        while e < k and abs(lam[e] - lam[e - 1]) < 1e-8 * abs(lam).max():
            e += 1
        wbar[s:e] = w[s:e].mean()
        s = e
    for ei in (0, 7, 100, 400):
        def fc(v, ei=ei):
            kap = edges["kappa"].copy()
            kap[ei] = v
            return np.dot(wbar, np.linalg.eigvalsh(P.assemble_diffusion(n, a, b, kap).to_dense())[:k])
        assert abs(_fd4(fc, 1.0, 1e-3) - g1[ei]) < 1e-6 * np.abs(g1).max()


class EigenSum(torch.autograd.Function):
    """f(kappa, mass) = sum_c w_c lambda_c(K(kappa), M(mass)) over the smallest k eigenpairs,
    forward by the GPU block Lanczos, backward by the adjoint SDDMM (test harness only)."""

    @staticmethod
    def forward(ctx, kappa, mass, edges, w, k, handle):
        kap = kappa.detach().cpu().numpy()
        ms = mass.detach().cpu().numpy()
        K = P.assemble_diffusion(ms.size, edges["a"], edges["b"], kap)
        X0 = P.initial_block(K.n, 4, seed=1)
        lam, X, info = G.solve_smallest(handle, K, ms, nev=k, bs=4, ncv=64, X0=X0, tol=1e-12)
        assert info["converged"], info
        ctx.save_for_backward(kappa, mass)
        ctx.stuff = (K, edges, X, lam, w, handle)
        return torch.tensor(float(np.dot(w, lam)), dtype=torch.float64)

    @staticmethod
    def backward(ctx, gout):
        K, edges, X, lam, w, handle = ctx.stuff
        dk, dm = G.eigen_sum_gradient(handle, K, K.n, edges, X, lam, w)
        return torch.from_numpy(dk) * gout, torch.from_numpy(dm) * gout, None, None, None, None


def test_autograd_function_through_the_gpu_solver(cuda_handle):
    K, mass, edges = P.diffusion2d_mass(24, sigma=0.5, seed=8)
    k = 4
    w = np.random.default_rng(9).uniform(size=k)
    kappa = torch.tensor(edges["kappa"], requires_grad=True)
    mt = torch.tensor(mass, requires_grad=True)
    f = EigenSum.apply(kappa, mt, edges, w, k, cuda_handle)
    lam_ref, X_ref = smallest_pairs(K, mass, k)
    assert abs(float(f) - np.dot(w, lam_ref)) < 1e-9 * abs(np.dot(w, lam_ref))
    f.backward()
    dk_ref, dm_ref = grad_from_vectors(cuda_handle, K, mass, edges, X_ref, lam_ref, w)
    assert np.max(np.abs(kappa.grad.numpy() - dk_ref)) < 1e-6 * np.abs(dk_ref).max()
    assert np.max(np.abs(mt.grad.numpy() - dm_ref)) < 1e-6 * np.abs(dm_ref).max()


def _identity_difference(K, mass, edges, which, idx, h, Xp, Xm, lam_m):
    """lambda_+ - lambda_- for every pair from the eigenvectors of the two perturbed problems,
    through the exact identities (K symmetric, x_+ and x_- exact eigenvectors):
      edge e (kappa_e scaled by 1 +- h):  (lambda_+ - lambda_-) x_+^T M x_- = x_-^T (K_+ - K_-) x_+
                                          = 2 h kappa_e (x_+[a] - x_+[b]) (x_-[a] - x_-[b]);
      mass i (m_i scaled by 1 +- h):      (lambda_+ - lambda_-) x_-^T M_+ x_+ = -lambda_- x_+^T (M_+ - M_-) x_-
                                          = -lambda_- 2 h m_i x_+[i] x_-[i].
    They give the difference of the two solves' eigenvalues without the cancellation of
    subtracting two nearly equal numbers (the smallest eigenvalues are ~1e-6 of the operator's
    norm here)."""
    if which == "edge":
        a, b = edges["a"][idx], edges["b"][idx]
        dp = Xp[a] - (Xp[b] if b >= 0 else 0.0)
        dm = Xm[a] - (Xm[b] if b >= 0 else 0.0)
        return 2 * h * edges["kappa"][idx] * dp * dm / np.einsum("ic,i,ic->c", Xp, mass, Xm)
    mp = mass.copy()
    mp[idx] *= 1 + h
    return -lam_m * 2 * h * mass[idx] * Xp[idx] * Xm[idx] / np.einsum("ic,i,ic->c", Xm, mp, Xp)


@pytest.mark.slow
def test_full_size_gradient_against_finite_differences(cuda_handle):
    """The 512 x 512 generalised problem (n = 262,144): the 16 smallest eigenpairs by the
    mixed-precision solver to 1e-12, the adjoint gradient of f = sum w_c lambda_c over every edge
    conductivity and mass, and central finite differences (relative step 1e-3) on 50 random
    entries (25 edges, 25 masses), each from two perturbed GPU solves."""
    K, mass, edges = P.diffusion2d_mass(512, sigma=1.0, seed=42)
    k, bs, ncv, tol, hstep = 16, 8, 256, 1e-12, 1e-3
    w = np.random.default_rng(7).uniform(size=k)
    X0 = P.initial_block(K.n, bs, seed=42)
    mode = native.TRL_MODE_MIXED

    def solve(Kx, mx):
        # the Chebyshev refinement, as the automatic choice takes it here: 0.55 s a solve
        # against ~8 s for the Lanczos refinement at these relative gaps (1e-7)
        lam, X, out = G.solve_smallest(cuda_handle, Kx, mx, k, bs, ncv, X0, tol=tol, mode=mode, refine=native.TRL_REFINE_CHEBYSHEV)
        assert out["converged"] and out["max_theta_residual"] < 10 * tol
        order = np.argsort(lam)
        return lam[order], X[:, order].cpu().numpy()

    lam, X = solve(K, mass)
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    dk, dm = G.eigen_sum_gradient(cuda_handle, K, K.n, edges, Xd, lam, w)
    rng = np.random.default_rng(11)
    picks = [("edge", int(i)) for i in rng.choice(edges["a"].size, 25, replace=False)] + [("mass", int(i)) for i in rng.choice(K.n, 25, replace=False)]
    errs = []
    for which, idx in picks:
        res = []
        for s in (+1, -1):
            if which == "edge":
                kap = edges["kappa"].copy()
                kap[idx] *= 1 + s * hstep
                res.append(solve(P.assemble_diffusion(K.n, edges["a"], edges["b"], kap), mass))
            else:
                mm = mass.copy()
                mm[idx] *= 1 + s * hstep
                res.append(solve(K, mm))
        (lp, Xp), (lm, Xm) = res
        d = _identity_difference(K, mass, edges, which, idx, hstep, Xp, Xm, lm)
        p = edges["kappa"][idx] if which == "edge" else mass[idx]
        fd = float(np.dot(w, d)) / (2 * hstep * p)
        adj = dk[idx] if which == "edge" else dm[idx]
        errs.append(abs(fd - adj) / max(abs(adj), 1e-300))
    print("full-size FD agreement: max rel err %.2e, median %.2e" % (max(errs), float(np.median(errs))))
    assert max(errs) < 1e-6, sorted(errs)[-5:]
