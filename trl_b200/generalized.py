"""Generalised eigenproblems K x = lambda M x with a lumped (diagonal) mass M, and the
adjoint of weighted eigenvalue sums with respect to edge conductivities and masses.

With M diagonal the problem is transformed in place of a shift-invert:
A_hat = M^{-1/2} K M^{-1/2} (same CSR pattern, scaled values), y = M^{1/2} x, and the
smallest eigenvalues of A_hat are the largest-magnitude eigenvalues of sigma*I - A_hat with
sigma = ||A_hat||_1 (Gershgorin), which the driver's |theta|-descending order
(evp_base.hh:103) selects. lambda = sigma - theta and x = M^{-1/2} y is M-normalised
(x^T M x = y^T y = 1). The reference's generalised example instead factors K - s M with a
sparse LU (examples/openmp/csrevp.hh:59-87), which has no GPU counterpart here.

Gradients (for M-normalised x):  d lambda / dK_ij = x_i x_j,  d lambda / dM_ij = -lambda x_i x_j.
For K = sum_e kappa_e (e_a - e_b)(e_a - e_b)^T (e_{-1} = 0 for a boundary edge) and
M = diag(m):  d lambda / d kappa_e = (x_a - x_b)^2,  d lambda / d m_i = -lambda x_i^2.
Both are evaluated through the SDDMM of the C ABI (trl_cuda_eigen_adjoint) over the CSR
patterns of K and of diag(M), then gathered per edge.
"""
from __future__ import annotations

import numpy as np

from . import native
from .problems import CSRMatrix, scale_symmetric


def diagonal_pattern(n: int) -> CSRMatrix:
    i = np.arange(n, dtype=np.int32)
    return CSRMatrix(n, np.arange(n + 1, dtype=np.int32), i, np.ones(n))


def edge_entry_index(K: CSRMatrix, a: np.ndarray, b: np.ndarray):
    """Positions in K's CSR arrays of the entries (a,a), (b,b), (a,b), (b,a) of every edge
    (-1 where b is the exterior)."""
    def pos(r, c):
        start = K.rowptr[r].astype(np.int64)
        end = K.rowptr[r + 1].astype(np.int64)
        out = np.empty(r.size, dtype=np.int64)
        # rows are sorted: search per row (vectorised over a loop of small widths)
        width = int((end - start).max()) if r.size else 0
        found = np.full(r.size, -1, dtype=np.int64)
        for o in range(width):
            p = start + o
            ok = (p < end) & (found < 0)
            hit = ok & (K.colind[np.minimum(p, K.nnz - 1)] == c)
            found[hit] = p[hit]
        out[:] = found
        return out

    inner = b >= 0
    bb = np.where(inner, b, a)
    paa = pos(a, a)
    pbb = np.where(inner, pos(bb, bb), -1)
    pab = np.where(inner, pos(a, bb), -1)
    pba = np.where(inner, pos(bb, a), -1)
    return paa, pbb, pab, pba


def solve_smallest(handle: native.Handle, K: CSRMatrix, mass: np.ndarray, nev: int, bs: int, ncv: int, X0: np.ndarray, tol: float = 1e-10,
                   max_restarts: int = 10000, mode: int = native.TRL_MODE_FP64, **kw):
    """Smallest nev eigenpairs of K x = lambda M x (M = diag(mass)) on the GPU.
    Returns (lam ascending, X device tensor n x nev M-normalised, info dict)."""
    import torch

    dinv = 1.0 / np.sqrt(mass)
    Ah = scale_symmetric(K, dinv)
    sigma = Ah.gershgorin_bound()
    A64 = native.DeviceCSRTensors.from_host(Ah, torch.float64)
    A32 = native.DeviceCSRTensors.from_host(Ah, torch.float32) if mode != native.TRL_MODE_FP64 else None
    X0d = torch.from_numpy(np.ascontiguousarray(X0, dtype=np.float64)).cuda()
    Y = torch.empty((K.n, nev), dtype=torch.float64, device="cuda")
    out = native.solve_csr_device(handle, A64, A32, X0d, evecs=Y, bs=bs, nev=nev, ncv=ncv, tol=tol, alpha=-1.0, beta=sigma,
                                  max_restarts=max_restarts, refine_max_restarts=max_restarts, mode=mode, **kw)
    lam = sigma - out["evals"]
    X = Y * torch.from_numpy(dinv).cuda()[:, None]
    out["sigma"] = sigma
    return lam, X, out


def eigen_sum_gradient(handle: native.Handle, K: CSRMatrix, n_mass: int, edges: dict, X, lam: np.ndarray, weights: np.ndarray,
                       cluster_rtol: float = 1e-8, K_dev=None, D_dev=None, index=None):
    """Gradient of f = sum_c w_c lambda_c with respect to the edge conductivities and the
    masses, from M-normalised eigenvectors X (device, n x k). Returns (d_kappa, d_mass)."""
    import torch

    Kd = K_dev or native.DeviceCSRTensors.from_host(K)
    Dd = D_dev or native.DeviceCSRTensors.from_host(diagonal_pattern(n_mass))
    gK = torch.empty(K.nnz, dtype=torch.float64, device="cuda")
    gM = torch.empty(n_mass, dtype=torch.float64, device="cuda")
    Xc = X.contiguous()
    handle.eigen_adjoint(Kd, Xc, lam, weights, gK, kind=0, cluster_rtol=cluster_rtol)
    handle.eigen_adjoint(Dd, Xc, lam, weights, gM, kind=1, cluster_rtol=cluster_rtol)
    torch.cuda.synchronize()
    gK = gK.cpu().numpy()
    paa, pbb, pab, pba = index if index is not None else edge_entry_index(K, edges["a"], edges["b"])
    inner = edges["b"] >= 0
    dk = gK[paa].copy()
    dk[inner] += gK[pbb[inner]] - gK[pab[inner]] - gK[pba[inner]]
    return dk, gM.cpu().numpy()
