"""Seeded synthetic sparse operators for the block-Lanczos hot path.

The reference ships no matrices of its own (its ``data/*.mtx`` are git-LFS pointers), and
its example drivers load MatrixMarket files into full-storage CSR with int32 indices and
FP64 values (``examples/sycl/csrevp.hh:16-23,26-124``). Every generator here returns that
layout: ``rowptr`` int32[n+1], ``colind`` int32[nnz] sorted within each row, ``values``
float64[nnz], with both triangles stored.

Workloads (sizes as named by the benchmark configurations):

* ``laplace2d``      2-D 5-point Dirichlet Laplacian, stencil 4/-1 (128x128: n=16,384).
* ``anisotropic3d``  3-D 7-point Dirichlet Laplacian with axis coefficients (cx, cy, cz)
                     (96^3 with (1,10,100): n=884,736, nnz=6,137,856).
* ``elasticity27``   3 dofs per node on an m^3 node grid with 27-point node coupling,
                     off-diagonal 3x3 blocks N(0,1) x log-uniform[1e-3,1] scale, diagonal
                     1.05 x the row's absolute off-diagonal sum (64^3: n=786,432).
* ``diffusion2d_mass`` generalised K x = lambda M x on an m x m grid: K a 5-point diffusion
                     operator with log-normal(0, sigma) edge conductivities (Dirichlet
                     boundary edges included), M a lumped diagonal mass U[0.5, 1.5].
* ``zipf_symmetric`` n x n random symmetric pattern, truncated Zipf(alpha) out-degrees
                     capped at ``cap``, uniform random columns, N(0,1) values mirrored.
* ``diagonal`` / ``laplace1d`` — the reference's own test operators
  (``tests/openmp/diagonal.hh:19``, ``tests/openmp/laplace.hh:19-31``) as CSR.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class CSRMatrix:
    n: int
    rowptr: np.ndarray  # int32[n+1]
    colind: np.ndarray  # int32[nnz]
    values: np.ndarray  # float64[nnz]
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.colind.shape[0])

    def to_dense(self) -> np.ndarray:
        a = np.zeros((self.n, self.n))
        rows = np.repeat(np.arange(self.n), np.diff(self.rowptr))
        np.add.at(a, (rows, self.colind), self.values)
        return a

    def row_indices(self) -> np.ndarray:
        return np.repeat(np.arange(self.n, dtype=np.int32), np.diff(self.rowptr))

    def matmat(self, x: np.ndarray) -> np.ndarray:
        """Y = A X for X of shape (n, b) in FP64 (host reference for checks)."""
        rows = self.row_indices()
        y = np.zeros((self.n,) + x.shape[1:], dtype=np.float64)
        np.add.at(y, rows, self.values[:, None] * x[self.colind] if x.ndim == 2 else self.values * x[self.colind])
        return y

    def gershgorin_bound(self) -> float:
        """max_i sum_j |a_ij| (an upper bound on |lambda|; also ||A||_inf = ||A||_1)."""
        rows = self.row_indices()
        s = np.zeros(self.n)
        np.add.at(s, rows, np.abs(self.values))
        return float(s.max()) if self.n else 0.0


def _from_coo(n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray, **meta) -> CSRMatrix:
    order = np.lexsort((cols, rows))
    rows = rows[order]
    cols = cols[order].astype(np.int32)
    vals = vals[order].astype(np.float64)
    counts = np.bincount(rows, minlength=n)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    if rowptr[-1] >= 2**31:
        raise ValueError("nnz exceeds the int32 index range of the CSR layout")
    return CSRMatrix(n, rowptr.astype(np.int32), cols, vals, dict(meta))


def _stencil(shape: tuple[int, ...], offsets: list[tuple[int, ...]], weights: list[float]) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """COO of a constant-coefficient stencil with Dirichlet truncation.

    Grid index: i = x0 + s0 * (x1 + s1 * (x2 ...)), i.e. the first axis is fastest.
    """
    n = int(np.prod(shape))
    coords = np.unravel_index(np.arange(n), shape[::-1])[::-1]  # x0 fastest
    rows_l, cols_l, vals_l = [], [], []
    strides = np.cumprod((1,) + tuple(shape[:-1]))
    idx = np.arange(n, dtype=np.int64)
    for off, w in zip(offsets, weights):
        ok = np.ones(n, dtype=bool)
        delta = 0
        for ax, o in enumerate(off):
            if o:
                c = coords[ax] + o
                ok &= (c >= 0) & (c < shape[ax])
                delta += o * int(strides[ax])
        rows_l.append(idx[ok])
        cols_l.append(idx[ok] + delta)
        vals_l.append(np.full(int(ok.sum()), w))
    return np.concatenate(rows_l), np.concatenate(cols_l), np.concatenate(vals_l)


def laplace2d(nx: int = 128, ny: int | None = None) -> CSRMatrix:
    ny = nx if ny is None else ny
    offs = [(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)]
    w = [4.0, -1.0, -1.0, -1.0, -1.0]
    r, c, v = _stencil((nx, ny), offs, w)
    return _from_coo(nx * ny, r, c, v, kind="laplace2d", grid=(nx, ny))


def laplace2d_eigenvalues(nx: int = 128, ny: int | None = None) -> np.ndarray:
    """All eigenvalues 4 - 2cos(p pi/(nx+1)) - 2cos(q pi/(ny+1)), descending."""
    ny = nx if ny is None else ny
    p = np.arange(1, nx + 1)
    q = np.arange(1, ny + 1)
    lam = (2 - 2 * np.cos(p * np.pi / (nx + 1)))[:, None] + (2 - 2 * np.cos(q * np.pi / (ny + 1)))[None, :]
    return np.sort(lam.ravel())[::-1]


def anisotropic3d(nx: int = 96, ny: int | None = None, nz: int | None = None, coef=(1.0, 10.0, 100.0)) -> CSRMatrix:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    cx, cy, cz = (float(c) for c in coef)
    offs = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    w = [2.0 * (cx + cy + cz), -cx, -cx, -cy, -cy, -cz, -cz]
    r, c, v = _stencil((nx, ny, nz), offs, w)
    return _from_coo(nx * ny * nz, r, c, v, kind="anisotropic3d", grid=(nx, ny, nz), coef=(cx, cy, cz))


def anisotropic3d_eigenvalues(nx: int = 96, ny: int | None = None, nz: int | None = None, coef=(1.0, 10.0, 100.0), k: int | None = None) -> np.ndarray:
    """Largest ``k`` (all if None) eigenvalues sum_d c_d (2 - 2cos(p_d pi/(n_d+1))), descending."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    ex = coef[0] * (2 - 2 * np.cos(np.arange(1, nx + 1) * np.pi / (nx + 1)))
    ey = coef[1] * (2 - 2 * np.cos(np.arange(1, ny + 1) * np.pi / (ny + 1)))
    ez = coef[2] * (2 - 2 * np.cos(np.arange(1, nz + 1) * np.pi / (nz + 1)))
    lam = (ex[:, None, None] + ey[None, :, None] + ez[None, None, :]).ravel()
    if k is None:
        return np.sort(lam)[::-1]
    part = np.partition(lam, lam.size - k)[lam.size - k:]
    return np.sort(part)[::-1]


def laplace1d(n: int) -> CSRMatrix:
    r, c, v = _stencil((n,), [(0,), (1,), (-1,)], [2.0, -1.0, -1.0])
    return _from_coo(n, r, c, v, kind="laplace1d")


def diagonal(n: int) -> CSRMatrix:
    i = np.arange(n, dtype=np.int64)
    return _from_coo(n, i, i, ((i + 1) ** 2).astype(np.float64), kind="diagonal")


def elasticity27(m: int = 64, seed: int = 42, dominance: float = 1.05) -> CSRMatrix:
    """3 dofs per node, 27-point node coupling on an m^3 node grid (boundary-trimmed).

    Each coupled node pair (p < q) gets a 3x3 block B = N(0,1) * s, s log-uniform in
    [1e-3, 1]; the pair contributes B at (p, q) and B^T at (q, p). Each node's own 3x3
    block gets symmetric off-diagonal entries drawn the same way. Finally every diagonal
    entry is set to ``dominance`` times the absolute off-diagonal sum of its row.
    """
    rng = np.random.default_rng(seed)
    nn = m ** 3
    coords = np.stack(np.unravel_index(np.arange(nn), (m, m, m))[::-1], axis=1)  # x fastest
    # forward half of the 26 neighbour offsets (lexicographically positive)
    fwd = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if (dz, dy, dx) > (0, 0, 0)]
    rows_l, cols_l, vals_l = [], [], []
    node = np.arange(nn, dtype=np.int64)
    for dx, dy, dz in fwd:
        c = coords + np.array([dx, dy, dz])
        ok = np.all((c >= 0) & (c < m), axis=1)
        p = node[ok]
        q = p + dx + m * (dy + m * dz)
        npair = p.size
        scale = 10.0 ** rng.uniform(-3.0, 0.0, size=npair)
        blk = rng.standard_normal((npair, 3, 3)) * scale[:, None, None]
        a = np.arange(3)
        for ia in range(3):
            for ib in range(3):
                rows_l.append(3 * p + ia)
                cols_l.append(3 * q + ib)
                vals_l.append(blk[:, ia, ib])
                rows_l.append(3 * q + ib)
                cols_l.append(3 * p + ia)
                vals_l.append(blk[:, ia, ib])
        del a
    # intra-node symmetric off-diagonals
    scale = 10.0 ** rng.uniform(-3.0, 0.0, size=nn)
    for ia, ib in ((0, 1), (0, 2), (1, 2)):
        v = rng.standard_normal(nn) * scale
        rows_l += [3 * node + ia, 3 * node + ib]
        cols_l += [3 * node + ib, 3 * node + ia]
        vals_l += [v, v]
    rows = np.concatenate(rows_l)
    cols = np.concatenate(cols_l)
    vals = np.concatenate(vals_l)
    n = 3 * nn
    offsum = np.zeros(n)
    np.add.at(offsum, rows, np.abs(vals))
    d = np.arange(n, dtype=np.int64)
    rows = np.concatenate([rows, d])
    cols = np.concatenate([cols, d])
    vals = np.concatenate([vals, dominance * offsum])
    return _from_coo(n, rows, cols, vals, kind="elasticity27", grid=(m, m, m), seed=seed)


def diffusion2d_mass(m: int = 512, sigma: float = 1.0, seed: int = 42):
    """Generalised problem K x = lambda M x on an m x m grid (Dirichlet boundary edges).

    Returns (K, mass, edges) where ``edges`` is a dict with int64 arrays ``a``, ``b`` (b=-1
    for a boundary edge to the fixed exterior) and float64 ``kappa``; K = sum_e kappa_e
    (e_a - e_b)(e_a - e_b)^T with e_{-1} = 0, and ``mass`` is the lumped diagonal of M.
    """
    rng = np.random.default_rng(seed)
    n = m * m
    idx = np.arange(n, dtype=np.int64).reshape(m, m)  # [y, x], x fastest
    a_l, b_l = [], []
    # interior horizontal / vertical edges
    a_l.append(idx[:, :-1].ravel()); b_l.append(idx[:, 1:].ravel())
    a_l.append(idx[:-1, :].ravel()); b_l.append(idx[1:, :].ravel())
    # boundary edges to the exterior (one per boundary face of a node)
    for sl in (idx[:, 0], idx[:, -1], idx[0, :], idx[-1, :]):
        a_l.append(sl.ravel()); b_l.append(np.full(sl.size, -1, dtype=np.int64))
    a = np.concatenate(a_l)
    b = np.concatenate(b_l)
    kappa = rng.lognormal(mean=0.0, sigma=sigma, size=a.size)
    mass = rng.uniform(0.5, 1.5, size=n)
    K = assemble_diffusion(n, a, b, kappa)
    return K, mass, {"a": a, "b": b, "kappa": kappa}


def assemble_diffusion(n: int, a: np.ndarray, b: np.ndarray, kappa: np.ndarray) -> CSRMatrix:
    inner = b >= 0
    diag = np.zeros(n)
    np.add.at(diag, a, kappa)
    np.add.at(diag, b[inner], kappa[inner])
    ai, bi, ki = a[inner], b[inner], kappa[inner]
    d = np.arange(n, dtype=np.int64)
    rows = np.concatenate([d, ai, bi])
    cols = np.concatenate([d, bi, ai])
    vals = np.concatenate([diag, -ki, -ki])
    return _from_coo(n, rows, cols, vals, kind="diffusion2d")


def scale_symmetric(A: CSRMatrix, dinv_sqrt: np.ndarray) -> CSRMatrix:
    """D^{-1/2} A D^{-1/2} for a positive diagonal D given as d^{-1/2}."""
    rows = A.row_indices()
    vals = A.values * dinv_sqrt[rows] * dinv_sqrt[A.colind]
    return CSRMatrix(A.n, A.rowptr, A.colind, vals, dict(A.meta, scaled=True))


def zipf_symmetric(n: int = 4_194_304, alpha: float = 1.5, cap: int = 512, seed: int = 42) -> CSRMatrix:
    """Random symmetric pattern: out-degree of row i drawn from Zipf(alpha) truncated to
    [1, cap] (values above ``cap`` are redrawn), columns uniform in [0, n), values N(0,1).
    Edges are made symmetric by mirroring and de-duplicated per unordered pair (the first
    draw of a pair keeps its value); self-pairs become diagonal entries.
    """
    rng = np.random.default_rng(seed)
    deg = rng.zipf(alpha, size=n)
    bad = deg > cap
    while bad.any():
        deg[bad] = rng.zipf(alpha, size=int(bad.sum()))
        bad = deg > cap
    rows = np.repeat(np.arange(n, dtype=np.int64), deg)
    cols = rng.integers(0, n, size=rows.size, dtype=np.int64)
    vals = rng.standard_normal(rows.size)
    lo = np.minimum(rows, cols)
    hi = np.maximum(rows, cols)
    key = lo * n + hi
    del lo, hi
    _, first = np.unique(key, return_index=True)
    del key
    rows, cols, vals = rows[first], cols[first], vals[first]
    off = rows != cols
    rows2 = np.concatenate([rows, cols[off]])
    cols2 = np.concatenate([cols, rows[off]])
    vals2 = np.concatenate([vals, vals[off]])
    del rows, cols, vals
    A = _from_coo(n, rows2, cols2, vals2, kind="zipf_symmetric", alpha=alpha, cap=cap, seed=seed)
    A.meta["mean_degree"] = A.nnz / n
    return A


def initial_block(n: int, b: int, seed: int = 42) -> np.ndarray:
    """Seeded N(0,1) starting block of shape (n, b), row-major (the reference fills
    ``initial_block()`` with std::mt19937(42) + normal_distribution, examples/openmp/csrtest.cc:94-96;
    the same values need not be reproduced — both backends receive this same array)."""
    return np.random.default_rng(seed).standard_normal((n, b))


def diffusion2d_consistent_mass(m: int = 12, seed: int = 42, coupling: float = 0.05):
    """K x = lambda M x on an m x m grid with a non-diagonal SPD mass: K as in
    ``diffusion2d_mass``, M = diag(U[0.5, 1.5]) plus ``coupling`` between grid neighbours
    (diagonally dominant for coupling < 1/8, hence SPD). Returns (K, M) as CSR."""
    K, mass, edges = diffusion2d_mass(m, seed=seed)
    a, b = edges["a"], edges["b"]
    inner = b >= 0
    n = m * m
    d = np.arange(n, dtype=np.int64)
    rows = np.concatenate([d, a[inner], b[inner]])
    cols = np.concatenate([d, b[inner], a[inner]])
    vals = np.concatenate([mass, np.full(int(inner.sum()), coupling), np.full(int(inner.sum()), coupling)])
    return K, _from_coo(n, rows, cols, vals, kind="consistent_mass")


def dense_csr(D: np.ndarray) -> CSRMatrix:
    """A dense matrix as CSR with every entry stored."""
    n = D.shape[0]
    rows = np.repeat(np.arange(n, dtype=np.int64), n)
    cols = np.tile(np.arange(n, dtype=np.int64), n)
    return _from_coo(n, rows, cols, D.ravel(), kind="dense")
