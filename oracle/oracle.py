"""TEST INFRASTRUCTURE ONLY — ctypes access to the CPU oracle (oracle/_ref/liboracle.so).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this module. The library runs the reference's own OpenMP backend (include/trl/impl/openmp/*)
and its BlockLanczos driver (include/trl/eigensolvers/lanczos.hh), compiled in place with the
Eigen-free EVPBase restatement in oracle/shim (see oracle/Makefile).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "liboracle.so")
REF_TESTS = [os.path.join(HERE, "_ref", f"ref_test_lanczos_{t}") for t in ("convergence", "extend")]

# op codes of oracle_block_view_op (reference BlockView methods)
OP_DOT, OP_MULT, OP_MULT_T, OP_MULT_ADD, OP_SUB_PROD, OP_SUB, OP_COPY, OP_ZERO = range(8)

_lib = None


def reference_root() -> str:
    """The reference checkout: $TRL_REFERENCE, else the default mount point."""
    return os.environ.get("TRL_REFERENCE", "/root/reference")


def build(ref: str | None = None) -> None:
    """Compile oracle/_ref from the reference sources (needs the reference checkout)."""
    subprocess.run(["make", "-C", HERE, f"REF={ref or reference_root()}", "-j4"], check=True, stdout=subprocess.DEVNULL)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_solve_csr.argtypes = [C.c_int, C.c_int64, P, P, P, C.c_double, C.c_double, C.c_uint, C.c_uint, C.c_uint, C.c_double, P, P, P, P, P, P]
        L.oracle_block_view_op.argtypes = [C.c_int, C.c_int, C.c_int64, P, P, P]
        L.oracle_solve_csr_minner.argtypes = [C.c_int, C.c_int64, P, P, P, P, P, P, C.c_uint, C.c_uint, C.c_uint, C.c_double, P, P, P, P]
        L.oracle_orthonormalize.argtypes = [C.c_int, C.c_int64, P, P]
        L.oracle_solve_small_dense.argtypes = [C.c_int, C.c_uint, P, P, C.c_uint, C.c_double, P, P, P]
        L.oracle_spmm.argtypes = [C.c_int, C.c_int64, P, P, P, C.c_double, C.c_double, P, P]
        L.oracle_symmetric_eigen.argtypes = [C.c_int64, P, P, P]
        L.oracle_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def solve_csr(A, bs: int, nev: int, ncv: int, X0: np.ndarray, tol: float = 1e-8, max_restarts: int = 1000,
              alpha: float = 1.0, beta: float = 0.0, ritz: bool = False) -> dict:
    """Run the reference BlockLanczos (default ModifiedGS) on Y = alpha*A*X + beta*X.
    ``cycle_seconds`` holds the duration of each restart cycle (cycle 1 includes the initial
    orthonormalisation)."""
    n = A.n
    X0 = np.ascontiguousarray(X0, dtype=np.float64).reshape(n, bs)
    evals = np.zeros(ncv)
    ritz_vecs = np.zeros((n, nev)) if ritz else None
    stats = np.zeros(3, dtype=np.int32)
    secs = np.zeros(1)
    cycles = np.zeros(max(1, max_restarts))
    rp = np.ascontiguousarray(A.rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(A.colind, dtype=np.int32)
    va = np.ascontiguousarray(A.values, dtype=np.float64)
    _check(lib().oracle_solve_csr(bs, n, _p(rp), _p(ci), _p(va), alpha, beta, nev, ncv, max_restarts, tol, _p(X0),
                                  _p(evals), _p(ritz_vecs), _p(stats), _p(secs), _p(cycles)))
    return {"converged": bool(stats[0]), "iterations": int(stats[1]), "n_op_apply": int(stats[2]),
            "seconds": float(secs[0]), "evals": evals, "ritz": ritz_vecs, "cycle_seconds": cycles[: int(stats[1])].copy()}


def solve_csr_minner(A, M, bs: int, nev: int, ncv: int, X0: np.ndarray, tol: float = 1e-10, max_restarts: int = 1000) -> dict:
    """The reference BlockLanczos (ModifiedGS) on the operator A with dot = V^T (M W) and
    CholQR in that inner product (the reference's generalised example's inner product,
    examples/openmp/csrevp.hh:89-97). Returns eigenvalues and M-orthonormal Ritz vectors."""
    n = A.n
    X0 = np.ascontiguousarray(X0, dtype=np.float64).reshape(n, bs)
    evals = np.zeros(ncv)
    ritz = np.zeros((n, nev))
    stats = np.zeros(3, dtype=np.int32)
    arrs = [np.ascontiguousarray(a, dtype=t) for a, t in ((A.rowptr, np.int32), (A.colind, np.int32), (A.values, np.float64),
                                                         (M.rowptr, np.int32), (M.colind, np.int32), (M.values, np.float64))]
    _check(lib().oracle_solve_csr_minner(bs, n, *[_p(a) for a in arrs], nev, ncv, max_restarts, tol, _p(X0), _p(evals), _p(ritz), _p(stats)))
    return {"converged": bool(stats[0]), "iterations": int(stats[1]), "n_op_apply": int(stats[2]), "evals": evals, "ritz": ritz}


def block_view_op(bs: int, op: int, X: np.ndarray, Y: np.ndarray, W: np.ndarray) -> None:
    n = X.shape[0]
    _check(lib().oracle_block_view_op(bs, op, n, _p(X), _p(Y), _p(W)))


def orthonormalize(V: np.ndarray) -> np.ndarray:
    n, bs = V.shape
    R = np.zeros((bs, bs))
    _check(lib().oracle_orthonormalize(bs, n, _p(V), _p(R)))
    return R


def solve_small_dense(T: np.ndarray, beta: np.ndarray, bs: int, nev: int, tol: float):
    """T in BlockMatrix layout [nblk][nblk][bs][bs]; returns (evals, evecs-in-block-layout, nconv)."""
    nblk = T.shape[0]
    T = np.ascontiguousarray(T, dtype=np.float64)
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    evals = np.zeros(nblk * bs)
    evecs = np.zeros_like(T)
    nconv = np.zeros(1, dtype=np.int32)
    _check(lib().oracle_solve_small_dense(bs, nblk, _p(T), _p(beta), nev, tol, _p(evals), _p(evecs), _p(nconv)))
    return evals, evecs, int(nconv[0])


def spmm(A, X: np.ndarray, alpha: float = 1.0, beta: float = 0.0) -> np.ndarray:
    n, bs = X.shape
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.zeros_like(X)
    rp = np.ascontiguousarray(A.rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(A.colind, dtype=np.int32)
    va = np.ascontiguousarray(A.values, dtype=np.float64)
    _check(lib().oracle_spmm(bs, n, _p(rp), _p(ci), _p(va), alpha, beta, _p(X), _p(Y)))
    return Y


def symmetric_eigen(A: np.ndarray):
    n = A.shape[0]
    A = np.ascontiguousarray(A, dtype=np.float64)
    w = np.zeros(n)
    V = np.zeros((n, n))
    _check(lib().oracle_symmetric_eigen(n, _p(A), _p(w), _p(V)))
    return w, V


def read_mtx(path: str):
    """Restatement of the reference's Matrix Market loader (examples/sycl/csrevp.hh:26-124),
    in plain Python for small files: header "symmetric" (any case) mirrors each off-diagonal
    entry right after it (:70-76), 1-based indices (:66-67), row counts and prefix sum
    (:93-98), then a scatter in reading order (:101-107). Returns (n_rows, n_cols, rowptr,
    colind, values). Extension read the same way as the library does: "pattern" files take
    value 1."""
    symmetric = pattern = False
    with open(path) as f:
        lines = f.read().split("\n")
    i = 0
    while i < len(lines):
        s = lines[i].strip()
        if not s:
            i += 1
            continue
        if s.startswith("%"):
            low = s.lower()
            if low.startswith("%%matrixmarket"):
                symmetric = "symmetric" in low
                pattern = "pattern" in low
            i += 1
            continue
        break
    rows, cols, entries = (int(t) for t in lines[i].split()[:3])
    toks = [t for ln in lines[i + 1:] if not ln.strip().startswith("%") for t in ln.split()]
    per = 2 if pattern else 3
    coo = []
    for e in range(entries):
        r, c = int(toks[per * e]) - 1, int(toks[per * e + 1]) - 1
        v = 1.0 if pattern else float(toks[per * e + 2])
        coo.append((r, c, v))
        if symmetric and r != c:
            coo.append((c, r, v))
    rowptr = np.zeros(rows + 1, dtype=np.int32)
    for r, _, _ in coo:
        rowptr[r + 1] += 1
    rowptr = np.cumsum(rowptr).astype(np.int32)
    pos = rowptr[:-1].copy()
    colind = np.zeros(len(coo), dtype=np.int32)
    values = np.zeros(len(coo))
    for r, c, v in coo:
        colind[pos[r]] = c
        values[pos[r]] = v
        pos[r] += 1
    return rows, cols, rowptr, colind, values
