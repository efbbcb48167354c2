"""ctypes bindings of the backend's C ABI (include/trl_cuda.h) and of the solver entry points
(include/trl_solver.h). The libraries are loaded from ``trl_b200/lib``; there is no fallback:
if they are missing the import of the bindings raises.

Kernel wrappers take torch CUDA tensors (device memory and streams come from torch; every
call is enqueued on torch's current stream through a handle bound to that stream).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
CUDA_LIB = os.path.join(LIB_DIR, "libtrl_cuda.so")
SOLVER_LIB = os.path.join(LIB_DIR, "libtrl_solver.so")
REF_TESTS_BIN = os.path.join(LIB_DIR, "trl_cuda_ref_tests")

TRL_OK, TRL_EINVAL, TRL_ENOMEM, TRL_ECUDA, TRL_ECHOLESKY, TRL_EEIGEN, TRL_ETIMEOUT, TRL_ENOTSUP = range(8)
TRL_F64, TRL_F32 = 0, 1
TRL_H2D, TRL_D2H, TRL_D2D = 0, 1, 2
TRL_MULT, TRL_MULT_TRANSPOSE, TRL_MULT_ADD, TRL_SUBTRACT, TRL_SUBTRACT_TRANSPOSE = 0, 1, 2, 3, 4
TRL_MODE_FP64, TRL_MODE_FP32, TRL_MODE_MIXED = 0, 1, 2
TRL_REORTH_MGS, TRL_REORTH_CGS2, TRL_REORTH_CGS_IFNEEDED, TRL_REORTH_CGS1, TRL_REORTH_PARTIAL = 0, 1, 2, 3, 4
TRL_CGS_ONE, TRL_CGS_TWO, TRL_CGS_IFNEEDED = 0, 1, 2
TRL_REFINE_LANCZOS, TRL_REFINE_CHEBYSHEV, TRL_REFINE_AUTO = 0, 1, 2

P = C.c_void_p
I64 = C.c_int64

# symbol -> (restype, argtypes); the full exported surface of include/trl_cuda.h
CUDA_SYMBOLS = {
    "trl_cuda_create": (C.c_int, [C.POINTER(P), C.c_int, P]),
    "trl_cuda_destroy": (C.c_int, [P]),
    "trl_cuda_synchronize": (C.c_int, [P]),
    "trl_cuda_stream": (P, [P]),
    "trl_cuda_last_error": (C.c_char_p, [P]),
    "trl_cuda_status_string": (C.c_char_p, [C.c_int]),
    "trl_cuda_launch_count": (C.c_uint64, [P]),
    "trl_cuda_inject_alloc_failures": (C.c_int, [P, C.c_int]),
    "trl_cuda_test_bounded_wait": (C.c_int, [P, C.c_uint]),
    "trl_cuda_measure_dmma_rate": (C.c_int, [P, C.POINTER(C.c_double)]),
    "trl_cuda_malloc": (C.c_int, [P, C.POINTER(P), C.c_size_t]),
    "trl_cuda_free": (C.c_int, [P, P]),
    "trl_cuda_memcpy": (C.c_int, [P, P, P, C.c_size_t, C.c_int]),
    "trl_cuda_memset_zero": (C.c_int, [P, P, C.c_size_t]),
    "trl_cuda_bv_zero": (C.c_int, [P, C.c_int, P, I64, C.c_int]),
    "trl_cuda_bv_copy": (C.c_int, [P, C.c_int, P, P, I64, C.c_int]),
    "trl_cuda_bv_sub": (C.c_int, [P, C.c_int, P, P, I64, C.c_int]),
    "trl_cuda_bv_mult": (C.c_int, [P, C.c_int, C.c_int, P, P, P, I64, C.c_int]),
    "trl_cuda_convert": (C.c_int, [P, C.c_int, P, C.c_int, P, I64]),
    "trl_cuda_unblock": (C.c_int, [P, P, I64, C.c_int, C.c_int, P]),
    "trl_cuda_block_dot": (C.c_int, [P, C.c_int, P, C.c_int, P, I64, C.c_int, P]),
    "trl_cuda_block_dot_noalloc": (C.c_int, [P, C.c_int, P, C.c_int, P, I64, C.c_int, P]),
    "trl_cuda_block_update": (C.c_int, [P, C.c_int, P, P, C.c_int, P, I64, C.c_int]),
    "trl_cuda_block_rotate": (C.c_int, [P, C.c_int, P, C.c_int, P, C.c_int, C.c_int, P, I64, C.c_int]),
    "trl_cuda_cholqr": (C.c_int, [P, C.c_int, P, I64, C.c_int, C.c_int, P]),
    "trl_cuda_cholqr_gram": (C.c_int, [P, C.c_int, P, I64, C.c_int, C.c_int, P, P]),
    "trl_cuda_project_out": (C.c_int, [P, C.c_int, P, C.c_int, P, I64, C.c_int, C.c_int, C.c_double, P]),
    "trl_cuda_project_out_sketch": (C.c_int, [P, C.c_int, P, C.c_int, P, I64, C.c_int, P, C.c_double, C.c_double, P, P]),
    "trl_cuda_spmm": (C.c_int, [P, P, C.c_int, P, P, C.c_int, C.c_double, C.c_double]),
    "trl_cuda_csr_norm1": (C.c_int, [P, P, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "trl_cuda_spmm3": (C.c_int, [P, P, C.c_int, P, P, C.c_int, C.c_double, C.c_double, C.c_double, P]),
    "trl_cuda_spmm_blocks": (C.c_int, [P, P, C.c_int, P, P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, P]),
    "trl_cuda_csr_gershgorin": (C.c_int, [P, P, C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "trl_cuda_op_create": (C.c_int, [P, P, C.c_int, C.POINTER(P)]),
    "trl_cuda_op_destroy": (C.c_int, [P, P]),
    "trl_cuda_op_info": (C.c_int, [P, C.POINTER(I64), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "trl_cuda_op_spmm": (C.c_int, [P, P, P, P, C.c_int, C.c_double, C.c_double, C.c_double, P]),
    "trl_cuda_sddmm": (C.c_int, [P, P, P, C.c_int, P, P]),
    "trl_cuda_eigen_adjoint": (C.c_int, [P, P, P, C.c_int, P, P, C.c_double, C.c_int, P]),
    "trl_cuda_mb_copy": (C.c_int, [P, P, P, C.c_int, C.c_int]),
    "trl_cuda_mb_zero": (C.c_int, [P, P, C.c_int]),
    "trl_cuda_mb_mult": (C.c_int, [P, P, P, P, C.c_int]),
    "trl_cuda_mb_set_diagonal": (C.c_int, [P, P, P, C.c_int]),
    "trl_cuda_small_eigen": (C.c_int, [P, P, C.c_int, C.c_int, P, C.c_int, C.c_double, P, P, P, C.POINTER(C.c_int)]),
    "trl_cuda_small_eigen_partial": (C.c_int, [P, P, C.c_int, C.c_int, P, C.c_int, C.c_double, C.c_int, P, P, P, C.POINTER(C.c_int)]),
    "trl_cuda_profile_enable": (C.c_int, [P, C.c_int]),
    "trl_cuda_profile_read": (C.c_int, [P, P]),
}

TRL_PROF_CLASSES = 12


class trl_kernel_stats(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("calls", C.c_uint64), ("seconds", C.c_double), ("bytes", C.c_double), ("flops", C.c_double)]


class trl_csr(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz", C.c_int64), ("rowptr", P), ("colind", P), ("values", P), ("value_dtype", C.c_int)]


class trl_solve_params(C.Structure):
    _fields_ = [("bs", C.c_int), ("mode", C.c_int), ("nev", C.c_uint), ("ncv", C.c_uint), ("max_restarts", C.c_uint),
                ("tol", C.c_double), ("alpha", C.c_double), ("beta", C.c_double), ("reorth", C.c_int),
                ("cholqr_passes", C.c_int), ("fp32_tol", C.c_double), ("refine_max_restarts", C.c_uint),
                ("want_vectors", C.c_int), ("batching", C.c_int), ("seed", C.c_uint), ("refine", C.c_int),
                ("fp32_ncv", C.c_uint), ("refine_fp32", C.c_int), ("small_eigen_full", C.c_int), ("partial_threshold", C.c_double),
                ("partial_pairs", C.c_int)]


class trl_solve_info(C.Structure):
    _fields_ = [("converged", C.c_int), ("restarts", C.c_uint), ("n_op_apply", C.c_uint), ("restarts_fp32", C.c_uint),
                ("n_op_apply_fp32", C.c_uint), ("seconds", C.c_double), ("seconds_fp32", C.c_double),
                ("seconds_vectors", C.c_double), ("max_rel_residual", C.c_double), ("max_theta_residual", C.c_double),
                ("op_norm1", C.c_double), ("kernel_launches", C.c_ulonglong), ("h2d_bytes", C.c_double), ("d2h_bytes", C.c_double),
                ("refine_rounds", C.c_uint), ("refine_degree", C.c_uint),
                ("refine_degree_fp32", C.c_uint), ("refine_used", C.c_int), ("refine_predicted_s", C.c_double),
                ("refine_lanczos_estimate_s", C.c_double)]


SOLVER_SYMBOLS = {
    "trl_solve_params_default": (None, [C.POINTER(trl_solve_params)]),
    "trl_solve_csr_host": (C.c_int, [C.POINTER(trl_solve_params), C.c_int, I64, I64, P, P, P, P, P, P, P, C.POINTER(trl_solve_info)]),
    "trl_solve_csr_device": (C.c_int, [P, C.POINTER(trl_solve_params), P, P, P, P, P, P, C.POINTER(trl_solve_info)]),
    "trl_solve_csr_minner_device": (C.c_int, [P, C.POINTER(trl_solve_params), P, P, P, P, P, P, C.POINTER(trl_solve_info)]),
    "trl_solver_last_error": (C.c_char_p, []),
    "trl_csr_read_mtx": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(C.POINTER(C.c_int32)),
                                   C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_double))]),
    "trl_csr_free_host": (None, [P, P, P]),
}

_cuda = None
_solver = None


def _load(path: str, symbols: dict):
    if not os.path.exists(path):
        raise RuntimeError(f"trl_b200 native library missing: {path} — run trl_b200.build (no CPU fallback exists)")
    lib = C.CDLL(path, mode=C.RTLD_GLOBAL)
    for name, (res, args) in symbols.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def cuda_lib():
    global _cuda
    if _cuda is None:
        _cuda = _load(CUDA_LIB, CUDA_SYMBOLS)
    return _cuda


def solver_lib():
    global _solver
    if _solver is None:
        cuda_lib()
        _solver = _load(SOLVER_LIB, SOLVER_SYMBOLS)
    return _solver


class TrlError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def _ptr(t) -> int | None:
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def _dtype(t) -> int:
    import torch

    if t.dtype == torch.float64:
        return TRL_F64
    if t.dtype == torch.float32:
        return TRL_F32
    raise TypeError(f"unsupported dtype {t.dtype}")


class Handle:
    """A C-ABI handle bound to a torch CUDA stream (the current one by default)."""

    def __init__(self, device: int = 0, stream=None):
        import torch

        self.lib = cuda_lib()
        s = stream if stream is not None else torch.cuda.current_stream(device)
        self.stream = s
        h = P()
        # torch's default stream is the legacy stream (handle 0): pass cudaStreamLegacy (1),
        # since NULL asks the ABI for a private stream
        st = self.lib.trl_cuda_create(C.byref(h), device, C.c_void_p(s.cuda_stream or 1))
        if st != TRL_OK:
            raise TrlError(st, self.lib.trl_cuda_status_string(st).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.trl_cuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, st: int):
        if st != TRL_OK:
            raise TrlError(st, self.lib.trl_cuda_last_error(self.h).decode())

    def sync(self):
        self.check(self.lib.trl_cuda_synchronize(self.h))

    def launches(self) -> int:
        return int(self.lib.trl_cuda_launch_count(self.h))

    def profile(self, on: bool) -> None:
        self.check(self.lib.trl_cuda_profile_enable(self.h, int(on)))

    def profile_read(self) -> dict:
        """Per-kernel-class totals: {name: {calls, seconds, bytes, flops}} (synchronises)."""
        arr = (trl_kernel_stats * TRL_PROF_CLASSES)()
        self.check(self.lib.trl_cuda_profile_read(self.h, C.cast(arr, P)))
        return {a.name.decode(): {"calls": int(a.calls), "seconds": a.seconds, "bytes": a.bytes, "flops": a.flops} for a in arr}

    # ---- block-vector kernels (X: torch tensor of shape (n, bs) or (nblk, n, bs)) -----
    def bv_sub(self, X, Y):
        n, bs = X.shape[-2], X.shape[-1]
        self.check(self.lib.trl_cuda_bv_sub(self.h, _dtype(X), _ptr(X), _ptr(Y), n, bs))

    def bv_mult(self, mode: int, X, W, Y):
        n, bs = X.shape[-2], X.shape[-1]
        self.check(self.lib.trl_cuda_bv_mult(self.h, _dtype(X), mode, _ptr(X), _ptr(W), _ptr(Y), n, bs))

    def block_dot(self, V, W, C_out):
        nblk, n, bs = V.shape
        self.check(self.lib.trl_cuda_block_dot(self.h, _dtype(V), _ptr(V), nblk, _ptr(W), n, bs, _ptr(C_out)))

    def block_update(self, W, V, Cm):
        nblk, n, bs = V.shape
        self.check(self.lib.trl_cuda_block_update(self.h, _dtype(V), _ptr(W), _ptr(V), nblk, _ptr(Cm), n, bs))

    def block_rotate(self, V, Y, k: int, W):
        """W[j] = sum_i V[i] Y(i, j) for j < k; Y is a block matrix of shape (m, ldy, bs, bs)."""
        m, n, bs = V.shape
        ldy = Y.shape[1]
        self.check(self.lib.trl_cuda_block_rotate(self.h, _dtype(V), _ptr(V), m, _ptr(Y), ldy, k, _ptr(W), n, bs))

    def cholqr(self, X, passes: int, R):
        n, bs = X.shape
        self.check(self.lib.trl_cuda_cholqr(self.h, _dtype(X), _ptr(X), n, bs, passes, _ptr(R)))

    def project_out(self, V, W, mode: int, G, eta: float = 0.7071067811865476):
        nblk, n, bs = V.shape
        self.check(self.lib.trl_cuda_project_out(self.h, _dtype(V), _ptr(V), nblk, _ptr(W), n, bs, mode, eta, _ptr(G)))

    def project_out_sketch(self, V, W, S, thr: float, G, eta: float = 0.7071067811865476, pair_state=None):
        """pair_state: optional int32 CUDA tensor (one element, zeroed) kept across the steps
        of one recurrence; a step whose sketch test fired then also projects the next."""
        nblk, n, bs = V.shape
        self.check(self.lib.trl_cuda_project_out_sketch(self.h, _dtype(V), _ptr(V), nblk, _ptr(W), n, bs, _ptr(S), thr, eta, _ptr(G), _ptr(pair_state)))

    def cholqr_gram(self, X, passes: int, R, G0):
        n, bs = X.shape
        self.check(self.lib.trl_cuda_cholqr_gram(self.h, _dtype(X), _ptr(X), n, bs, passes, _ptr(R), _ptr(G0)))

    def convert(self, dst, src):
        self.check(self.lib.trl_cuda_convert(self.h, _dtype(dst), _ptr(dst), _dtype(src), _ptr(src), src.numel()))

    def spmm(self, A: "DeviceCSRTensors", X, Y, alpha: float = 1.0, beta: float = 0.0):
        n, bs = X.shape
        self.check(self.lib.trl_cuda_spmm(self.h, C.byref(A.desc), _dtype(X), _ptr(X), _ptr(Y), bs, alpha, beta))

    def spmm3(self, A: "DeviceCSRTensors", X, Y, alpha: float, beta: float, gamma: float, W):
        n, bs = X.shape
        self.check(self.lib.trl_cuda_spmm3(self.h, C.byref(A.desc), _dtype(X), _ptr(X), _ptr(Y), bs, alpha, beta, gamma, _ptr(W)))

    def spmm_blocks(self, A: "DeviceCSRTensors", X, Y, alpha: float, beta: float, gamma: float, W):
        nb, n, bs = X.shape
        self.check(self.lib.trl_cuda_spmm_blocks(self.h, C.byref(A.desc), _dtype(X), _ptr(X), _ptr(Y), bs, nb, alpha, beta, gamma, _ptr(W)))

    def prepare(self, A: "DeviceCSRTensors", bs: int) -> "PreparedOp":
        """The operator converted for repeated SpMMs with block size bs (trl_cuda_op_create)."""
        op = P()
        self.check(self.lib.trl_cuda_op_create(self.h, C.byref(A.desc), bs, C.byref(op)))
        return PreparedOp(self, op, A.desc.value_dtype, bs)

    def csr_gershgorin(self, A: "DeviceCSRTensors", alpha: float = 1.0, beta: float = 0.0):
        lo, hi = C.c_double(0.0), C.c_double(0.0)
        self.check(self.lib.trl_cuda_csr_gershgorin(self.h, C.byref(A.desc), alpha, beta, C.byref(lo), C.byref(hi)))
        return lo.value, hi.value

    def csr_norm1(self, A: "DeviceCSRTensors", alpha: float = 1.0, beta: float = 0.0) -> float:
        out = C.c_double(0.0)
        self.check(self.lib.trl_cuda_csr_norm1(self.h, C.byref(A.desc), alpha, beta, C.byref(out)))
        return out.value

    def sddmm(self, A: "DeviceCSRTensors", X, w, out):
        n, k = X.shape
        self.check(self.lib.trl_cuda_sddmm(self.h, C.byref(A.desc), _ptr(X), k, _ptr(w), _ptr(out)))

    def eigen_adjoint(self, pattern: "DeviceCSRTensors", X, evals: np.ndarray, weights: np.ndarray, grad, kind: int = 0,
                      cluster_rtol: float = 1e-8):
        """grad[p] = d(sum_c w_c lambda_c)/d(entry p) over the CSR pattern (kind 0: operator /
        stiffness entries; kind 1: mass entries), cluster-averaged weights."""
        n, k = X.shape
        ev = np.ascontiguousarray(evals, dtype=np.float64)
        wt = np.ascontiguousarray(weights, dtype=np.float64)
        self.check(self.lib.trl_cuda_eigen_adjoint(self.h, C.byref(pattern.desc), _ptr(X), k, ev.ctypes.data, wt.ctypes.data,
                                                   cluster_rtol, kind, _ptr(grad)))

    def small_eigen_partial(self, T, beta, nev: int, tol: float, kvec: int):
        """As small_eigen, eigenvectors for the first kvec pairs (|theta| descending) only."""
        import torch

        nblk, _, bs, _ = T.shape
        N = nblk * bs
        evals = torch.empty(N, dtype=torch.float64, device=T.device)
        evecs = torch.full_like(T, float("nan"))
        host = np.zeros(N)
        nconv = C.c_int(0)
        self.check(self.lib.trl_cuda_small_eigen_partial(self.h, _ptr(T), nblk, bs, _ptr(beta), nev, tol, kvec, _ptr(evals), _ptr(evecs),
                                                         host.ctypes.data, C.byref(nconv)))
        return evals, evecs, host, nconv.value

    def small_eigen(self, T, beta, nev: int, tol: float):
        """T: block matrix (nblk, nblk, bs, bs) float64 on the device."""
        import torch

        nblk, _, bs, _ = T.shape
        N = nblk * bs
        evals = torch.empty(N, dtype=torch.float64, device=T.device)
        evecs = torch.empty_like(T)
        host = np.zeros(N)
        nconv = C.c_int(0)
        self.check(self.lib.trl_cuda_small_eigen(self.h, _ptr(T), nblk, bs, _ptr(beta), nev, tol, _ptr(evals), _ptr(evecs),
                                                 host.ctypes.data, C.byref(nconv)))
        return evals, evecs, host, nconv.value


class PreparedOp:
    """A trl_cuda_op (sliced-ELL copy of a CSR operator) owned by the handle that made it."""

    def __init__(self, handle: Handle, op, dtype: int, bs: int):
        self.handle, self.op, self.dtype, self.bs = handle, op, dtype, bs

    def info(self) -> dict:
        stored, c, longest = I64(0), C.c_int(0), C.c_int(0)
        self.handle.check(self.handle.lib.trl_cuda_op_info(self.op, C.byref(stored), C.byref(c), C.byref(longest)))
        return {"stored": stored.value, "slice_height": c.value, "longest_row": longest.value}

    def spmm(self, X, Y, alpha: float = 1.0, beta: float = 0.0, gamma: float = 0.0, W=None):
        """Y_j = alpha A X_j + beta X_j + gamma W_j; X, Y, W of shape (n, bs) or (nb, n, bs)."""
        nb = 1 if X.dim() == 2 else X.shape[0]
        self.handle.check(self.handle.lib.trl_cuda_op_spmm(self.handle.h, self.op, _ptr(X), _ptr(Y), nb, alpha, beta, gamma, _ptr(W)))

    def close(self):
        if self.op and getattr(self.handle, "h", None):
            self.handle.lib.trl_cuda_op_destroy(self.handle.h, self.op)
        self.op = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class DeviceCSRTensors:
    rowptr: object
    colind: object
    values: object
    desc: trl_csr

    @staticmethod
    def from_host(A, dtype=None, device="cuda"):
        import torch

        dtype = dtype or torch.float64
        rp = torch.from_numpy(np.ascontiguousarray(A.rowptr, dtype=np.int32)).to(device)
        ci = torch.from_numpy(np.ascontiguousarray(A.colind, dtype=np.int32)).to(device)
        va = torch.from_numpy(np.ascontiguousarray(A.values, dtype=np.float64)).to(device=device, dtype=dtype)
        desc = trl_csr(A.n, A.nnz, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), TRL_F64 if dtype == torch.float64 else TRL_F32)
        return DeviceCSRTensors(rp, ci, va, desc)


def default_params(**kw) -> trl_solve_params:
    p = trl_solve_params()
    solver_lib().trl_solve_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def _info_dict(info: trl_solve_info) -> dict:
    return {name: getattr(info, name) for name, _ in trl_solve_info._fields_}


def solve_csr_host(A, X0: np.ndarray, device: int = 0, vectors: bool = True, evecs_out: np.ndarray | None = None, **params) -> dict:
    """Host-in/host-out solve through trl_solve_csr_host.

    evecs_out: optional (n, nev) C-contiguous float64 array that receives the eigenvectors
    (implies vectors=True). A caller that solves repeatedly passes one page-locked buffer
    here: the download of a freshly allocated array runs at pageable-copy speed and faults
    in every page (about 50 ms for 226 MB)."""
    p = default_params(**params)
    n = A.n
    if evecs_out is not None:
        if not isinstance(evecs_out, np.ndarray) or evecs_out.dtype != np.float64 or evecs_out.shape != (n, p.nev) or not evecs_out.flags.c_contiguous:
            raise ValueError(f"evecs_out must be a C-contiguous float64 array of shape ({n}, {p.nev})")
        if not evecs_out.flags.writeable:
            raise ValueError("evecs_out must be writeable")
    X0 = np.ascontiguousarray(X0, dtype=np.float64).reshape(n, p.bs)
    rp = np.ascontiguousarray(A.rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(A.colind, dtype=np.int32)
    va = np.ascontiguousarray(A.values, dtype=np.float64)
    evals = np.zeros(p.nev)
    evecs = evecs_out if evecs_out is not None else (np.zeros((n, p.nev)) if vectors else None)
    resid = np.zeros(p.nev)
    info = trl_solve_info()
    L = solver_lib()
    st = L.trl_solve_csr_host(C.byref(p), device, n, A.nnz, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, X0.ctypes.data,
                              evals.ctypes.data, None if evecs is None else evecs.ctypes.data, resid.ctypes.data, C.byref(info))
    if st != TRL_OK:
        raise TrlError(st, L.trl_solver_last_error().decode())
    out = _info_dict(info)
    out.update(evals=evals, evecs=evecs, resid=resid)
    return out


def solve_csr_device(handle: Handle, A64: DeviceCSRTensors, A32: DeviceCSRTensors | None, X0, evecs=None, **params) -> dict:
    """Device-resident solve through trl_solve_csr_device (X0: (n, bs) float64 CUDA tensor)."""
    p = default_params(**params)
    evals = np.zeros(p.nev)
    resid = np.zeros(p.nev)
    info = trl_solve_info()
    L = solver_lib()
    st = L.trl_solve_csr_device(handle.h, C.byref(p), C.byref(A64.desc), None if A32 is None else C.byref(A32.desc), _ptr(X0),
                                evals.ctypes.data, _ptr(evecs), resid.ctypes.data, C.byref(info))
    if st != TRL_OK:
        raise TrlError(st, L.trl_solver_last_error().decode())
    out = _info_dict(info)
    out.update(evals=evals, resid=resid)
    return out


def solve_csr_minner_device(handle: Handle, op: DeviceCSRTensors, M: DeviceCSRTensors, X0, evecs=None, **params) -> dict:
    """Eigenpairs of an M-self-adjoint operator (e.g. M^{-1} K) with dot = V^T M W, through
    trl_solve_csr_minner_device (FP64; X0: (n, bs) float64 CUDA tensor)."""
    p = default_params(**params)
    evals = np.zeros(p.nev)
    resid = np.zeros(p.nev)
    info = trl_solve_info()
    L = solver_lib()
    st = L.trl_solve_csr_minner_device(handle.h, C.byref(p), C.byref(op.desc), C.byref(M.desc), _ptr(X0), evals.ctypes.data, _ptr(evecs), resid.ctypes.data,
                                       C.byref(info))
    if st != TRL_OK:
        raise TrlError(st, L.trl_solver_last_error().decode())
    out = _info_dict(info)
    out.update(evals=evals, resid=resid)
    return out


def read_mtx(path: str, threads: int = 0):
    """Matrix Market coordinate file -> problems.CSRMatrix in full storage, through
    trl_csr_read_mtx (the reference loader's semantics, examples/sycl/csrevp.hh:26-124)."""
    from trl_b200 import problems

    L = solver_lib()
    n, m, nnz = I64(0), I64(0), I64(0)
    rp, ci, va = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)(), C.POINTER(C.c_double)()
    st = L.trl_csr_read_mtx(os.fsencode(path), threads, C.byref(n), C.byref(m), C.byref(nnz), C.byref(rp), C.byref(ci), C.byref(va))
    if st != TRL_OK:
        raise TrlError(st, L.trl_solver_last_error().decode())
    try:
        rowptr = np.ctypeslib.as_array(rp, shape=(n.value + 1,)).copy()
        colind = np.ctypeslib.as_array(ci, shape=(nnz.value,)).copy() if nnz.value else np.zeros(0, np.int32)
        values = np.ctypeslib.as_array(va, shape=(nnz.value,)).copy() if nnz.value else np.zeros(0)
    finally:
        L.trl_csr_free_host(C.cast(rp, P), C.cast(ci, P), C.cast(va, P))
    if n.value != m.value:
        raise TrlError(TRL_EINVAL, f"matrix is {n.value} x {m.value}; the eigensolver needs a square one")
    return problems.CSRMatrix(n.value, rowptr, colind, values)
