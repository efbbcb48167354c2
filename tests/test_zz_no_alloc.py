"""The allocation-free block dot (trl_cuda_block_dot_noalloc) against the regular one.

Some callers cannot let a library allocate GPU memory: programs that route every device
allocation through their own pool, and loops that cannot afford an allocation or the
device-wide synchronisation of freeing one. For them the library keeps the partial sums of
this one kernel in a fixed device array. This test calls that entry point through the C ABI
twice in a row (different shapes, so the second call runs over what the first left in the
shared array) and compares both results with trl_cuda_block_dot, to the same 1e-12 relative
tolerance the other kernel tests use. It also checks that a request larger than the array
is refused without touching the output.

The file name sorts last so that a run stopping at the first failure has run every other
test before this one; it passes on its own in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from trl_b200 import native

pytestmark = pytest.mark.gpu

MAX_ENTRIES = 16384  # TRL_CUDA_NOALLOC_MAX_ENTRIES in include/trl_cuda.h


def _noalloc():
    lib = native.cuda_lib()
    fn = lib.trl_cuda_block_dot_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
    return fn


def _stream():
    # torch's default stream is the legacy stream; its cudaStream_t value is 0, which the
    # CUDA runtime also reads as the legacy stream
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _reference(V, W):
    h = native.Handle(0)
    out = torch.zeros((V.shape[0], V.shape[2], V.shape[2]), dtype=torch.float64, device="cuda")
    h.block_dot(V, W, out)
    torch.cuda.synchronize()
    h.close()
    return out.cpu().numpy()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_dot_matches_block_dot_twice(dtype):
    fn = _noalloc()
    rng = np.random.default_rng(123)
    cases = [(8, 24, 200_003), (16, 3, 70_001)]  # (bs, nblk, n): second call reuses the array
    for bs, nblk, n in cases:
        V = torch.from_numpy(rng.standard_normal((nblk, n, bs))).to("cuda", dtype)
        W = torch.from_numpy(rng.standard_normal((n, bs))).to("cuda", dtype)
        ref = _reference(V, W)
        out = torch.full((nblk, bs, bs), float("nan"), dtype=torch.float64, device="cuda")
        st = fn(_stream(), native.TRL_F64 if dtype == torch.float64 else native.TRL_F32, V.data_ptr(), nblk, W.data_ptr(), n, bs, out.data_ptr())
        assert st == native.TRL_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        scale = float((V.double().abs().transpose(1, 2) @ W.double().abs()).max())
        assert np.max(np.abs(got - ref)) <= 1e-12 * scale


def test_noalloc_dot_rejects_oversized_output():
    fn = _noalloc()
    bs, nblk, n = 16, MAX_ENTRIES // (16 * 16) + 1, 1000
    V = torch.zeros((nblk, n, bs), dtype=torch.float64, device="cuda")
    W = torch.zeros((n, bs), dtype=torch.float64, device="cuda")
    out = torch.full((nblk, bs, bs), 7.0, dtype=torch.float64, device="cuda")
    st = fn(_stream(), native.TRL_F64, V.data_ptr(), nblk, W.data_ptr(), n, bs, out.data_ptr())
    assert st == native.TRL_EINVAL
    torch.cuda.synchronize()
    assert torch.all(out == 7.0)
