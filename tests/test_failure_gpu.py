"""Failure detection without a GPU fault: the errors are made on the host or by a bounded
device wait that runs out, and the handle is checked to stay usable afterwards.

* A bounded wait that never completes (trl_cuda_test_bounded_wait: a shared-memory barrier
  expecting two arrivals gets one; no copies are in flight) gives up after its poll limit,
  records the timeout in the handle's status word, and the next trl_cuda_synchronize
  returns TRL_ETIMEOUT, the status every bounded wait of the library reports.
* A refused allocation (trl_cuda_inject_alloc_failures: the handle's memory pool refuses
  the next allocations, on the host) makes a solve return TRL_ENOMEM instead of crashing.
"""
import numpy as np
import pytest
import torch

from trl_b200 import native
from trl_b200 import problems as P

pytestmark = pytest.mark.gpu


def _dot_works(h):
    rng = np.random.default_rng(3)
    V = rng.standard_normal((2, 1000, 4))
    W = rng.standard_normal((1000, 4))
    C = torch.zeros((2, 4, 4), dtype=torch.float64, device="cuda")
    h.block_dot(torch.from_numpy(V).cuda(), torch.from_numpy(W).cuda(), C)
    h.sync()
    assert np.allclose(C.cpu().numpy(), np.einsum("jnb,nc->jbc", V, W), rtol=1e-12, atol=1e-10)


def test_bounded_wait_times_out_and_the_handle_stays_usable():
    h = native.Handle(0)
    try:
        assert h.lib.trl_cuda_test_bounded_wait(h.h, 1000) == native.TRL_OK
        assert h.lib.trl_cuda_synchronize(h.h) == native.TRL_ETIMEOUT
        assert b"timed out" in h.lib.trl_cuda_last_error(h.h)
        # the status word was read and cleared; the stream and context keep working
        assert h.lib.trl_cuda_synchronize(h.h) == native.TRL_OK
        _dot_works(h)
        # out-of-range poll limits are refused without launching
        assert h.lib.trl_cuda_test_bounded_wait(h.h, 0) == native.TRL_EINVAL
        assert h.lib.trl_cuda_test_bounded_wait(h.h, (1 << 24) + 1) == native.TRL_EINVAL
    finally:
        h.close()


def test_refused_allocation_makes_a_solve_return_enomem():
    A = P.laplace2d(32)
    X0 = torch.from_numpy(P.initial_block(A.n, 4, seed=42)).cuda()
    h = native.Handle(0)
    try:
        A64 = native.DeviceCSRTensors.from_host(A)
        assert h.lib.trl_cuda_inject_alloc_failures(h.h, 1) == native.TRL_OK
        with pytest.raises(native.TrlError) as e:
            native.solve_csr_device(h, A64, None, X0, bs=4, nev=8, ncv=48, tol=1e-10)
        assert e.value.status == native.TRL_ENOMEM
        assert "refused" in str(e.value)
        # later allocations succeed again and the same handle solves
        out = native.solve_csr_device(h, A64, None, X0, bs=4, nev=8, ncv=48, tol=1e-10)
        assert out["converged"]
        exact = P.laplace2d_eigenvalues(32)[:8]
        assert np.max(np.abs(out["evals"] - exact) / exact) < 1e-10
        # the refusal covers exactly `count` allocations
        assert h.lib.trl_cuda_inject_alloc_failures(h.h, 0) == native.TRL_OK
        p = native.C.c_void_p()
        assert h.lib.trl_cuda_inject_alloc_failures(h.h, 1) == native.TRL_OK
        assert h.lib.trl_cuda_malloc(h.h, native.C.byref(p), 1024) == native.TRL_ENOMEM
        assert h.lib.trl_cuda_malloc(h.h, native.C.byref(p), 1024) == native.TRL_OK
        assert h.lib.trl_cuda_free(h.h, p) == native.TRL_OK
    finally:
        h.close()
