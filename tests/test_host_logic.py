"""Host-side logic that needs no GPU.

* trl::cuda::Context's batching of the thick-restart rotation (include/trl/impl/cuda/context.hh)
  against a fake C ABI: the pattern of lanczos.hh:105-114 becomes one trl_cuda_block_rotate;
  any other sequence is replayed call by call in its original order.
* Its three-term fusion (lanczos.hh:243-262): product/subtract pairs become one kernel, the
  temporary's write is deferred, and written exactly when a later operation needs it.
* The C-ABI libraries load without a GPU and export every function include/*.h declares.
* The multi-rank reduction bench.py uses (max over ranks) on a 2-rank gloo group.
* The launch discipline of trl_b200/csrc: every kernel starts with the programmatic-
  dependent-launch wait, and every launch goes through the library's launch helper.
"""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def batching_output(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("host") / "context_batching")
    src = os.path.join(ROOT, "tests", "host", "context_batching.cc")
    subprocess.run(["/usr/bin/g++", "-std=c++20", "-O1", f"-I{ROOT}/include", src, "-o", exe], check=True)
    return subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines()


def line(out, key):
    return next(ln for ln in out if ln.startswith(key + " "))


def test_restart_pattern_becomes_one_rotation(batching_output):
    got = line(batching_output, "case1").split(" ", 2)
    assert got[1] == "1"
    assert got[2] == line(batching_output, "expect1").split(" ", 1)[1]


def test_irregular_sequences_are_replayed_in_order(batching_output):
    assert line(batching_output, "case2") == "case2 3 zero | mult 2 | mult 2"
    assert line(batching_output, "case3") == "case3 1 mult 2"
    assert line(batching_output, "case4") == "case4 3"


def test_single_input_block_and_flush_on_shape_change(batching_output):
    assert line(batching_output, "case5") == "case5 1 rotate"
    # the pending single-block group (zero + one mult_add) is itself a k=1, m=1 rotation
    assert line(batching_output, "case6") == "case6 2 rotate zero"
    assert line(batching_output, "case7") == "case7 1"
    assert line(batching_output, "fused") == "fused 3"


def test_three_term_step_runs_fused_with_its_temporary_deferred(batching_output):
    # nothing is issued while the driver's step is recorded; the projection issues it as
    # W -= V_{i-1} beta^T (one kernel), the dot, W -= V_i T_ii (one kernel)
    assert line(batching_output, "case8a") == "case8a 0"
    got = line(batching_output, "case8").split(" ", 1)[1]
    assert got == line(batching_output, "expect8").split(" ", 1)[1]
    # the deferred W0 survives unrelated operations and is dropped by the next step's overwrite
    assert line(batching_output, "case8b") == "case8b 3 0 4"


def test_deferred_product_is_written_before_it_is_needed(batching_output):
    got = line(batching_output, "case9").split(" ", 2)
    assert got[1] == "1" and got[2] == line(batching_output, "expect9").split(" ", 1)[1]
    assert line(batching_output, "case10") == "case10 1 mult 0"
    assert line(batching_output, "case10b") == "case10b 0"
    # the restart step: dot, two fused subtractions, and flush() writes the last product
    assert re.fullmatch(r"case11 4 dot \d+,mult 3,mult 4,mult 1,", line(batching_output, "case11"))


def test_reference_modified_gs_and_unbatched_calls(batching_output):
    # ModifiedGS's dot joins the record; its subtract_product issues everything in order
    assert re.fullmatch(r"case12 4 mult 4,dot \d+,mult 3,dot \d+,", line(batching_output, "case12"))
    # batching off: every call runs at once, nothing is fused
    assert line(batching_output, "case7b") == "case7b 5"


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(trl_[a-z0-9_]+)\s*\(", text)))


def test_cuda_library_exports_every_declared_symbol():
    from trl_b200 import native

    lib = ctypes.CDLL(native.CUDA_LIB)
    names = _declared("trl_cuda.h")
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(native.CUDA_SYMBOLS), set(names) - set(native.CUDA_SYMBOLS)


def test_solver_library_exports_every_declared_symbol():
    from trl_b200 import native

    if not os.path.exists(native.SOLVER_LIB):
        pytest.skip("solver library needs the reference headers at build time")
    ctypes.CDLL(native.CUDA_LIB, mode=ctypes.RTLD_GLOBAL)
    lib = ctypes.CDLL(native.SOLVER_LIB)
    for name in _declared("trl_solver.h"):
        assert hasattr(lib, name), name


def test_status_strings_without_gpu():
    from trl_b200 import native

    lib = native.cuda_lib()
    assert lib.trl_cuda_status_string(native.TRL_ECHOLESKY).decode() == "Cholesky factorization failed in orthonormalize"
    assert lib.trl_cuda_status_string(native.TRL_EEIGEN).decode() == "Eigendecomposition failed"


def _max_over_ranks(rank, world, port, q):
    import torch
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    t = torch.tensor([float(rank + 1) * 1.5], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    q.put((rank, float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_max_over_ranks, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    vals = sorted(q.get(timeout=10) for _ in range(2))
    assert vals == [(0, 3.0), (1, 3.0)]


def test_solve_csr_host_rejects_bad_eigenvector_buffers():
    """The caller's eigenvector buffer is checked before anything reaches the library."""
    import numpy as np

    from trl_b200 import native
    from trl_b200 import problems as P

    A = P.laplace2d(8)
    X0 = np.zeros((A.n, 4))
    ro = np.zeros((A.n, 10))
    ro.flags.writeable = False
    for bad in (np.zeros((A.n, 9)), np.zeros((A.n, 10), dtype=np.float32), np.zeros((10, A.n)).T, ro, [[0.0] * 10] * A.n):
        with pytest.raises(ValueError):
            native.solve_csr_host(A, X0, evecs_out=bad, bs=4, nev=10, ncv=160)


def _csrc_files():
    d = os.path.join(ROOT, "trl_b200", "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d)) if f.endswith(".cu")]


def _strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def test_every_kernel_waits_for_its_predecessor_first():
    """Kernels are launched with programmatic stream serialization (trl_detail::launch), so a
    kernel may be scheduled while the previous one of its stream still runs. Each must
    begin with pdl_enter() (griddepcontrol.wait) before it touches global memory; this
    checks that the first statement of every __global__ function is that call."""
    kernels = 0
    for path in _csrc_files():
        src = _strip_comments(open(path).read())
        for m in re.finditer(r"__global__", src):
            body = src.index("{", m.end())
            first = src[body + 1:].lstrip()
            name = re.search(r"(k_\w+)\s*\(", src[m.end():body]).group(1)
            assert first.startswith("::trl_detail::pdl_enter();"), f"{os.path.basename(path)}: {name} does not start with pdl_enter()"
            kernels += 1
    assert kernels >= 40


def test_every_launch_goes_through_the_launch_helper():
    """No kernel is launched with <<<>>> (which would bypass the launch attributes the
    library sets); the cluster launch of the tridiagonalisation uses cudaLaunchKernelEx."""
    for path in _csrc_files():
        src = _strip_comments(open(path).read())
        assert "<<<" not in src, os.path.basename(path)


def test_integration_example_compiles():
    """The documented C++ usage (tests/host/integration_example.cc) compiles against the
    reference's headers and this repository's include/."""
    from oracle import oracle as O

    ref_inc = os.path.join(O.reference_root(), "include")
    if not os.path.isdir(os.path.join(ref_inc, "trl")):
        pytest.skip("the reference headers are not present")
    src = os.path.join(ROOT, "tests", "host", "integration_example.cc")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    r = subprocess.run(["/usr/bin/g++", "-std=c++20", "-fsyntax-only", f"-I{ref_inc}", f"-I{ROOT}/include", f"-I{cuda_inc}", src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
