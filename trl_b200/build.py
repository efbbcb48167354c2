"""Build recipe of the B200 backend (run by ``__graft_entry__.build()`` or
``python -m trl_b200.build``). Outputs go to ``trl_b200/lib/`` (git-ignored; the built files
travel with the source tree to the GPU host):

* ``libtrl_cuda.so``       the sm_100a kernels behind the C ABI (include/trl_cuda.h);
* ``libtrl_solver.so``     trl's BlockLanczos driver, unchanged, on the CUDA backend
                           (include/trl_solver.h) — compiled against the reference headers;
* ``trl_cuda_ref_tests``   the reference's own test bodies on the CUDA backend (a test
                           program; source in tests/host/).

The last two need the reference checkout (trl is header-only); without it only
``libtrl_cuda.so`` is built.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
OBJ = os.path.join(ROOT, "_build")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# The image exports CXX pointing at a wrapper compiler; the system g++ is used explicitly.
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["context.cu", "blockvec.cu", "spmm.cu", "sell.cu", "small.cu"]
# TRL_DEBUG_TRACE=1 at build time compiles the stderr traces of the partial
# reorthogonalisation and of the mixed-mode refinement in (enabled at run time by
# TRL_PARTIAL_TRACE / TRL_REFINE_TRACE); rebuild from scratch after changing it
DEBUG = ["-DTRL_DEBUG_TRACE"] if os.environ.get("TRL_DEBUG_TRACE") else []
# the header-only reference checkout (build time only): $TRL_REFERENCE or the default mount
DEFAULT_REF = os.environ.get("TRL_REFERENCE", "/root/reference")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers(*dirs: str) -> list[str]:
    out = []
    for d in dirs:
        for base, _, files in os.walk(d):
            out += [os.path.join(base, f) for f in files if f.endswith((".h", ".hh", ".cuh"))]
    return out


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_cuda(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers(CSRC, INCLUDE)
    objs, cmds = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if _newer(o, [s] + hdrs):
            cmds.append([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", *DEBUG, f"-I{INCLUDE}", "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(lambda c: _run(c, verbose), cmds))
    so = os.path.join(LIB, "libtrl_cuda.so")
    if _newer(so, objs):
        _run([NVCC, *ARCH, "-shared", "-o", so, *objs, f"-L{CUDA_HOME}/lib64", "-lcusolver"], verbose)
    return so


def build_solver(ref: str = DEFAULT_REF, verbose: bool = False) -> list[str]:
    ref_inc = os.path.join(ref, "include")
    ref_tests = os.path.join(ref, "tests")
    if not os.path.isdir(ref_inc):
        return []
    hdrs = _headers(INCLUDE) + _headers(ref_inc)
    common = [CXX, "-std=c++20", "-O2", "-fPIC", *DEBUG, f"-I{INCLUDE}", f"-I{ref_inc}", f"-I{CUDA_HOME}/include"]
    link = [f"-L{LIB}", "-ltrl_cuda", f"-L{CUDA_HOME}/lib64", "-lcudart", "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{CUDA_HOME}/lib64"]
    out = []
    srcs = [os.path.join(CSRC, "solver", f) for f in ("solver_capi.cc", "mtx.cc")]
    so = os.path.join(LIB, "libtrl_solver.so")
    if _newer(so, srcs + [os.path.join(LIB, "libtrl_cuda.so")] + hdrs):
        _run(common + ["-shared", "-o", so, *srcs] + link + ["-pthread"], verbose)
    out.append(so)
    src = os.path.join(ROOT, "tests", "host", "ref_tests_cuda.cc")  # a test program
    exe = os.path.join(LIB, "trl_cuda_ref_tests")
    if os.path.isdir(ref_tests) and _newer(exe, [src, os.path.join(LIB, "libtrl_cuda.so")] + hdrs + _headers(ref_tests)):
        _run(common + [f"-I{ref_tests}", "-o", exe, src] + link, verbose)
    out.append(exe)
    return out


def build(ref: str = DEFAULT_REF, verbose: bool = False) -> None:
    build_cuda(verbose)
    build_solver(ref, verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
