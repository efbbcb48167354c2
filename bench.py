#!/usr/bin/env python
"""Benchmark: time to k eigenpairs at relative residual 1e-10 on one B200, FP64 and mixed
precision, through trl's unchanged BlockLanczos driver on the CUDA backend; SpMM GB/s.

Headline workload (`value`, `e2e`): the 96^3 3-D 7-point anisotropic Laplacian, axis
coefficients (1, 10, 100) (n = 884,736, nnz = 6,137,856, FP64 CSR), block size 8, the 32
largest eigenpairs, basis 48 blocks (ncv = 384), thick restart, tolerance 1e-10; seeded
synthetic start block. A "step" is one complete solve (Ritz vectors and true residuals
included) from the same start block with the operator resident in HBM.

On one GPU the same JSON line carries the other workloads of the benchmark configurations,
each solved once in FP64 and once in mixed precision after a short warm-up solve
(`workloads`; not repeated by the replicas of a multi-GPU run):
  elast64  3 dofs per node on a 64^3 node grid, 27-point coupling (n = 786,432, 61.7M
           entries), the 64 smallest eigenpairs through sigma*I - A, block size 8;
  diff512  generalised K x = lambda M x on a 512^2 grid (log-normal edge conductivities,
           lumped mass) as M^-1/2 K M^-1/2, the 16 smallest eigenpairs, block size 8;
  zipf4m   n = 4,194,304 random symmetric pattern with Zipf(1.5) row degrees capped at 512
           (145.5M entries), the 100 largest-magnitude eigenpairs, block sizes 4, 8, 16 with
           ncv = 32 * block size.
Each also reports the prepared operator's SpMM GB/s (CUDA events, behind an L2 flush).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl trl|reference]
                    [--workloads aniso96,elast64,diff512,zipf4m]

--impl reference times the reference's own OpenMP implementation (the oracle built from the
reference sources) on the host cores: one run of the reference BlockLanczos on the headline
workload, timed per restart cycle; the first W + 1 cycles are the warm-up, the next K the
steps; the full solve is projected as cycle 1 + (R - 1) x the mean steady-state cycle, R the
reference's own restart count for this workload. With --gpus N > 1 (torchrun), each rank
solves the same workload on its own GPU (replicas only); timings are the max over ranks.

--case selects a profiling driver instead (see profile_case).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to k eigenpairs at rel. residual 1e-10: mixed vs FP64 on B200; SpMM GB/s"
CFG = dict(grid=96, coef=(1.0, 10.0, 100.0), bs=8, nev=32, ncv=384, tol=1e-10, seed=42)
WORKLOAD = "anisotropic3d-96^3 (1,10,100) n=884736 nnz=6137856 bs=8 nev=32 ncv=384 tol=1e-10"


def make_workload(name: str):
    """(CSRMatrix, alpha, beta, description) of a named workload; the operator is alpha*A + beta*I."""
    from trl_b200 import problems as P

    if name == "aniso96":
        A = P.anisotropic3d(CFG["grid"], coef=CFG["coef"])
        return A, 1.0, 0.0, WORKLOAD
    if name == "elast64":
        A = P.elasticity27(64, seed=42)
        sigma = A.gershgorin_bound()
        return A, -1.0, sigma, (f"elasticity27 64^3 nodes x 3 dofs n={A.n} nnz={A.nnz} (boundary-trimmed), 64 smallest via sigma*I - A, "
                                f"sigma = Gershgorin bound {sigma:.6f}, bs=8 ncv=384 tol=1e-10")
    if name == "zipf4m":
        A = P.zipf_symmetric(int(os.environ.get("TRL_BENCH_ZIPF_N", 4_194_304)), alpha=1.5, cap=512, seed=42)
        return A, 1.0, 0.0, f"zipf_symmetric n={A.n} nnz={A.nnz} (Zipf(1.5) degrees capped at 512, mirrored), 100 largest |lambda|, ncv=32*bs, tol=1e-10"
    if name == "diff512":
        K, mass, _ = P.diffusion2d_mass(512, sigma=1.0, seed=42)
        A = P.scale_symmetric(K, 1.0 / np.sqrt(mass))
        sigma = A.gershgorin_bound()
        return A, -1.0, sigma, (f"generalised K x = lambda M x on a 512^2 grid (K: 5-point diffusion, log-normal(0,1) edge conductivities; M: lumped mass "
                                f"U[0.5,1.5]) as M^-1/2 K M^-1/2, n={A.n} nnz={A.nnz}, 16 smallest via sigma*I - A, sigma = Gershgorin bound {sigma:.6f}, tol=1e-10")
    raise ValueError(name)


REFINE_NAMES = {0: "lanczos", 1: "chebyshev", 2: "auto"}

# solve shapes of the secondary workloads: (bs, nev, ncv)
SHAPES = {"elast64": [(8, 64, 384)], "zipf4m": [(4, 100, 128), (8, 100, 256), (16, 100, 512)], "diff512": [(8, 16, 256)]}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], d.get("bf16_tflops"), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---- the reference's OpenMP path on the host cores ----------------------------------------

def cpu_info() -> dict:
    """CPU model, logical CPUs this process may use, and the physical cores among them."""
    cpus = sorted(os.sched_getaffinity(0))
    model, phys = None, set()
    try:
        cur = {}
        with open("/proc/cpuinfo") as f:
            for line in f.read().split("\n") + [""]:
                if not line.strip():
                    if "processor" in cur and int(cur["processor"]) in cpus:
                        phys.add((cur.get("physical id", "0"), cur.get("core id", cur["processor"])))
                        model = model or cur.get("model name")
                    cur = {}
                    continue
                k, _, v = line.partition(":")
                cur[k.strip()] = v.strip()
    except OSError:
        pass
    return {"model": model, "logical_cpus": len(cpus), "physical_cores": len(phys) or len(cpus)}


def load_reference_counts() -> dict:
    with open(os.path.join(ROOT, "tests", "golden", "aniso96_reference.json")) as f:
        return json.load(f)


def cpu_cycles(cycles: int) -> dict:
    """Runs the reference BlockLanczos on the headline workload for `cycles` restart cycles in
    a child process with OMP_NUM_THREADS = physical cores and OMP_PROC_BIND = close (set
    before the OpenMP runtime starts); returns the per-cycle seconds."""
    info = cpu_info()
    env = dict(os.environ, OMP_NUM_THREADS=str(info["physical_cores"]), OMP_PROC_BIND="close", OMP_PLACES="cores")
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-cycles", str(cycles)], env=env, capture_output=True, text=True, timeout=3600)
    if r.returncode != 0:
        raise RuntimeError(f"CPU baseline child failed: {r.stderr[-2000:]}")
    out = json.loads(r.stdout.strip().split("\n")[-1])
    out["cpu"] = info
    return out


def cpu_cycles_child(cycles: int) -> None:
    from oracle import oracle as O
    from trl_b200 import problems as P

    A = P.anisotropic3d(CFG["grid"], coef=CFG["coef"])
    X0 = P.initial_block(A.n, CFG["bs"], seed=CFG["seed"])
    r = O.solve_csr(A, CFG["bs"], CFG["nev"], CFG["ncv"], X0, tol=CFG["tol"], max_restarts=cycles)
    print(json.dumps({"cycle_seconds": [float(x) for x in r["cycle_seconds"]], "threads": O.num_threads()}))


def project(cycle_seconds: list[float], first: int, restarts: int) -> dict:
    """Full-solve time from per-cycle times: cycle 1 + (restarts - 1) x the mean of the
    steady-state cycles cycle_seconds[first:], with their spread."""
    steady = cycle_seconds[first:]
    mean = statistics.mean(steady)
    sd = statistics.stdev(steady) if len(steady) > 1 else 0.0
    value = cycle_seconds[0] + (restarts - 1) * mean
    return {"value": value, "cycle1_s": cycle_seconds[0], "cycle_mean_s": mean, "cycle_stdev_s": sd, "cycles_used": len(steady),
            "spread_s": (restarts - 1) * sd}


def reference_arm(args, world, rank):
    """The reference's OpenMP path on the host cores (rank 0 only)."""
    if rank != 0:
        return
    from oracle import oracle as O

    if not O.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference checkout at build time)"}))
        return
    ref = load_reference_counts()
    # one run: cycle 1 and W more warm-up cycles, then K timed cycles (the steps)
    c = cpu_cycles(1 + args.warmup + args.steps)
    cyc = c["cycle_seconds"]
    est = project(cyc, 1 + args.warmup, ref["restarts"])
    value = est["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": est["cycle_mean_s"] * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": "host OpenMP", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": c["threads"], "kind": "reference", "cpu_model": c["cpu"]["model"],
                         "physical_cores": c["cpu"]["physical_cores"], "logical_cpus": c["cpu"]["logical_cpus"], "omp_proc_bind": "close",
                         "projected_from_cycles": est,
                         "sample": f"reference BlockLanczos (ModifiedGS, CholQR) on the headline workload: one run of {len(cyc)} restart cycles; "
                                   f"each step is one steady-state cycle (cycles {2 + args.warmup}..{len(cyc)}, mean {est['cycle_mean_s']:.3f} s, "
                                   f"sd {est['cycle_stdev_s']:.3f} s); full solve projected as cycle 1 + {ref['restarts'] - 1} x mean "
                                   f"({ref['restarts']} restarts: the reference's own count for this workload, tests/golden/aniso96_reference.json)"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(cycles: int = 5):
    """The GPU arm's CPU leg: the same estimator on a run of `cycles` cycles (mean of 2..cycles)."""
    try:
        from oracle import oracle as O
    except Exception as e:  # pragma: no cover
        return {"value": None, "unavailable": str(e)}
    if not O.available():
        return {"value": None, "unavailable": "oracle/_ref not built"}
    ref = load_reference_counts()
    c = cpu_cycles(cycles)
    est = project(c["cycle_seconds"], 1, ref["restarts"])
    return {"value": est["value"], "unit": "s", "cores": c["threads"], "kind": "reference", "cpu_model": c["cpu"]["model"],
            "physical_cores": c["cpu"]["physical_cores"], "logical_cpus": c["cpu"]["logical_cpus"], "omp_proc_bind": "close",
            "projected_from_cycles": est,
            "sample": f"reference OpenMP BlockLanczos (ModifiedGS, CholQR) on the headline workload, one run of {cycles} restart cycles: "
                      f"cycle 1 {est['cycle1_s']:.2f} s, cycles 2..{cycles} mean {est['cycle_mean_s']:.3f} s (sd {est['cycle_stdev_s']:.3f} s); "
                      f"projected to {ref['restarts']} restarts (the reference's own count for this workload)"}


# ---- the CUDA backend ---------------------------------------------------------------------

class GpuSolver:
    """One workload resident on the device: FP64 and FP32 CSR, the seeded start block, a
    buffer for the eigenvectors, and the handle's timed solves (CUDA events on its stream)."""

    def __init__(self, h, A, alpha: float, beta: float, bs: int, nev: int, ncv: int, tol: float = 1e-10):
        import torch

        from trl_b200 import native
        from trl_b200 import problems as P

        self.h, self.A, self.native = h, A, native
        self.A64 = native.DeviceCSRTensors.from_host(A, torch.float64)
        self.A32 = native.DeviceCSRTensors.from_host(A, torch.float32)
        self.X0 = torch.from_numpy(P.initial_block(A.n, bs, seed=CFG["seed"])).cuda()
        self.evecs = torch.empty((A.n, nev), dtype=torch.float64, device="cuda")
        self.common = dict(bs=bs, nev=nev, ncv=ncv, tol=tol, alpha=alpha, beta=beta, max_restarts=3000, refine_max_restarts=3000, want_vectors=1)

    def solve(self, mode, **kw):
        return self.native.solve_csr_device(self.h, self.A64, self.A32, self.X0, evecs=self.evecs, mode=mode, **dict(self.common, **kw))

    def timed(self, mode, steps: int, barrier=lambda: None, profile=False, **kw):
        """Mean device milliseconds per solve over `steps` solves, their outputs, the profile
        (if requested) and the kernel launches of the solves."""
        import torch

        barrier()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if profile:
            self.h.profile(True)
        launches0 = self.h.launches()
        outs = []
        start.record()
        for _ in range(steps):
            outs.append(self.solve(mode, **kw))
        end.record()
        torch.cuda.synchronize()
        prof = self.h.profile_read() if profile else None
        if profile:
            self.h.profile(False)
        barrier()
        return start.elapsed_time(end) / steps, outs, prof, self.h.launches() - launches0


def spmm_rate(h, A, bs: int, nb: int = 1, reps: int = 7) -> dict:
    """The prepared operator's SpMM on A (block size bs, nb blocks), FP64 and FP32: median of
    `reps` launches, each behind a 256 MB L2 flush; algorithmic bytes nnz*(s_v+4) + 4(n+1) +
    2*nb*n*bs*s_x over the launch time, and the fraction of the measured copy peak."""
    import torch

    from trl_b200 import native

    hbm, _, src = peaks()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    out = {}
    for dt, es, name in ((torch.float64, 8, "f64"), (torch.float32, 4, "f32")):
        Ad = native.DeviceCSRTensors.from_host(A, dt)
        op = h.prepare(Ad, bs)
        X = torch.randn((nb, A.n, bs) if nb > 1 else (A.n, bs), dtype=dt, device="cuda")
        Y = torch.empty_like(X)
        for _ in range(3):
            op.spmm(X, Y)
        ts = []
        for _ in range(reps):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            op.spmm(X, Y)
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) * 1e-3)
        t = statistics.median(ts)
        nbytes = A.nnz * (es + 4) + 4 * (A.n + 1) + 2 * nb * A.n * bs * es
        info = op.info()
        out[name] = {"us": t * 1e6, "gbs": nbytes / t / 1e9, "frac": nbytes / t / 1e9 / hbm, "algorithmic_bytes": nbytes,
                     "stored_entries": info["stored"], "slice_height": info["slice_height"]}
        op.close()
        del Ad, X, Y
    out["peak_source"] = src
    return out


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def secondary(h, name: str, modes: list[str]) -> list[dict]:
    """FP64 and mixed solves of a secondary workload, one timed solve each after a warm-up
    solve capped at two restarts per precision (kernels, operator copies and the memory pool
    warm); the prepared SpMM's rate."""
    import torch

    from trl_b200 import native

    t0 = time.time()
    A, alpha, beta, desc = make_workload(name)
    gen_s = time.time() - t0
    res = []
    for bs, nev, ncv in SHAPES[name]:
        S = GpuSolver(h, A, alpha, beta, bs, nev, ncv)
        S.solve(native.TRL_MODE_FP64, max_restarts=2)
        S.solve(native.TRL_MODE_FP32, max_restarts=2)
        row = {"workload": name, "desc": desc, "bs": bs, "nev": nev, "ncv": ncv, "n": A.n, "nnz": A.nnz, "generate_s": gen_s}
        evs = {}
        for mode in modes:
            m = {"fp64": native.TRL_MODE_FP64, "mixed": native.TRL_MODE_MIXED, "mixed-lanczos": native.TRL_MODE_MIXED, "mixed-chebyshev": native.TRL_MODE_MIXED}[mode]
            kw = {"mixed-lanczos": {"refine": native.TRL_REFINE_LANCZOS}, "mixed-chebyshev": {"refine": native.TRL_REFINE_CHEBYSHEV}}.get(mode, {})
            ms, outs, _, launches = S.timed(m, 1, **kw)
            o = outs[-1]
            evs[mode] = o["evals"]
            r = {"seconds": ms / 1e3, "converged": bool(o["converged"]), "restarts": o["restarts"], "n_op_apply": o["n_op_apply"],
                 "max_rel_residual": o["max_rel_residual"], "max_theta_residual": o["max_theta_residual"], "kernel_launches": launches}
            if m == native.TRL_MODE_MIXED:
                r.update(restarts_fp32=o["restarts_fp32"], n_op_apply_fp32=o["n_op_apply_fp32"], seconds_fp32_phase=o["seconds_fp32"],
                         refine_used=REFINE_NAMES.get(o["refine_used"]), refine_predicted_chebyshev_s=o["refine_predicted_s"],
                         refine_estimated_lanczos_s=o["refine_lanczos_estimate_s"],
                         refine_rounds=o["refine_rounds"], refine_degree=o["refine_degree"], refine_degree_fp32=o["refine_degree_fp32"])
            row[mode] = r
        if "fp64" in evs:
            for mode in evs:
                if mode != "fp64":
                    row[mode]["max_rel_eval_diff_vs_fp64"] = rel_err(evs[mode], evs["fp64"])
                    row[mode]["speedup_vs_fp64"] = row["fp64"]["seconds"] / row[mode]["seconds"]
                    if alpha == -1.0:  # eigenvalues of A itself: sigma - theta
                        row[mode]["max_rel_eval_diff_of_A_vs_fp64"] = rel_err(beta - evs[mode], beta - evs["fp64"])
            row["evals_fp64_first_last"] = [float(evs["fp64"][0]), float(evs["fp64"][-1])]
        del S
        torch.cuda.synchronize()
        row["spmm"] = spmm_rate(h, A, bs)
        res.append(row)
    return res


def breakdown(prof: dict) -> dict:
    """Per kernel class: calls, device seconds, share, algorithmic bytes per call, GB/s, TF/s."""
    kern = {}
    for name, s in prof.items():
        if s["calls"] == 0:
            continue
        kern[name] = {"calls": s["calls"], "seconds": s["seconds"], "share": None, "bytes_per_call": s["bytes"] / s["calls"],
                      "gbs": s["bytes"] / s["seconds"] / 1e9 if s["seconds"] > 0 else None,
                      "tflops": s["flops"] / s["seconds"] / 1e12 if s["seconds"] > 0 else None}
    tot = sum(v["seconds"] for v in kern.values())
    for v in kern.values():
        v["share"] = v["seconds"] / tot if tot else None
    return kern


def load_traffic(kernel: str, algorithmic_bytes_per_call: float):
    """DRAM bytes per call: the committed ncu ratio (DRAM traffic / algorithmic bytes, from a
    capture of the same kernel) times this run's algorithmic bytes per call."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            r = json.load(f).get(kernel)
        return None if r is None else r["traffic_per_algorithmic"] * algorithmic_bytes_per_call
    except Exception:
        return None


def roofline_of(kern: dict, cls: str, hbm: float, src: str, traffic_key: str) -> dict:
    """achieved = algorithmic bytes per call / mean call duration (CUDA events on the solver's
    stream around every call of the class during the profiled solve)."""
    d = kern[cls]
    achieved = d["bytes_per_call"] / (d["seconds"] / d["calls"]) / 1e9
    return {"kernel": cls, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": load_traffic(traffic_key, d["bytes_per_call"]), "algorithmic_bytes_per_call": d["bytes_per_call"], "peak_source": src,
            "calls": d["calls"], "share_of_profiled_solve": d["share"]}


def trl_arm(args, world, rank, local):
    import torch
    import torch.distributed as dist

    from trl_b200 import native
    from trl_b200 import problems as P

    torch.cuda.set_device(local)
    # the library's kernels run on a stream of their own: programmatic dependent launch
    # (each kernel scheduled while its predecessor drains) is not used on the legacy
    # default stream
    torch.cuda.set_stream(torch.cuda.Stream(local))
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    A, _, _, _ = make_workload("aniso96")
    exact = P.anisotropic3d_eigenvalues(CFG["grid"], coef=CFG["coef"], k=CFG["nev"])
    ref_counts = load_reference_counts()
    ref_evals = np.asarray(ref_counts["evals"][: CFG["nev"]])
    h = native.Handle(local)
    S = GpuSolver(h, A, 1.0, 0.0, CFG["bs"], CFG["nev"], CFG["ncv"], CFG["tol"])
    S.common["fp32_tol"] = args.fp32_tol

    for _ in range(args.warmup):
        S.solve(native.TRL_MODE_FP64)
    for _ in range(args.warmup):
        S.solve(native.TRL_MODE_MIXED)
    # the timed solves run with the per-class profiler off (its events would add to the time)
    clocks = ClockSampler(local).start()
    ms64, outs64, _, launches = S.timed(native.TRL_MODE_FP64, args.steps, barrier)
    ms64 = max_over_ranks(ms64)
    msmx, outsmx, _, _ = S.timed(native.TRL_MODE_MIXED, args.steps, barrier)
    msmx = max_over_ranks(msmx)
    clk = clocks.stop()
    o64, omx = outs64[-1], outsmx[-1]
    # one further FP64 solve with the profiler on: kernel breakdown and roofline
    _, _, prof, _ = S.timed(native.TRL_MODE_FP64, 1, barrier, profile=True)
    _, _, profmx, _ = S.timed(native.TRL_MODE_MIXED, 1, barrier, profile=True)

    # ---- e2e: host buffers through trl_solve_csr_host, H2D/D2H inside the timed region ----
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    Ah = P.CSRMatrix(A.n, pin(A.rowptr), pin(A.colind), pin(A.values))
    X0h = pin(P.initial_block(A.n, CFG["bs"], seed=CFG["seed"]))
    evecs_h = pin(np.zeros((A.n, CFG["nev"])))  # one page-locked buffer, reused by every call
    common = dict(bs=CFG["bs"], nev=CFG["nev"], ncv=CFG["ncv"], tol=CFG["tol"], max_restarts=3000, refine_max_restarts=3000, fp32_tol=args.fp32_tol,
                  want_vectors=1)

    def e2e_run(mode, steps):
        times, last = [], None
        for i in range(1 + steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            last = native.solve_csr_host(Ah, X0h, device=local, evecs_out=evecs_h, **dict(common, mode=mode))
            torch.cuda.synchronize()
            if i > 0:
                times.append(time.perf_counter() - t0)
        return max_over_ranks(statistics.mean(times)), times, last

    e2e_clocks = ClockSampler(local).start()
    e2e_s, e2e_times, e2e = e2e_run(native.TRL_MODE_FP64, args.steps)
    e2e_mx_s, e2e_mx_times, e2e_mx = e2e_run(native.TRL_MODE_MIXED, min(args.steps, 5))
    e2e_clk = e2e_clocks.stop()

    # ---- roofline: the metric's kernel (SpMM) and the dominant streaming class ----
    hbm, _, src = peaks()
    kern = breakdown(prof)
    kernmx = breakdown(profmx)
    roofline = roofline_of(kern, "spmm", hbm, src, "spmm_sell")
    not_hbm = ("small_eigen", "reorth_pass2", "block_ops")
    dominant = max((k for k in kern if k not in not_hbm and kern[k]["bytes_per_call"] > 0), key=lambda k: kern[k]["seconds"])
    roofline["dominant_streaming_class"] = roofline_of(kern, dominant, hbm, src, dominant)
    roofline["not_hbm_classes"] = {k: round(kern[k]["share"], 4) for k in not_hbm if k in kern}
    roofline["mixed_mode_spmm"] = roofline_of(kernmx, "spmm", hbm, src, "spmm_sell")

    # ---- the other workloads of the benchmark configurations ----
    wl = {}
    # single-GPU runs only: replicas on more GPUs would repeat the same per-GPU solves (and
    # each rank would generate the 145M-entry Zipf pattern on the host)
    names = [w for w in args.workloads.split(",") if w and w != "aniso96"] if world == 1 else []
    for name in names:
        t0 = time.time()
        wl[name] = secondary(h, name, args.secondary_modes.split(","))
        for row in wl[name]:
            row["wall_s"] = time.time() - t0
    spmm_head = spmm_rate(h, A, CFG["bs"])

    result = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline()
        result = {
            "metric": METRIC, "value": ms64 / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms64, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "mode": "fp64",
                       "reorth": "partial: block classical Gram-Schmidt (DGKS second pass) at the steps where a random sketch of the basis shows orthogonality loss > 1e-12",
                       "orthonormalize": "CholQR2", "operator": "prepared sliced-ELL copy (SELL-C-sigma, C = 16 rows, sigma = 4096), built inside each solve",
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (basis 2.8 GB, CSR 113 MB, per-step working set >> 126 MB)"},
            "fp64": {"seconds": ms64 / 1e3, "restarts": o64["restarts"], "n_op_apply": o64["n_op_apply"], "converged": bool(o64["converged"]),
                     "max_rel_residual": o64["max_rel_residual"], "max_rel_err_vs_analytic": rel_err(o64["evals"], exact),
                     "max_rel_err_vs_reference": rel_err(o64["evals"], ref_evals)},
            "mixed": {"seconds": msmx / 1e3, "speedup_vs_fp64": ms64 / msmx,
                      "refine": "automatic: Chebyshev-filtered subspace iteration + Rayleigh-Ritz on nev/bs+2 blocks when predicted faster than a BlockLanczos restart from the FP32 Ritz vectors",
                      "refine_used": REFINE_NAMES.get(omx["refine_used"]), "refine_predicted_chebyshev_s": omx["refine_predicted_s"],
                      "refine_estimated_lanczos_s": omx["refine_lanczos_estimate_s"],
                      "restarts_fp32": omx["restarts_fp32"], "n_op_apply_fp32": omx["n_op_apply_fp32"], "seconds_fp32_phase": omx["seconds_fp32"],
                      "refine_rounds": omx["refine_rounds"], "refine_degree": omx["refine_degree"],
                      "refine_degree_fp32": omx["refine_degree_fp32"], "fp32_tol": args.fp32_tol,
                      "converged": bool(omx["converged"]), "max_rel_residual": omx["max_rel_residual"], "max_theta_residual": omx["max_theta_residual"],
                      "max_rel_err_vs_analytic": rel_err(omx["evals"], exact), "max_rel_err_vs_reference": rel_err(omx["evals"], ref_evals),
                      "e2e_s": e2e_mx_s},
            "spmm": spmm_head,
            "kernels": kern,
            "kernels_mixed": kernmx,
            "roofline": roofline,
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(e2e["h2d_bytes"]), "d2h_bytes_per_step": int(e2e["d2h_bytes"]),
                    "api": "trl_solve_csr_host (pinned host CSR + start block in, eigenvalues + eigenvectors out into a pinned buffer)",
                    "steps_s": e2e_times, "device_s_last": e2e["seconds"], "clocks": e2e_clk,
                    "mixed": {"value": e2e_mx_s, "steps_s": e2e_mx_times, "h2d_bytes_per_step": int(e2e_mx["h2d_bytes"]),
                              "d2h_bytes_per_step": int(e2e_mx["d2h_bytes"])}},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
            "workloads": wl,
        }
        print(json.dumps(result), flush=True)
    del S
    h.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


def profile_case(args):
    """Profiling drivers: run one piece of a workload (--workload, default aniso96) and exit.
    solve        one FP64 solve capped at --restarts restart cycles (launch lists);
    mixed        one complete mixed-mode solve;
    solves       complete solves of --bs in each of --modes (fp64, fp32, mixed, mixed-lanczos),
                 one JSON line each (restarts, applies, refinement rounds, residuals, seconds);
    spmm         the prepared operator's SpMM, --reps launches (--nb blocks, --fp32);
    spmm-csr     the CSR kernel (trl_cuda_spmm / _blocks) on the same operands;
                 (fp64-fullreorth, fp64-cgs2: FP64 with every step projected);
    spmm-rates   prepared operator against the CSR kernel, one JSON line per dtype and block
                 count, each timed launch behind an L2 flush;
    dot / update one multi-block inner product / projection update against --nblk blocks;
    project      one Gram-Schmidt pass as the solver issues it, against --nblk blocks;
    rotate       the thick-restart rotation V (48 blocks) x Y -> 5 blocks;
    small-eigen  the projected eigenproblem of a thick-restart matrix (N = --nblk x 8, the
                 kept 40 eigenvectors), --reps calls;
    dmma-peak    the FP64 tensor-core (DMMA) throughput of the GPU (trl_cuda_measure_dmma_rate).
    Every case on the default workload reads and writes more than the 126 MB L2 and holds at
    most a few GB."""
    import torch

    from trl_b200 import native
    from trl_b200 import problems as P

    A, alpha, beta, _ = make_workload(args.workload)
    bs = args.bs
    dt = torch.float32 if args.fp32 else torch.float64
    torch.cuda.set_stream(torch.cuda.Stream(0))  # as in the bench proper
    h = native.Handle(0)
    if args.case in ("solve", "mixed", "solves"):
        nev, ncv = {"aniso96": (CFG["nev"], CFG["ncv"]), "elast64": (64, 384), "zipf4m": (100, 32 * bs), "diff512": (16, 32 * bs)}[args.workload]
        S = GpuSolver(h, A, alpha, beta, bs, nev, ncv)
        S.common["fp32_tol"] = args.fp32_tol
        if args.case == "solve":
            S.solve(native.TRL_MODE_FP32 if args.fp32 else native.TRL_MODE_FP64, max_restarts=args.restarts, want_vectors=0)
        elif args.case == "mixed":
            S.solve(native.TRL_MODE_MIXED)
        else:
            modes = {"fp64": (native.TRL_MODE_FP64, {}), "fp32": (native.TRL_MODE_FP32, {}), "mixed": (native.TRL_MODE_MIXED, {}),
                     "mixed-lanczos": (native.TRL_MODE_MIXED, {"refine": native.TRL_REFINE_LANCZOS}),
                     "mixed-chebyshev": (native.TRL_MODE_MIXED, {"refine": native.TRL_REFINE_CHEBYSHEV}),
                     "fp64-fullreorth": (native.TRL_MODE_FP64, {"reorth": native.TRL_REORTH_CGS_IFNEEDED}),
                     "fp64-cgs2": (native.TRL_MODE_FP64, {"reorth": native.TRL_REORTH_CGS2})}
            for name in args.modes.split(","):
                mode, kw = modes[name]
                ms, outs, _, launches = S.timed(mode, 1, max_restarts=args.restarts, refine_max_restarts=args.restarts, **dict(kw, **json.loads(args.params)))
                o = outs[-1]
                keep = ("converged", "restarts", "n_op_apply", "restarts_fp32", "n_op_apply_fp32", "seconds_fp32", "refine_rounds", "refine_degree",
                        "refine_degree_fp32", "max_rel_residual", "max_theta_residual")
                print(json.dumps({"case": "solves", "workload": args.workload, "bs": bs, "mode": name, "params": json.loads(args.params), "seconds": ms / 1e3, "launches": launches,
                                  **{k: o[k] for k in keep}, "evals_head": [float(x) for x in o["evals"][:3]],
                                  "evals_tail": [float(x) for x in o["evals"][-3:]]}), flush=True)
    elif args.case == "spmm-rates":
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        hbm, _, _ = peaks()

        def tm(fn, reps=7):
            for _ in range(3):
                fn()
            ts = []
            for _ in range(reps):
                flush.fill_(1)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                fn()
                b.record()
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b) * 1e-3)
            return statistics.median(ts)

        for dtt, es in ((torch.float64, 8), (torch.float32, 4)):
            Ad = native.DeviceCSRTensors.from_host(A, dtt)
            op = h.prepare(Ad, bs)
            for nb in sorted({1, args.nb}):
                X = torch.randn(nb, A.n, bs, dtype=dtt, device="cuda")
                Y = torch.empty_like(X)
                tc = tm(lambda: h.spmm(Ad, X[0], Y[0]) if nb == 1 else h.spmm_blocks(Ad, X, Y, 1.0, 0.0, 0.0, None))
                to = tm(lambda: op.spmm(X[0] if nb == 1 else X, Y[0] if nb == 1 else Y))
                nbytes = A.nnz * (es + 4) + 4 * (A.n + 1) + nb * 2 * A.n * bs * es
                print(json.dumps({"case": "spmm-rates", "workload": args.workload, "dtype": "f64" if es == 8 else "f32", "bs": bs, "nb": nb,
                                  "csr_us": tc * 1e6, "op_us": to * 1e6, "csr_frac": nbytes / tc / 1e9 / hbm, "op_frac": nbytes / to / 1e9 / hbm,
                                  **op.info()}), flush=True)
                del X, Y
            op.close()
            del Ad
    elif args.case in ("spmm", "spmm-csr"):
        Ad = native.DeviceCSRTensors.from_host(A, dt)
        X = torch.randn(args.nb, A.n, bs, dtype=dt, device="cuda")
        Y = torch.empty_like(X)
        if args.case == "spmm":
            op = h.prepare(Ad, bs)
            for _ in range(args.reps):
                op.spmm(X[0] if args.nb == 1 else X, Y[0] if args.nb == 1 else Y)
            torch.cuda.synchronize()
            op.close()
        else:
            for _ in range(args.reps):
                if args.nb == 1:
                    h.spmm(Ad, X[0], Y[0])
                else:
                    h.spmm_blocks(Ad, X, Y, 1.0, 0.0, 0.0, None)
    elif args.case == "project":
        store = torch.randn(args.nblk + 1, A.n, bs, dtype=dt, device="cuda")
        G = torch.empty(bs, bs, dtype=torch.float64, device="cuda")
        for _ in range(args.reps):
            h.project_out(store[: args.nblk], store[args.nblk], native.TRL_CGS_ONE, G)
    elif args.case in ("dot", "update"):
        V = torch.randn(args.nblk, A.n, bs, dtype=dt, device="cuda")
        w = torch.randn(A.n, bs, dtype=dt, device="cuda")
        Cm = torch.randn(args.nblk, bs, bs, dtype=torch.float64, device="cuda") * 1e-3
        for _ in range(args.reps):
            if args.case == "dot":
                h.block_dot(V, w, Cm)
            else:
                h.block_update(w, V, Cm)
    elif args.case == "rotate":
        V = torch.randn(48, A.n, bs, dtype=dt, device="cuda")
        Y = torch.randn(48, 48, bs, bs, dtype=torch.float64, device="cuda")
        W = torch.empty(5, A.n, bs, dtype=dt, device="cuda")
        for _ in range(args.reps):
            h.block_rotate(V, Y, 5, W)
    elif args.case == "dmma-peak":
        tf = native.C.c_double(0.0)
        h.check(h.lib.trl_cuda_measure_dmma_rate(h.h, native.C.byref(tf)))
        print(json.dumps({"case": "dmma-peak", "tflops": tf.value, "how": "independent DMMA m8n8k4 chains on every SM, CUDA events"}), flush=True)
    elif args.case == "small-eigen":
        # a thick-restart projected matrix (lanczos.hh:119-150): kept Ritz values on the
        # diagonal, their coupling to the next block, block-tridiagonal below
        rng = np.random.default_rng(5)
        nblk, kr, b8 = args.nblk, 5, 8
        N = nblk * b8
        T = np.zeros((N, N))
        T[: kr * b8, : kr * b8] = np.diag(np.sort(rng.uniform(440, 444, kr * b8))[::-1])
        for b in range(kr, nblk):
            D = rng.standard_normal((b8, b8)) * 50 + np.eye(b8) * 200
            T[b * b8:(b + 1) * b8, b * b8:(b + 1) * b8] = D + D.T
            if b + 1 < nblk:
                Bt = np.triu(rng.standard_normal((b8, b8))) * 20
                T[(b + 1) * b8:(b + 2) * b8, b * b8:(b + 1) * b8] = Bt
                T[b * b8:(b + 1) * b8, (b + 1) * b8:(b + 2) * b8] = Bt.T
        C = rng.standard_normal((b8, kr * b8)) * 1e-3
        T[kr * b8:(kr + 1) * b8, : kr * b8] = C
        T[: kr * b8, kr * b8:(kr + 1) * b8] = C.T
        Tb = torch.from_numpy(T.reshape(nblk, b8, nblk, b8).transpose(0, 2, 1, 3).copy()).cuda()
        beta_ = torch.from_numpy(np.triu(rng.standard_normal((b8, b8))) * 1e-9).cuda()
        times = []
        for _ in range(args.reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(torch.cuda.current_stream())
            h.small_eigen_partial(Tb, beta_, 32, 1e-10, (kr + 1) * b8)
            b.record(torch.cuda.current_stream())
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        print(json.dumps({"case": "small-eigen", "N": N, "kvec": (kr + 1) * b8, "ms": times}), flush=True)
    torch.cuda.synchronize()
    h.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["trl", "reference"], default="trl")
    ap.add_argument("--fp32-tol", type=float, default=3e-3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workloads", default="aniso96,elast64,diff512,zipf4m", help="headline workload plus the secondary ones solved once per mode")
    ap.add_argument("--secondary-modes", default="fp64,mixed")
    ap.add_argument("--cpu-cycles", type=int, default=0, help=argparse.SUPPRESS)  # child process of the CPU legs
    ap.add_argument("--case", choices=["solve", "mixed", "solves", "spmm", "spmm-csr", "spmm-rates", "dot", "update", "project", "rotate", "small-eigen", "dmma-peak"],
                    default=None, help="profiling driver: run one piece of a workload and exit (see profile_case)")
    ap.add_argument("--workload", default="aniso96", choices=["aniso96", "elast64", "zipf4m", "diff512"])
    ap.add_argument("--modes", default="fp64,mixed")
    ap.add_argument("--params", default="{}", help="solves: extra solver parameters (JSON object of trl_solve_params fields)")
    ap.add_argument("--bs", type=int, default=8)
    ap.add_argument("--nb", type=int, default=1)
    ap.add_argument("--restarts", type=int, default=3)
    ap.add_argument("--nblk", type=int, default=24)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--fp32", action="store_true")
    args = ap.parse_args()
    if args.cpu_cycles:
        cpu_cycles_child(args.cpu_cycles)
        return
    if args.case:
        profile_case(args)
        return
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        reference_arm(args, world, rank)
        return
    trl_arm(args, world, rank, local)


if __name__ == "__main__":
    main()
