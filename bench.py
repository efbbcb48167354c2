#!/usr/bin/env python
"""Benchmark: time to k eigenpairs at relative residual 1e-10 on one B200 (FP64 and mixed
precision) through trl's unchanged BlockLanczos driver on the CUDA backend, with SpMM and
block-kernel GB/s measured live (CUDA events) during one further profiled FP64 solve.

Workload (default): the 96^3 3-D 7-point anisotropic Laplacian, axis coefficients
(1, 10, 100) (n = 884,736, nnz = 6,137,856, FP64 CSR), block size 8, the 32 largest
eigenpairs, basis 48 blocks (ncv = 384), thick restart, tolerance 1e-10; seeded synthetic
start block. A "step" is one complete solve (Ritz vectors and true residuals included) from
the same start block with the operator already resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl trl|reference]

--impl reference times the reference's own OpenMP implementation (the oracle built from the
reference sources) on the host cores: each step is a bounded sample (the first two restart
cycles), projected to a full solve with the reference's restart count for this workload.
With --gpus N > 1 (torchrun), each rank solves the same workload on its own GPU (the
eigensolver does not shard: replicas only); timings are the max over ranks.
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


def reference_arm(args, world, rank):
    """The reference's OpenMP path on the host cores (rank 0 only)."""
    if rank != 0:
        return
    from oracle import oracle as O
    from trl_b200 import problems as P

    if not O.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference checkout at build time)"}))
        return
    ref = load_reference_counts()
    A = P.anisotropic3d(CFG["grid"], coef=CFG["coef"])
    X0 = P.initial_block(A.n, CFG["bs"], seed=CFG["seed"])
    per_restart = []
    for i in range(args.warmup + args.steps):
        s = cpu_restart_sample(O, A, X0)
        if i >= args.warmup:
            per_restart.append(s["per_restart"])
    t_restart = statistics.mean(per_restart)
    value = t_restart * ref["restarts"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": "host OpenMP", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": O.num_threads(), "kind": "reference",
                         "sample": f"first 2 restart cycles of the reference BlockLanczos (ModifiedGS, CholQR) per step; steady-state restart "
                                   f"{t_restart:.3f} s x {ref['restarts']} restarts (the reference's count for this workload, "
                                   f"tests/golden/cfg2_reference.json)"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def load_reference_counts() -> dict:
    path = os.path.join(ROOT, "tests", "golden", "cfg2_reference.json")
    with open(path) as f:
        return json.load(f)


def cpu_restart_sample(O, A, X0) -> dict:
    """Times 1 and 2 restart cycles of the oracle; the difference is one steady-state cycle."""
    r1 = O.solve_csr(A, CFG["bs"], CFG["nev"], CFG["ncv"], X0, tol=CFG["tol"], max_restarts=1)
    r2 = O.solve_csr(A, CFG["bs"], CFG["nev"], CFG["ncv"], X0, tol=CFG["tol"], max_restarts=2)
    return {"first": r1["seconds"], "two": r2["seconds"], "per_restart": max(r2["seconds"] - r1["seconds"], 1e-9)}


def trl_arm(args, world, rank, local):
    import torch
    import torch.distributed as dist

    from trl_b200 import native
    from trl_b200 import problems as P

    torch.cuda.set_device(local)
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

    bs, nev, ncv, tol = CFG["bs"], CFG["nev"], CFG["ncv"], CFG["tol"]
    A = P.anisotropic3d(CFG["grid"], coef=CFG["coef"])
    exact = P.anisotropic3d_eigenvalues(CFG["grid"], coef=CFG["coef"], k=nev)
    X0 = P.initial_block(A.n, bs, seed=CFG["seed"])
    h = native.Handle(local)
    A64 = native.DeviceCSRTensors.from_host(A, torch.float64)
    A32 = native.DeviceCSRTensors.from_host(A, torch.float32)
    X0d = torch.from_numpy(X0).cuda()
    evecs = torch.empty((A.n, nev), dtype=torch.float64, device="cuda")
    common = dict(bs=bs, nev=nev, ncv=ncv, tol=tol, max_restarts=2000, refine_max_restarts=2000, fp32_tol=args.fp32_tol, want_vectors=1)

    def solve(mode, **kw):
        return native.solve_csr_device(h, A64, A32, X0d, evecs=evecs, mode=mode, **dict(common, **kw))

    def timed(mode, steps, profile=False, **kw):
        barrier()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if profile:
            h.profile(True)
        launches0 = h.launches()
        outs = []
        start.record()
        for _ in range(steps):
            outs.append(solve(mode, **kw))
        end.record()
        torch.cuda.synchronize()
        prof = h.profile_read() if profile else None
        if profile:
            h.profile(False)
        barrier()
        ms = start.elapsed_time(end) / steps
        return max_over_ranks(ms), outs, prof, h.launches() - launches0

    for _ in range(args.warmup):
        solve(native.TRL_MODE_FP64)
    for _ in range(args.warmup):
        solve(native.TRL_MODE_MIXED)
    # the timed solves run with the per-class profiler off (its events would add to the time)
    clocks = ClockSampler(local)
    clocks.start()
    ms64, outs64, _, launches = timed(native.TRL_MODE_FP64, args.steps)
    msmx, outsmx, _, _ = timed(native.TRL_MODE_MIXED, args.steps)
    clk = clocks.stop()
    o64, omx = outs64[-1], outsmx[-1]
    # one further FP64 solve of the timed configuration with the profiler on: kernel breakdown
    # and roofline (the profiler's events would add to the timed solves' time)
    _, _, prof, _ = timed(native.TRL_MODE_FP64, 1, profile=True)
    # the FP64 solve with the full reorthogonalisation, timed (one solve)
    msfull, outsfull, _, _ = timed(native.TRL_MODE_FP64, 1, reorth=native.TRL_REORTH_CGS_IFNEEDED)
    ofull = outsfull[-1]
    # the mixed mode with the BlockLanczos refinement instead of the Chebyshev one (one solve)
    mslz, outslz, _, _ = timed(native.TRL_MODE_MIXED, 1, refine=native.TRL_REFINE_LANCZOS)
    olz = outslz[-1]

    # ---- e2e: host buffers through trl_solve_csr_host, H2D/D2H inside the timed region ----
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    Ah = P.CSRMatrix(A.n, pin(A.rowptr), pin(A.colind), pin(A.values))
    X0h = pin(X0)
    # the eigenvectors land in one page-locked buffer, reused by every call
    evecs_h = pin(np.zeros((A.n, CFG["nev"])))
    e2e_times, e2e = [], None
    e2e_clocks = ClockSampler(local)
    e2e_clocks.start()
    for i in range(1 + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e = native.solve_csr_host(Ah, X0h, device=local, evecs_out=evecs_h, **dict(common, mode=native.TRL_MODE_FP64))
        torch.cuda.synchronize()
        if i > 0:
            e2e_times.append(time.perf_counter() - t0)
    e2e_clk = e2e_clocks.stop()
    e2e_s = max_over_ranks(statistics.mean(e2e_times))
    e2e_device_s = e2e["seconds"]  # device time of the last call's solve (its copies excluded)

    # ---- roofline of the dominant kernel class (live, over the profiled FP64 solve) ----
    hbm, bf16, src = peaks()
    kern = breakdown(prof)
    # the same breakdown for an FP32-mode solve to the mixed mode's FP32 tolerance
    h.profile(True)
    solve32 = native.solve_csr_device(h, A64, A32, X0d, evecs=evecs, mode=native.TRL_MODE_FP32, **dict(common, tol=args.fp32_tol))
    kern32 = breakdown(h.profile_read())
    h.profile(False)
    # the dominant streaming class: the projected eigensolver (one 8-CTA cluster, bound by
    # per-step latency) has no HBM roofline, reorth_pass2 runs behind a device flag (its bytes
    # are not credited per call), block_ops are bs x bs matrices
    not_hbm = ("small_eigen", "reorth_pass2", "block_ops")
    dominant = max((k for k in kern if k not in not_hbm and kern[k]["bytes_per_call"] > 0), key=lambda k: kern[k]["seconds"])
    d = kern[dominant]
    # achieved = algorithmic bytes per call / mean call duration (CUDA events on the solver's
    # stream around every call of the class during the profiled solve)
    achieved = d["bytes_per_call"] / (d["seconds"] / d["calls"]) / 1e9
    traffic = load_traffic(dominant, d["bytes_per_call"])
    roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "algorithmic_bytes_per_call": d["bytes_per_call"], "peak_source": src,
                "share_of_profiled_solve": d["share"],
                "not_hbm_classes": {k: round(kern[k]["share"], 4) for k in not_hbm if k in kern}}
    spmm = kern.get("spmm", {})

    result = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(A, X0, o64["restarts"])
        err64 = float(np.max(np.abs(o64["evals"] - exact) / exact))
        errmx = float(np.max(np.abs(omx["evals"] - exact) / exact))
        result = {
            "metric": METRIC, "value": ms64 / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms64, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "mode": "fp64",
                       "reorth": "partial: block classical Gram-Schmidt (DGKS second pass) at the steps where a random sketch of the basis shows orthogonality loss > 1e-12",
                       "orthonormalize": "CholQR2",
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (basis 2.8 GB, CSR 113 MB, per-step working set >> 126 MB)"},
            "fp64": {"seconds": ms64 / 1e3, "restarts": o64["restarts"], "n_op_apply": o64["n_op_apply"], "converged": bool(o64["converged"]),
                     "max_rel_residual": o64["max_rel_residual"], "max_rel_err_vs_analytic": err64},
            "mixed": {"seconds": msmx / 1e3, "speedup_vs_fp64": ms64 / msmx,
                      "refine": "Chebyshev-filtered subspace iteration + Rayleigh-Ritz on nev/bs+2 blocks (FP32 filter rounds, then FP64)",
                      "restarts_fp32": omx["restarts_fp32"], "n_op_apply_fp32": omx["n_op_apply_fp32"], "seconds_fp32_phase": omx["seconds_fp32"],
                      "refine_rounds": omx["refine_rounds"], "refine_degree": omx["refine_degree"],
                      "refine_degree_fp32": omx["refine_degree_fp32"], "fp32_tol": args.fp32_tol,
                      "converged": bool(omx["converged"]), "max_rel_residual": omx["max_rel_residual"], "max_theta_residual": omx["max_theta_residual"],
                      "max_rel_err_vs_analytic": errmx},
            "fp64_full_reorth": {"seconds": msfull / 1e3, "restarts": ofull["restarts"], "converged": bool(ofull["converged"]),
                                 "max_rel_residual": ofull["max_rel_residual"],
                                 "max_rel_err_vs_analytic": float(np.max(np.abs(ofull["evals"] - exact) / exact))},
            "mixed_lanczos_refine": {"seconds": mslz / 1e3, "speedup_vs_fp64": ms64 / mslz, "restarts_fp32": olz["restarts_fp32"],
                                     "restarts_fp64": olz["restarts"], "converged": bool(olz["converged"]), "max_rel_residual": olz["max_rel_residual"],
                                     "max_rel_err_vs_analytic": float(np.max(np.abs(olz["evals"] - exact) / exact))},
            "spmm": {"gbs": spmm.get("gbs"), "frac_of_hbm": (spmm.get("gbs") or 0) / hbm, "calls": spmm.get("calls"),
                     "bytes_per_call": 6137856 * 12 + 4 * 884737 + 2 * 884736 * 8 * 8},
            "kernels": kern,
            "kernels_fp32": {"restarts": solve32["restarts"], "seconds": solve32["seconds"], "classes": kern32},
            "roofline": roofline,
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(e2e["h2d_bytes"]), "d2h_bytes_per_step": int(e2e["d2h_bytes"]),
                    "api": "trl_solve_csr_host (pinned host CSR + start block in, eigenvalues + eigenvectors out into a pinned buffer)",
                    "steps_s": e2e_times, "device_s_last": e2e_device_s, "clocks": e2e_clk},
            "gpu_launches": launches // max(1, args.steps) * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(result), flush=True)
    h.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


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
    capture of the same kernel on a smaller case) times this run's algorithmic bytes per call."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            r = json.load(f).get(kernel)
        return None if r is None else r["traffic_per_algorithmic"] * algorithmic_bytes_per_call
    except Exception:
        return None


def cpu_baseline(A, X0, restarts_gpu: int):
    try:
        from oracle import oracle as O
    except Exception as e:  # pragma: no cover
        return {"value": None, "unavailable": str(e)}
    if not O.available():
        return {"value": None, "unavailable": "oracle/_ref not built"}
    s = cpu_restart_sample(O, A, X0)
    try:
        restarts_ref = load_reference_counts()["restarts"]
    except Exception:
        restarts_ref = restarts_gpu
    return {"value": s["per_restart"] * restarts_ref, "unit": "s", "cores": O.num_threads(), "kind": "reference",
            "sample": f"reference OpenMP BlockLanczos (ModifiedGS, CholQR) on the same workload: 1 and 2 restart cycles timed "
                      f"({s['first']:.2f} s, {s['two']:.2f} s); steady-state cycle {s['per_restart']:.3f} s x {restarts_ref} restarts "
                      f"(the reference's restart count for this workload)"}


def profile_case(args):
    """Runs one piece of the workload for profiler captures (without timing output, except
    spmm-zipf, which prints one JSON line of throughput per block size and precision):
    solve   one FP64 solve capped at --restarts restart cycles (launch lists);
    mixed   one complete mixed-mode solve (FP32 phase, FP32 and FP64 filter rounds, residuals);
    spmm-zipf  SpMM throughput on the 4M-row Zipf operator, block sizes 4/8/16, FP64 and FP32;
    spmm    the operator apply on the full workload (CSR 113 MB, X and Y 57 MB each);
    dot / update   one multi-block inner product / projection update against --nblk
            basis blocks of the workload (n x 8 FP64 each);
    project one Gram-Schmidt pass as the solver issues it (dot + update with the Gram of
            the result) against --nblk basis blocks;
    rotate  the thick-restart rotation V (48 blocks) x Y -> 5 blocks.
    Every case reads and writes more than the 126 MB L2 and holds at most ~3 GB."""
    import torch

    from trl_b200 import native
    from trl_b200 import problems as P

    bs = CFG["bs"]
    dt = torch.float32 if args.fp32 else torch.float64
    A = P.anisotropic3d(CFG["grid"], coef=CFG["coef"])
    h = native.Handle(0)
    if args.case == "solve":
        A64 = native.DeviceCSRTensors.from_host(A)
        A32 = native.DeviceCSRTensors.from_host(A, torch.float32)
        X0 = torch.from_numpy(P.initial_block(A.n, bs, seed=CFG["seed"])).cuda()
        mode = native.TRL_MODE_FP32 if args.fp32 else native.TRL_MODE_FP64
        native.solve_csr_device(h, A64, A32, X0, bs=bs, nev=CFG["nev"], ncv=CFG["ncv"], tol=CFG["tol"], mode=mode, max_restarts=args.restarts, want_vectors=0)
    elif args.case == "mixed":
        A64 = native.DeviceCSRTensors.from_host(A)
        A32 = native.DeviceCSRTensors.from_host(A, torch.float32)
        X0 = torch.from_numpy(P.initial_block(A.n, bs, seed=CFG["seed"])).cuda()
        native.solve_csr_device(h, A64, A32, X0, bs=bs, nev=CFG["nev"], ncv=CFG["ncv"], tol=CFG["tol"], mode=native.TRL_MODE_MIXED, fp32_tol=args.fp32_tol,
                                max_restarts=2000, refine_max_restarts=2000, want_vectors=1)
    elif args.case == "spmm-zipf":
        # the bandwidth-stress operator: n = 4,194,304, Zipf(1.5) out-degrees capped at 512,
        # mirrored (about 145M entries); SpMM throughput per block size and precision, each
        # timed launch behind an L2 flush
        hbm, _, src = peaks()
        Z = P.zipf_symmetric(4_194_304, cap=512, seed=42)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        for dt, name in ((torch.float64, "f64"), (torch.float32, "f32")):
            Zd = native.DeviceCSRTensors.from_host(Z, dt)
            es = 8 if dt == torch.float64 else 4
            for b in (4, 8, 16):
                X = torch.randn(Z.n, b, dtype=dt, device="cuda")
                Y = torch.empty_like(X)
                for _ in range(3):
                    h.spmm(Zd, X, Y)
                times = []
                for _ in range(max(args.reps, 5)):
                    flush.fill_(1)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    h.spmm(Zd, X, Y)
                    e1.record()
                    torch.cuda.synchronize()
                    times.append(e0.elapsed_time(e1) / 1e3)
                t = statistics.median(times)
                nbytes = Z.nnz * (es + 4) + 4 * (Z.n + 1) + 2 * Z.n * b * es
                print(json.dumps({"case": "spmm-zipf", "dtype": name, "bs": b, "n": Z.n, "nnz": int(Z.nnz), "us": t * 1e6, "gbs": nbytes / t / 1e9,
                                  "frac_of_hbm": nbytes / t / 1e9 / hbm, "peak_source": src}), flush=True)
                del X, Y
            del Zd
    elif args.case == "spmm":
        Ad = native.DeviceCSRTensors.from_host(A, dt)
        X = torch.randn(A.n, bs, dtype=dt, device="cuda")
        Y = torch.empty_like(X)
        for _ in range(args.reps):
            h.spmm(Ad, X, Y)
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
    ap.add_argument("--case", choices=["solve", "mixed", "spmm", "spmm-zipf", "dot", "update", "project", "rotate"], default=None,
                    help="profiling driver: run one piece of the workload and exit (see profile_case)")
    ap.add_argument("--restarts", type=int, default=3)
    ap.add_argument("--nblk", type=int, default=24)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--fp32", action="store_true")
    args = ap.parse_args()
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
