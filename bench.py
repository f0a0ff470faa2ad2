#!/usr/bin/env python
"""Signature-kernel throughput benchmark on B200.

Default workload (the headline configuration): SigPDE.gram(x, y) with the
linear static kernel, X and Y each 256 Brownian paths of length 128 in 8
dimensions, dyadic order 2, float32 inputs, float64 PDE cells (the default,
"accurate" precision).  One step = one full 256x256 Gram = 65,536 entries =
1.69e10 refined-grid cell updates.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32]
    python bench.py --impl reference ...   # the float64 CPU oracle (C/OpenMP) on the host cores

Multi-GPU (one process per GPU, launched by torchrun): every rank solves its
own Gram (weak scaling, replicas: the entries are independent and no data
crosses GPUs); `value` = all ranks' entries / the slowest rank's time.
Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOADS = {
    # SigPDE.gram(x, y), LinearKernel, X,Y 256 Brownian paths, L=128, d=8, dyadic order 2
    "gram256": dict(nx=256, ny=256, L=128, d=8, order=2, seed_x=2001, seed_y=2002),
    # SigPDE pairwise over 4096 (x, y) pairs, lengths uniform in [16, 512] per path, d=32,
    # dyadic order uniform in {0, 1, 2, 3} per pair, Brownian N(0, 1/(L-1)) increments
    # RobustSigPDE.gram(x) (normalisation + symmetric Gram), default normaliser, N=512 Brownian paths
    # scaled by a per-path factor log-uniform in [0.5, 4], L=64, d=16, dyadic order 1
    "robust512": dict(kind="robust", n=512, L=64, d=16, order=1, seed=512, smin=0.5, smax=4.0),
    # Serving stream: Poisson arrivals (mean 200 req/s) of Gram requests, N log-uniform in [8, 1024],
    # L log-uniform in [32, 1024], d in {2, 8, 32}, order in {0, 1, 2}, 30% RobustSigPDE (default
    # normaliser), float32 Brownian paths; run as a finite trace of `requests` requests
    "serve": dict(kind="serve", requests=120, rate=200.0, nmin=8, nmax=1024, lmin=32, lmax=1024, dims=(2, 8, 32),
                  orders=(0, 1, 2), robust=0.3, seed=5),
    # the same stream with N and L capped at 256 (service-sized requests)
    "serve_light": dict(kind="serve", requests=400, rate=200.0, nmin=8, nmax=256, lmin=32, lmax=256, dims=(2, 8, 32),
                        orders=(0, 1, 2), robust=0.3, seed=6),
    # SigPDE.gram(x, y) with RBFKernel(sigma=1): the gram256 paths and shape, static kernel evaluated on
    # the device from the points
    "rbf256": dict(kind="static", nx=256, ny=256, L=128, d=8, order=2, seed_x=2001, seed_y=2002, static="rbf",
                   sigma=1.0),
    # forward + backward of sum(SigPDE.gram(x, y)) with LinearKernel: X, Y 128 Brownian paths, L=128, d=8,
    # dyadic order 2 (gradients with respect to both sides' points)
    "grad128": dict(kind="grad", nx=128, ny=128, L=128, d=8, order=2, seed_x=2001, seed_y=2002),
    "uneven4096": dict(kind="ragged", npairs=4096, lmin=16, lmax=512, d=32, orders=(0, 1, 2, 3), seed=4096),
}

L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"],
                    help="ours | reference: the float64 oracle port on the host cores | reference-gpu: the "
                         "unmodified stojl/SigPDE Numba GPU path installed under baseline/_ref")
    ap.add_argument("--workload", default="gram256", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "tc32", "tc64"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target length of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: the ranks solve row blocks of ONE Gram and all-gather them (strong scaling, "
                         "sigpde_b200.distributed) instead of one replica each")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="skip the short runs of robust512, uneven4096 and serve_light after the default Gram")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's Numba GPU path beside the default Gram")
    ap.add_argument("--autotune", action="store_true", help="uneven batches: measure rows per lane per bucket "
                    "before timing (sigpde_b200.torch.autotune)")
    ap.add_argument("--resident", action="store_true",
                    help="serving traces: requests draw their paths from a pool of 40 path sets kept resident on "
                         "the device (GramServer.put); the per-request baseline copies them from the host")
    ap.add_argument("--burst", action="store_true", help="serving traces: every request arrives at t=0 "
                    "(saturated throughput) instead of Poisson arrivals")
    return ap.parse_args()


# ----------------------------------------------------------------------------- workload
def workload_units(w):
    n = (w["L"] - 1) << w["order"]
    entries = w["nx"] * w["ny"]
    cells = entries * n * n
    coarse = entries * (w["L"] - 1) ** 2
    # algorithmic FLOPs: 4 per refined cell ((a+b)*A - c*B), 2d + 8 per coarse cell
    # (the increment dot product and the stencil coefficients)
    flops = 4 * cells + (2 * w["d"] + 8) * coarse
    return entries, cells, flops


def workload_name(w):
    kern = {"linear": "LinearKernel", "rbf": f"RBFKernel(sigma={w.get('sigma')})",
            "l1rbf": f"L1RBFKernel(sigma={w.get('sigma')})"}[w.get("static", "linear")]
    return f"SigPDE.gram {w['nx']}x{w['ny']}, L={w['L']}, d={w['d']}, dyadic_order={w['order']}, {kern}"


def issue_roofline(w, precision, ms, gemm_tflops):
    """The wavefront's arithmetic pipe in instructions rather than FLOPs.

    A refined cell is 3 instructions of the cell type (float64: add, mul, fma;
    the stencil's add and mul each take a full issue slot but count as one FLOP),
    and a coarse cell adds 4 for its coefficients plus d fmas for its increment
    when the CUDA cores form it (fp64 / fp32; tc32 / tc64 take it from the tensor
    cores).  float32 cells take 5 instructions a cell (the one-rounding form).
    The ceiling is the pipe's measured fma rate: the in-run cuBLAS GEMM's FLOP/s
    over 2, so a kernel that kept the pipe busy with useful instructions would
    read 1.0."""
    entries, cells, _ = workload_units(w)
    coarse = entries * (w["L"] - 1) ** 2
    per_cell = 3 if precision in ("fp64", "tc64") else 5
    per_coarse = 4 + (w["d"] if precision in ("fp64", "fp32") else 0)
    instr = per_cell * cells + per_coarse * coarse
    achieved = instr / (ms * 1e-3) / 1e12
    peak = gemm_tflops / 2
    return {"unit": "T instructions/s", "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "instructions_per_launch": instr,
            "note": "same time and GEMM as frac above, counted in pipe instructions (ncu's FP64-pipe activity "
                    "reads the same quantity)"}


def other_workloads(args):
    """Short runs of the other benchmark configurations, after (outside) the
    default Gram's timed region, so that one bench line records them too: the
    robust Gram (robust512), the uneven batch (uneven4096) and the serving trace
    (serve_light, burst arrivals: served stream against per-request plain
    launches; the median of three runs).  Each runner prints its own line; the
    figures kept here are its times, with 5 timed steps after 3 warm-ups and no
    CPU baselines."""
    import argparse
    import contextlib
    import io

    def run(fn, workload, **over):
        a = argparse.Namespace(**vars(args))
        a.steps, a.warmup, a.no_cpu_baseline, a.autotune, a.burst = 5, 3, True, False, False
        for k, v in over.items():
            setattr(a, k, v)
        buf = io.StringIO()
        try:
            with contextlib.redirect_stdout(buf):
                fn(a, WORKLOADS[workload])
            return json.loads([l for l in buf.getvalue().splitlines() if l.startswith("{")][-1])
        except Exception as e:  # a failed side run must not lose the headline line
            return {"error": f"{type(e).__name__}: {e}"[:200]}

    out = {"note": "5 timed steps after 3 warm-ups each, measured after the headline's timed region"}
    for prec in ("fp64", "tc64"):
        r = run(run_ours_robust, "robust512", precision=prec)
        out[f"robust512_{prec}"] = {k: r.get(k) for k in ("ms_per_step", "value", "unit", "phases_ms", "error")
                                    if k in r}
        r = run(run_ours_ragged, "uneven4096", precision=prec)
        out[f"uneven4096_{prec}"] = {k: r.get(k) for k in ("ms_per_step", "value", "unit", "error") if k in r}
    # the served stream is a host-side Python loop, so one short run moves with the host's load:
    # three runs, the one of median ratio reported, all three ratios listed
    runs = [run(run_serve, "serve_light", precision="tc64", burst=True) for _ in range(3)]
    ok = [x for x in runs if "error" not in x]
    r = sorted(ok, key=lambda x: x["throughput_ratio_vs_plain"])[len(ok) // 2] if ok else runs[0]
    out["serve_light_tc64_burst"] = {
        "runs": 3, "ratios_of_the_runs": [round(x["throughput_ratio_vs_plain"], 3) if "throughput_ratio_vs_plain" in x
                               else None for x in runs],
        "served_requests_per_s": r.get("served", {}).get("requests_per_s"),
        "plain_requests_per_s": r.get("per_request_plain_launches", {}).get("requests_per_s"),
        "throughput_ratio_vs_plain": r.get("throughput_ratio_vs_plain"),
        "served_p50_p99_ms": [r.get("served", {}).get("p50_ms"), r.get("served", {}).get("p99_ms")],
        "plain_p50_p99_ms": [r.get("per_request_plain_launches", {}).get("p50_ms"),
                             r.get("per_request_plain_launches", {}).get("p99_ms")],
        "results_identical_alone_and_in_mix": r.get("results_identical_alone_and_in_mix"),
        **({"error": r["error"]} if "error" in r else {})}
    return out


def gram_config(w, world, precision):
    """The `config` of a Gram workload's bench line, shared by every arm so that
    the GPU line and the reference line describe the same workload."""
    entries, _, _ = workload_units(w)
    return {"workload": workload_name(w), "global_batch": entries * world, "seq_len": w["L"],
            "parallelism": f"replicas x{world}", "precision": precision,
            "l2": "GPU arm: flushed between timed steps (256 MB write); CPU arm: host memory"}


def static_kernel_of(kernels, w):
    st = w.get("static", "linear")
    if st == "rbf":
        return kernels.RBFKernel(w["sigma"])
    if st == "l1rbf":
        return kernels.L1RBFKernel(w["sigma"])
    return kernels.LinearKernel()


def make_inputs(w, device=None, dtype=None):
    from sigpde_b200 import synthetic
    x = synthetic.brownian(w["nx"], w["L"], w["d"], w["seed_x"], dtype=dtype, device=device)
    y = synthetic.brownian(w["ny"], w["L"], w["d"], w["seed_y"], dtype=dtype, device=device)
    return x, y


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, power and clock-event reasons sampled during the timed region.

    NVML is polled from a thread every `period_s` (20 ms: a config-2 run of 20
    steps lasts ~0.1 s, which a 200 ms nvidia-smi loop sees once).  Reading NVML
    changes no GPU setting.  Without NVML the sampler falls back to nvidia-smi.
    """

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))

    def __init__(self, gpu_index, period_s=0.02):
        self.gpu_index = gpu_index
        self.period_s = period_s
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []
        self.stop_evt = threading.Event()
        self.nvml = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        idx = self.gpu_index
        try:  # CUDA_VISIBLE_DEVICES may renumber devices; torch knows the NVML index
            idx = torch.cuda._get_nvml_device_index(self.gpu_index)
        except Exception:
            pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _poll(self):
        nv, h = self.nvml
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop_evt.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.rows.append((sm, mx, pw, reasons))
            except Exception:
                pass
            self.stop_evt.wait(self.period_s)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_evt.set()
            self.thread.join(timeout=5)
            rows = self.rows
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
            reasons = set()
            for r in rows:
                for name, bit in self.REASON_BITS:
                    if r[3] & bit:
                        reasons.add(name)
            return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                    "reasons": sorted(reasons), "samples": len(rows), "power_w_max": max(r[2] for r in rows),
                    "source": f"nvml every {int(self.period_s * 1000)} ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows), "source": "nvidia-smi every 50 ms"}


# ----------------------------------------------------------------------------- timing
def device_peak_tflops(torch, dtype, n=4096, reps=5):
    """Measured dense GEMM rate for `dtype` (cuBLAS through torch.matmul); the
    float64 figure is the denominator of the float64 wavefront's roofline."""
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = math.inf
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b)
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e))
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


LAUNCHES = {"last": None}  # libsigk kernels enqueued by the last timed region


def _launch_count():
    mod = sys.modules.get("sigpde_b200._lib")
    return mod.launch_count() if mod is not None else None


def timed_steps(torch, step, K, W, flush_buf, barrier):
    for _ in range(W):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    evs = []
    c0 = _launch_count()
    for _ in range(K):
        flush_buf.zero_()  # L2 flush between timed steps (outside the events)
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        step()
        e.record(stream)
        evs.append((s, e))
    c1 = _launch_count()
    LAUNCHES["last"] = None if c0 is None else c1 - c0
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in evs]


def max_over_ranks(torch, dist, world, value, device=None):
    """The largest of every rank's `value` (every rank calls this, in the same order)."""
    if world <= 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, steps, slowest_ms):
    """Whole-job throughput of weak-scaled replicas: every rank's units over the slowest rank's time."""
    return world * units_per_rank * steps / (slowest_ms * 1e-3)


def percentile(v, q):
    v = sorted(v)
    if not v:
        return None
    k = (len(v) - 1) * q
    f, c = math.floor(k), math.ceil(k)
    return v[f] + (v[c] - v[f]) * (k - f)


def read_traffic(kernel_key):
    """Per-launch DRAM bytes from the committed ncu summary (profiles/traffic.txt)."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        line = line.strip()
        if line.startswith(kernel_key + "="):
            try:
                return float(line.split("=", 1)[1].split("#")[0].split()[0])
            except ValueError:
                return None
    return None


# ----------------------------------------------------------------------------- CPU legs
def cpu_oracle_rate(w, target_s, seed=7, max_entries=None):
    """Float64 oracle (C, OpenMP over entries, all host threads) on a sample of
    the Gram's entries; returns (entries/s, cores, sample description)."""
    import numpy as np

    from oracle import oracle
    from sigpde_b200 import synthetic
    oracle.build()
    x = synthetic.brownian_np(w["nx"], w["L"], w["d"], w["seed_x"]).astype(np.float32).astype(np.float64)
    y = synthetic.brownian_np(w["ny"], w["L"], w["d"], w["seed_y"]).astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(seed)
    cores = oracle.num_threads()
    n = max(cores, 8)
    while True:
        flat = rng.choice(w["nx"] * w["ny"], n, replace=False)
        t0 = time.perf_counter()
        oracle.gram(x, y, w["order"], pairs=flat, static=w.get("static", "linear"), static_param=w.get("sigma", 1.0))
        dt = time.perf_counter() - t0
        if dt >= target_s or n >= w["nx"] * w["ny"] or (max_entries and n >= max_entries):
            break
        n = min(w["nx"] * w["ny"], max(n * 2, int(n * target_s / max(dt, 1e-3) * 1.1)))
        if max_entries:
            n = min(n, max_entries)
    return n / dt, cores, f"{n} random entries of the {w['nx']}x{w['ny']} Gram in {dt:.1f} s"


def run_reference(args, w, rank):
    if rank != 0:
        return
    entries, cells, _ = workload_units(w)
    per_step = []
    cores = None
    sample = None
    step_s = max(1.0, args.cpu_seconds / 2)
    for i in range(args.warmup + args.steps):
        rate, cores, sample = cpu_oracle_rate(w, step_s, seed=100 + i)
        if i >= args.warmup:
            per_step.append(rate)
    value = statistics.mean(per_step)
    line = {
        "impl": "reference",
        "metric": "gram_entries_per_s",
        "value": value,
        "unit": "entries/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": entries / value * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic Brownian paths (seeded), float32 inputs upcast to float64",
        "config": gram_config(w, args.gpus, "fp64"),
        "cells_per_s": value * cells / entries,
        "cpu_baseline": {"value": value, "unit": "entries/s", "cores": cores, "kind": "port",
                         "sample": f"per step: {sample}; float64 C restatement of the reference solver"},
        "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- our arm
def run_ours(args, w):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    import sigpde_b200.torch as sig
    from sigpde_b200 import _lib

    entries, cells, flops = workload_units(w)
    X, Y = make_inputs(w, device=dev)
    k = sig.SigPDE(sig.kernels.LinearKernel(), w["order"], precision=args.precision)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    shard = args.shard and world > 1
    if shard:  # one Gram, its rows split over the ranks and all-gathered (NCCL)
        from sigpde_b200 import distributed as D

        def gram(a, b):
            return D.sharded_gram(a, b, static_kernel=sig.kernels.LinearKernel(), dyadic_order=w["order"],
                                  precision=args.precision)
    else:
        gram = k.gram
    out = gram(X, Y)  # also loads libsigk.so
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    times = timed_steps(torch, lambda: gram(X, Y), args.steps, args.warmup, flush, barrier)
    launches = LAUNCHES["last"]
    clk = clocks.stop()
    total_ms = max_over_ranks(torch, dist, world, sum(times), dev)
    value = job_rate(1 if shard else world, entries, args.steps, total_ms)

    # end to end through the public API: pinned host paths -> device -> Gram -> pinned host result
    Xh = X.cpu().pin_memory()
    Yh = Y.cpu().pin_memory()
    Rh = torch.empty((w["nx"], w["ny"]), dtype=X.dtype).pin_memory()

    def e2e_step():
        Xd = Xh.to(dev, non_blocking=True)
        Yd = Yh.to(dev, non_blocking=True)
        Rh.copy_(gram(Xd, Yd), non_blocking=True)

    e2e_times = timed_steps(torch, e2e_step, args.steps, args.warmup, flush, barrier)
    e2e_ms = max_over_ranks(torch, dist, world, sum(e2e_times), dev)
    e2e_value = job_rate(1 if shard else world, entries, args.steps, e2e_ms)

    line = None
    if rank == 0:
        ms = statistics.mean(times)
        fp64 = args.precision in ("fp64", "tc64")  # float64 cells
        peak = device_peak_tflops(torch, torch.float64 if fp64 else torch.float32)
        achieved = flops / (ms * 1e-3) / 1e12
        traffic = read_traffic(f"gram256_{args.precision}")
        # accuracy of this run on a sample of entries against the float64 oracle
        acc = None
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            from oracle import oracle
            G = out.double().cpu().numpy()
            rng = np.random.default_rng(1)
            flat = rng.choice(entries, 64, replace=False)
            xin, yin = X.double().cpu().numpy(), Y.double().cpu().numpy()
            want = oracle.gram(xin, yin, w["order"], pairs=flat)
            got = G.reshape(-1)[flat]
            kxx = oracle.pairwise(xin[flat // w["ny"]], None, w["order"])
            kyy = oracle.pairwise(yin[flat % w["ny"]], None, w["order"])
            acc = {"max_rel_err": float(np.max(np.abs(got - want) / np.abs(want))),
                   "max_cs_err": float(np.max(np.abs(got - want) / np.sqrt(kxx * kyy))),
                   "sample": "64 random entries vs the float64 oracle"}
            # the other precision modes on the same inputs and sample: time and error
            modes = {}
            for prec in ("fp64", "fp32", "tc32", "tc64"):
                if prec == args.precision:
                    continue
                km = sig.SigPDE(sig.kernels.LinearKernel(), w["order"], precision=prec)
                tm = timed_steps(torch, lambda: km.gram(X, Y), args.steps, args.warmup, flush, lambda: None)
                gm = km.gram(X, Y).double().cpu().numpy().reshape(-1)[flat]
                modes[prec] = {"ms_per_step": statistics.mean(tm),
                               "entries_per_s": entries / (statistics.mean(tm) * 1e-3),
                               "max_rel_err": float(np.max(np.abs(gm - want) / np.abs(want))),
                               "max_cs_err": float(np.max(np.abs(gm - want) / np.sqrt(kxx * kyy)))}
            acc["other_precision_modes"] = modes
            rate, cores, sample = cpu_oracle_rate(w, args.cpu_seconds)
            cpu = {"value": rate, "unit": "entries/s", "cores": cores, "kind": "port",
                   "sample": f"{sample}; float64 C restatement of the reference solver (OpenMP)"}
        line = {
            "metric": "gram_entries_per_s",
            "value": value,
            "unit": "entries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "p50_ms": percentile(times, 0.5),
            "p99_ms": percentile(times, 0.99),
            "higher_is_better": True,
            "scaling": "strong" if shard else "weak",
            "vs_baseline": None,
            "dtype": "f64" if fp64 else "f32",
            "data": "synthetic Brownian paths (seeded PCG64), float32",
            "config": (dict(gram_config(w, 1, args.precision), parallelism=f"Gram rows sharded x{world}")
                       if shard else gram_config(w, world, args.precision)),
            "cells_per_s": value * cells / entries,
            "accuracy": acc,
            "roofline": {"bound": "fp64" if fp64 else "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                         "issue": issue_roofline(w, args.precision, ms, peak),
                         "peak_source": ("measured cuBLAS " + ("DGEMM" if fp64 else "SGEMM (no TF32)") +
                                         " 4096^3 on this device (the wavefront is bound by the "
                                         + ("FP64" if fp64 else "FP32") + " pipe, not HBM or tensor cores)"),
                         "algorithmic_flops_per_launch": flops},
            "e2e": {"value": e2e_value, "unit": "entries/s", "h2d_bytes_per_step": X.numel() * X.element_size()
                    + Y.numel() * Y.element_size(), "d2h_bytes_per_step": Rh.numel() * Rh.element_size(),
                    "ms_per_step": statistics.mean(e2e_times)},
            "gpu_launches": launches,
            "clocks": clk,
            "lib": _lib.version(),
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if world == 1 and not args.no_other_workloads:
            line["other_workloads"] = other_workloads(args)
        if world == 1 and not args.no_reference_gpu:
            # the reference's own Numba GPU path on the same inputs, timed after (outside) our timed region
            r = measure_reference_gpu(w, steps=3, warmup=2, accuracy=False)
            if "unavailable" in r:
                line["reference_numba_gpu"] = r
            else:
                line["reference_numba_gpu"] = {
                    "ms_per_step": r["ms_per_step"], "entries_per_s": r["value"], "steps": 3, "warmup": 2,
                    "speedup": value / r["value"],
                    "note": "unmodified stojl/SigPDE from baseline/_ref through sigpde.torch.SigPDE.gram on this "
                            "GPU, host-timed between synchronisations (the reference synchronises inside each "
                            "call), measured after this line's timed region"}
    if world > 1:
        barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


def run_ours_static(args, w):
    """Gram with an RBF / L1-RBF static kernel evaluated on the device from the
    points (sigk_gram_static).  Beside it, the reference's route on this
    library's solver: torch builds the float32 static Gram and its 4-term
    difference per 32x32 tile of paths, the CUDA wavefront reads them."""
    import numpy as np
    import torch
    import sigpde_b200.torch as sig
    from sigpde_b200 import _lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    entries, cells, _ = workload_units(w)
    coarse = entries * (w["L"] - 1) ** 2
    flops = 4 * cells + 8 * coarse  # the wavefront's stencil and coefficients
    X, Y = make_inputs(w, device=dev)
    k = sig.SigPDE(static_kernel_of(sig.kernels, w), w["order"], precision=args.precision)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    out = k.gram(X, Y)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    times = timed_steps(torch, lambda: k.gram(X, Y), args.steps, args.warmup, flush, lambda: None)
    launches = LAUNCHES["last"]
    clk = clocks.stop()
    kg = sig.SigPDE(static_kernel_of(sig.kernels, w), w["order"], precision=args.precision)
    kg._device_static = False
    out_g = kg.gram(X, Y)
    t_generic = timed_steps(torch, lambda: kg.gram(X, Y), max(1, args.steps // 4), 1, flush, lambda: None)
    Xh, Yh = X.cpu().pin_memory(), Y.cpu().pin_memory()
    Rh = torch.empty((w["nx"], w["ny"]), dtype=X.dtype).pin_memory()

    def e2e_step():
        Rh.copy_(k.gram(Xh.to(dev, non_blocking=True), Yh.to(dev, non_blocking=True)), non_blocking=True)

    e2e_times = timed_steps(torch, e2e_step, args.steps, args.warmup, flush, lambda: None)
    ms = statistics.mean(times)
    acc = cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle
        st = dict(static=w["static"], static_param=w["sigma"])
        rng = np.random.default_rng(1)
        flat = rng.choice(entries, 64, replace=False)
        xin, yin = X.double().cpu().numpy(), Y.double().cpu().numpy()
        want = oracle.gram(xin, yin, w["order"], pairs=flat, **st)
        kxx = oracle.pairwise(xin[flat // w["ny"]], None, w["order"], **st)
        kyy = oracle.pairwise(yin[flat % w["ny"]], None, w["order"], **st)
        acc = {}
        for name, G in (("device_static", out), ("generic_route", out_g)):
            got = G.double().cpu().numpy().reshape(-1)[flat]
            acc[name] = {"max_rel_err": float(np.max(np.abs(got - want) / np.abs(want))),
                         "max_cs_err": float(np.max(np.abs(got - want) / np.sqrt(kxx * kyy)))}
        acc["sample"] = "64 random entries vs the float64 oracle"
        rate, cores, sample = cpu_oracle_rate(w, args.cpu_seconds)
        cpu = {"value": rate, "unit": "entries/s", "cores": cores, "kind": "port",
               "sample": f"{sample}; float64 C restatement of the reference solver (OpenMP), numpy static Gram"}
    peak = device_peak_tflops(torch, torch.float64)
    achieved = flops / (ms * 1e-3) / 1e12
    line = {
        "metric": "gram_entries_per_s", "value": entries / (ms * 1e-3), "unit": "entries/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "p50_ms": percentile(times, 0.5),
        "p99_ms": percentile(times, 0.99), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic Brownian paths (seeded PCG64), float32",
        "config": {"workload": workload_name(w), "global_batch": entries, "seq_len": w["L"],
                   "parallelism": "single GPU", "precision": args.precision,
                   "l2": "flushed between timed steps (256 MB write)"},
        "cells_per_s": cells / (ms * 1e-3),
        "generic_route_ms_per_step": statistics.mean(t_generic),
        "accuracy": acc,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": None, "scope": "whole step (static-kernel increments + wavefront): the stencil's "
                     "4 FLOPs per refined cell and 8 per coarse cell over the step time",
                     "peak_source": "measured cuBLAS DGEMM 4096^3 on this device"},
        "e2e": {"value": entries / (statistics.mean(e2e_times) * 1e-3), "unit": "entries/s",
                "h2d_bytes_per_step": 2 * Xh.numel() * Xh.element_size(),
                "d2h_bytes_per_step": Rh.numel() * Rh.element_size(), "ms_per_step": statistics.mean(e2e_times)},
        "gpu_launches": launches, "clocks": clk, "lib": _lib.version(),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def run_ours_grad(args, w):
    """Forward + backward of sum(k.gram(X, Y)) (LinearKernel, float64 paths): the
    gradients with respect to every point of X and Y through sigk_backward."""
    import numpy as np
    import torch
    import sigpde_b200.torch as sig
    from sigpde_b200 import _lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    entries, cells, _ = workload_units(w)
    X0, Y0 = make_inputs(w, device=dev, dtype=torch.float64)
    X = X0.clone().requires_grad_()
    Y = Y0.clone().requires_grad_()
    k = sig.SigPDE(sig.kernels.LinearKernel(), w["order"])
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def step():
        X.grad = None
        Y.grad = None
        k.gram(X, Y).sum().backward()

    step()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    times = timed_steps(torch, step, args.steps, args.warmup, flush, lambda: None)
    launches = LAUNCHES["last"]
    clk = clocks.stop()
    t_fwd = timed_steps(torch, lambda: k.gram(X0, Y0), args.steps, args.warmup, flush, lambda: None)
    Xh, Yh = X0.cpu().pin_memory(), Y0.cpu().pin_memory()
    GXh, GYh = torch.empty_like(Xh).pin_memory(), torch.empty_like(Yh).pin_memory()

    def e2e_step():
        Xd = Xh.to(dev, non_blocking=True).requires_grad_()
        Yd = Yh.to(dev, non_blocking=True).requires_grad_()
        k.gram(Xd, Yd).sum().backward()
        GXh.copy_(Xd.grad, non_blocking=True)
        GYh.copy_(Yd.grad, non_blocking=True)

    e2e_times = timed_steps(torch, e2e_step, args.steps, args.warmup, flush, lambda: None)
    ms = statistics.mean(times)
    acc = cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle
        # the gradient of the sum over an 8 x 8 corner of the Gram, ours against the oracle's adjoint
        Xs = X0[:8].clone().requires_grad_()
        Ys = Y0[:8].clone().requires_grad_()
        k.gram(Xs, Ys).sum().backward()
        xs, ys = X0[:8].cpu().numpy(), Y0[:8].cpu().numpy()
        t0 = time.perf_counter()
        gx, gy = oracle.grad_gram(xs, ys, w["order"], np.ones((8, 8)))
        t_cpu = time.perf_counter() - t0
        scale = max(np.abs(gx).max(), np.abs(gy).max())
        acc = {"max_abs_err_rel_to_max_grad": float(max(np.abs(Xs.grad.cpu().numpy() - gx).max(),
                                                        np.abs(Ys.grad.cpu().numpy() - gy).max()) / scale),
               "sample": "gradients of the sum over the 8 x 8 corner of the Gram vs the float64 oracle's adjoint"}
        cpu = {"value": 64 / t_cpu, "unit": "entries/s", "cores": oracle.num_threads(), "kind": "port",
               "sample": f"forward + adjoint of the 64 pairs of the 8 x 8 corner in {t_cpu:.1f} s "
                         "(float64 C restatement, OpenMP over pairs)"}
    # algorithmic FLOPs: the forward stencil (4 per cell) three times (forward, recompute, adjoint)
    flops = 3 * 4 * cells
    peak = device_peak_tflops(torch, torch.float64)
    achieved = flops / (ms * 1e-3) / 1e12
    line = {
        "metric": "gram_gradient_entries_per_s", "value": entries / (ms * 1e-3), "unit": "entries/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "p50_ms": percentile(times, 0.5),
        "p99_ms": percentile(times, 0.99), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic Brownian paths (seeded PCG64), float64",
        "config": {"workload": "forward + backward of sum(SigPDE.gram(x, y)) 128x128, L=128, d=8, dyadic_order=2, "
                               "LinearKernel", "global_batch": entries, "seq_len": w["L"],
                   "parallelism": "single GPU", "l2": "flushed between timed steps (256 MB write)"},
        "forward_ms_per_step": statistics.mean(t_fwd),
        "accuracy": acc,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": None, "scope": "whole step: 4 FLOPs per refined cell for each of the forward, "
                     "the recompute and the adjoint, over the step time",
                     "peak_source": "measured cuBLAS DGEMM 4096^3 on this device"},
        "e2e": {"value": entries / (statistics.mean(e2e_times) * 1e-3), "unit": "entries/s",
                "h2d_bytes_per_step": 2 * Xh.numel() * Xh.element_size(),
                "d2h_bytes_per_step": 2 * GXh.numel() * GXh.element_size(), "ms_per_step": statistics.mean(e2e_times)},
        "gpu_launches": launches, "clocks": clk, "lib": _lib.version(),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def measure_reference_gpu(w, steps, warmup, accuracy=True):
    """Time the reference's own GPU path: stojl/SigPDE installed unmodified under
    baseline/_ref, called through its public API (sigpde.torch.SigPDE.gram with
    the default max_batch / max_threads) on the same float32 inputs.  The
    reference synchronises the device inside every call, so each call is timed
    on the host between two synchronisations; the L2 is flushed between calls.
    Returns the fields of a bench line, or {"unavailable": why}."""
    import numpy as np
    import torch

    ref_dir = os.path.join(ROOT, "baseline", "_ref")
    entries, cells, _ = workload_units(w)
    if not os.path.isdir(os.path.join(ref_dir, "sigpde")):
        return {"unavailable": "reference not installed under baseline/_ref"}
    if ref_dir not in sys.path:
        sys.path.insert(0, ref_dir)
    try:
        import warnings
        warnings.filterwarnings("ignore")
        import sigpde.torch as refsig
    except Exception as e:  # numba or its CUDA target missing
        return {"unavailable": f"import failed: {type(e).__name__}: {e}"[:300]}
    dev = torch.device("cuda", torch.cuda.current_device())
    X, Y = make_inputs(w, device=dev)
    k = refsig.SigPDE(static_kernel_of(refsig.kernels, w), w["order"])
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    try:
        out = k.gram(X, Y)
    except Exception as e:
        return {"unavailable": f"reference call failed: {type(e).__name__}: {e}"[:300]}
    for _ in range(max(0, warmup - 1)):
        k.gram(X, Y)
    times = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        k.gram(X, Y)
        torch.cuda.synchronize()
        times.append((time.perf_counter() - t0) * 1e3)
    ms = statistics.mean(times)
    acc = None
    if accuracy:
        from oracle import oracle
        G = out.double().cpu().numpy()
        rng = np.random.default_rng(1)
        flat = rng.choice(entries, 64, replace=False)
        xin, yin = X.double().cpu().numpy(), Y.double().cpu().numpy()
        st = dict(static=w.get("static", "linear"), static_param=w.get("sigma", 1.0))
        want = oracle.gram(xin, yin, w["order"], pairs=flat, **st)
        got = G.reshape(-1)[flat]
        kxx = oracle.pairwise(xin[flat // w["ny"]], None, w["order"], **st)
        kyy = oracle.pairwise(yin[flat % w["ny"]], None, w["order"], **st)
        acc = {"max_rel_err": float(np.max(np.abs(got - want) / np.abs(want))),
               "max_cs_err": float(np.max(np.abs(got - want) / np.sqrt(kxx * kyy))),
               "sample": "64 random entries vs the float64 oracle"}
    return dict(value=entries / (ms * 1e-3), steps=steps, warmup=warmup, ms_per_step=ms,
                p50_ms=percentile(times, 0.5), p99_ms=percentile(times, 0.99), cells_per_s=cells / (ms * 1e-3),
                accuracy=acc)


def run_reference_gpu(args, w):
    """The reference's Numba GPU path as its own bench line (--impl reference-gpu)."""
    entries, _, _ = workload_units(w)
    base = {"impl": "reference-gpu", "metric": "gram_entries_per_s", "unit": "entries/s"}
    r = measure_reference_gpu(w, args.steps, args.warmup, accuracy=not args.no_cpu_baseline)
    if "unavailable" in r:
        print(json.dumps(dict(base, **r)), flush=True)
        return
    line = dict(base, n_gpus=1, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32 storage / f64 arithmetic", data="synthetic Brownian paths (seeded PCG64), float32",
                config=gram_config(w, 1, "reference (float64 arithmetic, float32 storage)"),
                note="unmodified stojl/SigPDE (Numba CUDA) through sigpde.torch.SigPDE.gram, host-timed "
                     "(the reference synchronises inside each call)", **r)
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- uneven batched pairwise
def ragged_spec(w):
    """Seeded lengths and orders of the uneven workload."""
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(w["seed"]))
    lx = rng.integers(w["lmin"], w["lmax"] + 1, w["npairs"])
    ly = rng.integers(w["lmin"], w["lmax"] + 1, w["npairs"])
    orders = rng.choice(np.array(w["orders"]), w["npairs"])
    return lx.tolist(), ly.tolist(), orders.tolist()


def ragged_paths(w, lx, ly):
    """Brownian paths of the given lengths (float64 numpy), seeded per pair."""
    from sigpde_b200 import synthetic
    xs = [synthetic.brownian_np(1, int(L), w["d"], w["seed"] * 100003 + 2 * b)[0] for b, L in enumerate(lx)]
    ys = [synthetic.brownian_np(1, int(L), w["d"], w["seed"] * 100003 + 2 * b + 1)[0] for b, L in enumerate(ly)]
    return xs, ys


def ragged_cells(lx, ly, orders):
    return int(sum(((a - 1) << o) * ((b - 1) << o) for a, b, o in zip(lx, ly, orders)))


def ragged_config(w, precision):
    """The `config` of the uneven-batch bench line, shared by every arm."""
    return {"workload": "pairwise 4096 uneven pairs, L~U[16,512] per path, d=32, order~U{0..3} per pair",
            "global_batch": w["npairs"], "seq_len": "16-512", "parallelism": "single GPU",
            "precision": precision, "l2": "GPU arm: flushed between timed steps (256 MB write); CPU arm: host memory",
            "launch": "GPU arm: one persistent ragged launch, CUDA-graph replay"}


def cpu_oracle_ragged(w, xs, ys, orders, target_s, seed=7):
    """Float64 oracle on a random sample of pairs; returns (cells/s, cores, sample)."""
    import numpy as np
    from oracle import oracle
    oracle.build()
    rng = np.random.default_rng(seed)
    n = max(oracle.num_threads(), 8)
    idx = []
    t_used = 0.0
    cells = 0
    perm = rng.permutation(len(xs))
    pos = 0
    while t_used < target_s and pos < len(perm):
        take = perm[pos:pos + n]
        pos += n
        t0 = time.perf_counter()
        for b in take:  # one pair at a time (lengths differ); OpenMP inside is over one pair only
            x = xs[b].astype(np.float32).astype(np.float64)[None]
            y = ys[b].astype(np.float32).astype(np.float64)[None]
            oracle.pairwise(x, y, int(orders[b]))
        t_used += time.perf_counter() - t0
        idx.extend(int(b) for b in take)
        cells += sum(((len(xs[b]) - 1) << orders[b]) * ((len(ys[b]) - 1) << orders[b]) for b in take)
    return cells / t_used, 1, f"{len(idx)} random pairs of the uneven batch ({cells:.3e} cells) in {t_used:.1f} s, 1 thread"


def run_ours_ragged(args, w):
    import numpy as np
    import torch
    import sigpde_b200.torch as sig
    from sigpde_b200 import _lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    lx, ly, orders = ragged_spec(w)
    xs, ys = ragged_paths(w, lx, ly)
    cells = ragged_cells(lx, ly, orders)
    X = [torch.tensor(a, dtype=torch.float32, device=dev) for a in xs]
    Y = [torch.tensor(a, dtype=torch.float32, device=dev) for a in ys]
    tuning = None
    tuner = None
    if args.autotune:  # increment source, tile width and rows per lane, measured before and outside the timed region
        import time as _time
        t0 = _time.perf_counter()
        tuner = sig.autotune.RaggedTuner(w["d"], args.precision, torch.float32, dev)
        tuner.tune_for(lx, ly, orders)
        tuning = dict(tuner.report(), seconds=_time.perf_counter() - t0,
                      batch_timings_ms={str(k): v for k, v in tuner.batch_timings.items()})
        # the default rule on the same batch, for comparison (timed like the tuned plan below)
        dflt = sig.ragged.RaggedPairwise(lx, ly, orders, w["d"], torch.float32, dev, args.precision)
        dflt.load(X, Y)
        dflt.capture()
        fl = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
        tuning["default_rule_ms_per_step"] = statistics.mean(
            timed_steps(torch, dflt.solve, args.steps, args.warmup, fl, lambda: None))
        del dflt, fl
    solver = sig.ragged.RaggedPairwise(lx, ly, orders, w["d"], torch.float32, dev, args.precision, tuner=tuner)
    solver.load(X, Y)
    solver.capture()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    clocks = ClockSampler(0)
    clocks.start()
    times = timed_steps(torch, solver.solve, args.steps, args.warmup, flush, lambda: None)
    launches = solver.graph_kernels * args.steps  # graph replays: the captured kernels, once per step
    clk = clocks.stop()
    ms = statistics.mean(times)
    out = solver.out.double().cpu().numpy()
    # end to end: packed paths from pinned host memory, one graph replay, result back to pinned host memory
    xh = solver.x_pack.cpu().pin_memory()
    yh = solver.y_pack.cpu().pin_memory()
    oh = torch.empty_like(solver.out, device="cpu").pin_memory()

    def e2e_step():
        solver.x_pack.copy_(xh, non_blocking=True)
        solver.y_pack.copy_(yh, non_blocking=True)
        oh.copy_(solver.solve(), non_blocking=True)

    e2e_times = timed_steps(torch, e2e_step, args.steps, args.warmup, flush, lambda: None)
    acc = cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle
        rng = np.random.default_rng(1)
        pick = rng.choice(len(xs), 32, replace=False)
        want = np.array([oracle.pairwise(xs[b].astype(np.float32).astype(np.float64)[None],
                                         ys[b].astype(np.float32).astype(np.float64)[None], int(orders[b]))[0]
                         for b in pick])
        acc = {"max_rel_err": float(np.max(np.abs(out[pick] - want) / np.abs(want))),
               "sample": "32 random pairs vs the float64 oracle"}
        rate, cores, sample = cpu_oracle_ragged(w, xs, ys, orders, args.cpu_seconds)
        cpu = {"value": rate, "unit": "cells/s", "cores": cores, "kind": "port", "sample": sample}
    line = {
        "metric": "pde_cell_updates_per_s", "value": cells / (ms * 1e-3), "unit": "cells/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "p50_ms": percentile(times, 0.5),
        "p99_ms": percentile(times, 0.99), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision in ("fp64", "tc64") else "f32",
        "data": "synthetic Brownian paths (seeded PCG64), float32",
        "config": ragged_config(w, args.precision),
        "pairs_per_s": w["npairs"] / (ms * 1e-3), "cells_per_step": cells, "accuracy": acc,
        "e2e": {"value": cells / (statistics.mean(e2e_times) * 1e-3), "unit": "cells/s",
                "h2d_bytes_per_step": xh.numel() * xh.element_size() + yh.numel() * yh.element_size(),
                "d2h_bytes_per_step": oh.numel() * oh.element_size(), "ms_per_step": statistics.mean(e2e_times)},
        "gpu_launches": launches, "clocks": clk, "lib": _lib.version(),
    }
    if tuning is not None:
        line["autotune"] = tuning
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def run_reference_ragged(args, w):
    """The CPU reference arm of the uneven batch: the float64 oracle on a sample of its pairs per step."""
    lx, ly, orders = ragged_spec(w)
    xs, ys = ragged_paths(w, lx, ly)
    cells = ragged_cells(lx, ly, orders)
    step_s = max(1.0, args.cpu_seconds / 2)
    rates = []
    cores = sample = None
    for i in range(args.warmup + args.steps):
        rate, cores, sample = cpu_oracle_ragged(w, xs, ys, orders, step_s, seed=7 + i)
        if i >= args.warmup:
            rates.append(rate)
    value = statistics.mean(rates)
    print(json.dumps({
        "impl": "reference", "metric": "pde_cell_updates_per_s", "value": value, "unit": "cells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": cells / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic Brownian paths (seeded PCG64), float32 inputs upcast to float64",
        "config": ragged_config(w, "fp64"),
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "port",
                         "sample": f"per step: {sample}; float64 C restatement of the reference solver"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def run_reference_gpu_ragged(args, w):
    """The reference's Numba path: one SigPDE.pairwise call per (len x, len y, order) bucket."""
    import torch
    ref_dir = os.path.join(ROOT, "baseline", "_ref")
    base = {"impl": "reference-gpu", "metric": "pde_cell_updates_per_s", "unit": "cells/s"}
    if not os.path.isdir(os.path.join(ref_dir, "sigpde")):
        print(json.dumps(dict(base, unavailable="reference not installed under baseline/_ref")), flush=True)
        return
    sys.path.insert(0, ref_dir)
    import warnings
    warnings.filterwarnings("ignore")
    import sigpde.torch as refsig
    lx, ly, orders = ragged_spec(w)
    xs, ys = ragged_paths(w, lx, ly)
    cells = ragged_cells(lx, ly, orders)
    buckets = {}
    for b, key in enumerate(zip(lx, ly, orders)):
        buckets.setdefault(key, []).append(b)
    dev = torch.device("cuda", 0)
    calls = []
    for (a, c, o), idx in buckets.items():
        import numpy as np
        X = torch.tensor(np.stack([xs[b] for b in idx]), dtype=torch.float32, device=dev)
        Y = torch.tensor(np.stack([ys[b] for b in idx]), dtype=torch.float32, device=dev)
        calls.append((refsig.SigPDE(refsig.kernels.LinearKernel(), o), X, Y))
    lin_calls = calls

    def step():
        for k, X, Y in lin_calls:
            k.pairwise(X, Y)

    step()  # JIT
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step()
        torch.cuda.synchronize()
        times.append((time.perf_counter() - t0) * 1e3)
    ms = statistics.mean(times)
    print(json.dumps(dict(base, value=cells / (ms * 1e-3), ms_per_step=ms, steps=args.steps, n_gpus=1,
                          calls_per_step=len(calls), pairs_per_s=w["npairs"] / (ms * 1e-3),
                          config={"workload": "pairwise 4096 uneven pairs, L~U[16,512], d=32, order~U{0..3}"},
                          note="one reference SigPDE.pairwise call per (len x, len y, order) bucket")), flush=True)


# ----------------------------------------------------------------------------- robust Gram
def robust_inputs(w):
    from sigpde_b200 import synthetic
    scales = synthetic.log_uniform(w["n"], w["smin"], w["smax"], w["seed"] + 1)
    return synthetic.brownian_np(w["n"], w["L"], w["d"], w["seed"], scale=scales)


def run_ours_robust(args, w):
    import numpy as np
    import torch
    import sigpde_b200.torch as sig
    from sigpde_b200 import _lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    x = robust_inputs(w)
    X = torch.tensor(x, dtype=torch.float32, device=dev)
    rk = sig.RobustSigPDE(sig.kernels.LinearKernel(), w["order"], precision=args.precision)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    out = rk.gram(X)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    times = timed_steps(torch, lambda: rk.gram(X), args.steps, args.warmup, flush, lambda: None)
    launches = LAUNCHES["last"]
    clk = clocks.stop()
    # the two phases separately: lambda root-find, then the scaled symmetric Gram
    lam = rk.normalization(X)
    t_norm = timed_steps(torch, lambda: rk.normalization(X), args.steps, args.warmup, flush, lambda: None)
    k = sig.SigPDE(sig.kernels.LinearKernel(), w["order"], precision=args.precision)
    t_gram = timed_steps(torch, lambda: k.gram(X, None, lam), args.steps, args.warmup, flush, lambda: None)
    Xh = X.cpu().pin_memory()
    Rh = torch.empty((w["n"], w["n"]), dtype=X.dtype).pin_memory()

    def e2e_step():
        Rh.copy_(rk.gram(Xh.to(dev, non_blocking=True)), non_blocking=True)

    e2e_times = timed_steps(torch, e2e_step, args.steps, args.warmup, flush, lambda: None)
    entries = w["n"] * w["n"]
    ms = statistics.mean(times)
    acc = cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle
        xin = X.double().cpu().numpy()
        lam_o = oracle.normalization(xin, w["order"])
        lam_g = lam.double().cpu().numpy()
        G = out.double().cpu().numpy()
        rng = np.random.default_rng(1)
        flat = rng.choice(entries, 64, replace=False)
        want = oracle.gram(xin, xin, w["order"], lam_o, lam_o, pairs=flat)
        got = G.reshape(-1)[flat]
        nz = lam_o > 0
        acc = {"lambda_max_rel_err": float(np.max(np.abs(lam_g[nz] - lam_o[nz]) / lam_o[nz])),
               "lambda_zero_match": bool(np.all((lam_g == 0) == (lam_o == 0))),
               "gram_max_rel_err": float(np.max(np.abs(got - want) / np.abs(want))),
               "sample": "all 512 lambdas and 64 random Gram entries vs the float64 oracle"}
        t0 = time.perf_counter()
        oracle.normalization(xin, w["order"])
        t_lam = time.perf_counter() - t0
        t0 = time.perf_counter()
        sub = rng.choice(entries, 4096, replace=False)
        oracle.gram(xin, xin, w["order"], lam_o, lam_o, pairs=sub)
        t_g = time.perf_counter() - t0
        cpu_ms = (t_lam + t_g * entries / 2 / 4096) * 1e3  # unique (lower-triangle) entries
        cpu = {"value": entries / (cpu_ms * 1e-3), "unit": "entries/s", "cores": oracle.num_threads(),
               "kind": "port", "sample": f"all 512 lambdas ({t_lam:.1f} s) + 4096 random Gram entries ({t_g:.1f} s), "
                                         "extrapolated to the 131,328 unique entries"}
    line = {
        "metric": "gram_entries_per_s", "value": entries / (ms * 1e-3), "unit": "entries/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "p50_ms": percentile(times, 0.5),
        "p99_ms": percentile(times, 0.99), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision in ("fp64", "tc64") else "f32",
        "data": "synthetic Brownian paths (seeded PCG64), per-path scale log-uniform [0.5, 4], float32",
        "config": {"workload": "RobustSigPDE.gram(x) N=512, L=64, d=16, dyadic_order=1, default normaliser",
                   "global_batch": entries, "seq_len": w["L"], "parallelism": "single GPU",
                   "precision": args.precision, "l2": "flushed between timed steps (256 MB write)"},
        "unique_entries_per_s": w["n"] * (w["n"] + 1) / 2 / (ms * 1e-3),
        "phases_ms": {"normalization": statistics.mean(t_norm), "scaled_symmetric_gram": statistics.mean(t_gram)},
        "accuracy": acc,
        "e2e": {"value": entries / (statistics.mean(e2e_times) * 1e-3), "unit": "entries/s",
                "h2d_bytes_per_step": Xh.numel() * Xh.element_size(), "d2h_bytes_per_step": Rh.numel() * Rh.element_size(),
                "ms_per_step": statistics.mean(e2e_times)},
        "gpu_launches": launches, "clocks": clk, "lib": _lib.version(),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def run_reference_gpu_robust(args, w):
    """The reference's Numba path: RobustSigPDE.gram(x) through its public API."""
    import torch
    ref_dir = os.path.join(ROOT, "baseline", "_ref")
    base = {"impl": "reference-gpu", "metric": "gram_entries_per_s", "unit": "entries/s"}
    if not os.path.isdir(os.path.join(ref_dir, "sigpde")):
        print(json.dumps(dict(base, unavailable="reference not installed under baseline/_ref")), flush=True)
        return
    sys.path.insert(0, ref_dir)
    import warnings
    warnings.filterwarnings("ignore")
    import sigpde.torch as refsig
    dev = torch.device("cuda", 0)
    X = torch.tensor(robust_inputs(w), dtype=torch.float32, device=dev)
    rk = refsig.RobustSigPDE(refsig.kernels.LinearKernel(), w["order"])
    out = rk.gram(X)
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rk.gram(X)
        torch.cuda.synchronize()
        times.append((time.perf_counter() - t0) * 1e3)
    ms = statistics.mean(times)
    acc = None
    if not args.no_cpu_baseline:
        import numpy as np
        from oracle import oracle
        xin = X.double().cpu().numpy()
        lam_o = oracle.normalization(xin, w["order"])
        lam_r = rk.normalization(X).double().cpu().numpy()
        nz = lam_o > 0
        acc = {"lambda_max_rel_err": float(np.max(np.abs(lam_r[nz] - lam_o[nz]) / lam_o[nz])),
               "nonfinite_entries": int((~np.isfinite(out.double().cpu().numpy())).sum())}
    entries = w["n"] * w["n"]
    print(json.dumps(dict(base, value=entries / (ms * 1e-3), ms_per_step=ms, steps=args.steps, n_gpus=1,
                          accuracy=acc, config={"workload": "RobustSigPDE.gram(x) N=512, L=64, d=16, order 1"},
                          note="unmodified stojl/SigPDE, host-timed (it synchronises inside each call)")),
          flush=True)


# ----------------------------------------------------------------------------- serving trace
def serve_trace(w, nreq=None, pool=0):
    """Seeded request trace: (arrival offsets in s, list of GramRequest with pinned host paths).
    pool > 0: the paths come from `pool` path sets drawn like the requests' (each request takes one
    at random, so sets recur); returns (arrivals, requests, sets, set index of each request)."""
    import numpy as np
    import torch
    from sigpde_b200 import synthetic
    from sigpde_b200.serving import GramRequest
    nreq = nreq or w["requests"]
    rng = np.random.Generator(np.random.PCG64(w["seed"]))
    gaps = rng.exponential(1.0 / w["rate"], nreq)
    arrivals = np.cumsum(gaps) - gaps[0]
    if pool:
        sets = []
        for _ in range(pool):
            N = int(round(np.exp(rng.uniform(np.log(w["nmin"]), np.log(w["nmax"])))))
            L = int(round(np.exp(rng.uniform(np.log(w["lmin"]), np.log(w["lmax"])))))
            d = int(rng.choice(w["dims"]))
            x = synthetic.brownian_np(N, L, d, int(rng.integers(1 << 31)))
            sets.append(torch.tensor(x, dtype=torch.float32).pin_memory())
        idx = [int(rng.integers(pool)) for _ in range(nreq)]
        reqs = [GramRequest(x=sets[k], order=int(rng.choice(w["orders"])),
                            kind="robust" if rng.random() < w["robust"] else "gram", rid=i) for i, k in enumerate(idx)]
        return arrivals, reqs, sets, idx
    reqs = []
    for i in range(nreq):
        N = int(round(np.exp(rng.uniform(np.log(w["nmin"]), np.log(w["nmax"])))))
        L = int(round(np.exp(rng.uniform(np.log(w["lmin"]), np.log(w["lmax"])))))
        d = int(rng.choice(w["dims"]))
        o = int(rng.choice(w["orders"]))
        kind = "robust" if rng.random() < w["robust"] else "gram"
        x = synthetic.brownian_np(N, L, d, int(rng.integers(1 << 31)))
        reqs.append(GramRequest(x=torch.tensor(x, dtype=torch.float32).pin_memory(), order=o, kind=kind, rid=i))
    return arrivals, reqs


def _req_cells(r):
    N, L, _ = r.x.shape
    n = (L - 1) << r.order
    return N * N * n * n


def run_serve(args, w):
    import numpy as np
    import torch
    from sigpde_b200 import _lib
    from sigpde_b200.serving import GramServer, serve_sequential
    torch.cuda.set_device(0)
    if args.resident:
        arrivals, reqs, pool, pool_idx = serve_trace(w, pool=40)
    else:
        arrivals, reqs = serve_trace(w)
    if args.burst:
        arrivals = np.zeros_like(arrivals)
    cells = sum(_req_cells(r) for r in reqs)
    entries = sum(r.x.shape[0] ** 2 for r in reqs)
    # warm up the kernel variants once (first-use costs are not part of serving)
    _, warm = serve_trace(w, 8)
    serve_sequential(warm, args.precision)

    def summarize(handles, t_first, t_last):
        lat = [h.latency * 1e3 for h in handles]
        span = t_last - t_first
        return {"requests_per_s": len(handles) / span, "entries_per_s": entries / span, "cells_per_s": cells / span,
                "p50_ms": percentile(lat, 0.5), "p99_ms": percentile(lat, 0.99), "makespan_s": span,
                "errors": sum(h.error is not None for h in handles)}

    # continuous-batching server, Poisson arrivals
    clocks = ClockSampler(0)
    clocks.start()
    with GramServer(max_inflight=8, precision=args.precision) as srv:
        if args.resident:  # stored before the clock starts: residency is the point
            stored = [srv.put(f"p{i}", t) for i, t in enumerate(pool)]
            for r, k in zip(reqs, pool_idx):
                r.x = stored[k]
        t0 = time.perf_counter()
        handles = []
        for i, r in enumerate(reqs):
            target = t0 + arrivals[i]
            while time.perf_counter() < target:
                time.sleep(max(0.0, min(1e-3, target - time.perf_counter())))
            r.arrival = target
            handles.append(srv.submit(r))
        for h in handles:
            h.wait(timeout=600)
        peak = srv.peak_inflight
        batching = {"batches": srv.batches, "batched_requests": srv.batched_requests}
        store = srv.store_stats()
    clk = clocks.stop()
    served = summarize(handles, t0, max(h.t_done for h in handles))
    served["peak_inflight"] = peak
    served["kernel_level_batching"] = batching
    if args.resident:
        served["path_store"] = {"sets": len(store), "bytes": sum(v["bytes"] for v in store.values()),
                                "scale_hits": sum(v["scale_hits"] for v in store.values()),
                                "scale_misses": sum(v["scale_misses"] for v in store.values())}
    # per-request plain launches, same arrivals
    for r in reqs:
        r.arrival = 0.0
    t1 = time.perf_counter()
    seq = serve_sequential(reqs, args.precision, arrivals=arrivals)
    plain = summarize(seq, t1, max(h.t_done for h in seq))
    # identical results alone and in the mix
    same = all(np.array_equal(a.result.numpy(), b.result.numpy()) for a, b in zip(handles, seq))
    # float64 spot checks on ~1% of the outputs (entries sampled across requests)
    spot = None
    if not args.no_cpu_baseline:
        from oracle import oracle
        rng = np.random.default_rng(0)
        errs = []
        budget = max(8, entries // 100)
        picks = rng.choice(len(reqs), min(len(reqs), 12), replace=False)
        for k in picks:
            r, h = reqs[k], handles[k]
            N = r.x.shape[0]
            x = (r.x.host if hasattr(r.x, "host") else r.x).double().numpy()
            if r.kind == "robust":
                lam = oracle.normalization(x, r.order)
                npick = 2
            else:
                lam = None
                npick = 4
            for _ in range(npick):
                i, j = int(rng.integers(N)), int(rng.integers(N))
                if r.x.shape[1] * (1 << r.order) > 1200 and r.x.shape[0] > 256:
                    continue  # keep the CPU check bounded
                want = oracle.gram(x, x, r.order, lam, lam, pairs=[i * N + j])[0]
                got = float(h.result[i, j])
                errs.append(abs(got - want) / abs(want))
        spot = {"checked_entries": len(errs), "max_rel_err": float(max(errs)) if errs else None,
                "target_entries_1pct": int(budget),
                "note": "entries sampled from 12 random requests (robust: lambda from the oracle too)"}
    line = {
        "metric": "served_requests_per_s", "value": served["requests_per_s"], "unit": "requests/s", "n_gpus": 1,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision in ("fp64", "tc64") else "f32",
        "data": "synthetic Brownian paths (seeded PCG64), float32, pinned host memory",
        "config": {"workload": f"serving trace: {len(reqs)} Gram requests, Poisson {w['rate']}/s, "
                               f"N~logU[{w['nmin']},{w['nmax']}], L~logU[{w['lmin']},{w['lmax']}], d in {{2,8,32}}, "
                               "order in {0,1,2}, 30% robust" + (" (burst: all at t=0)" if args.burst else "")
                               + (", paths from 40 path sets kept resident by the server (the per-request "
                                  "baseline copies each request's paths in)" if args.resident else ""),
                   "parallelism": "single GPU, 8 in-flight streams, HBM-footprint admission"},
        "served": served, "per_request_plain_launches": plain,
        "throughput_ratio_vs_plain": served["requests_per_s"] / plain["requests_per_s"],
        "results_identical_alone_and_in_mix": same, "fp64_spot_check": spot,
        "trace_cells": cells, "trace_entries": entries, "clocks": clk, "lib": _lib.version(),
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    w = WORKLOADS[args.workload]
    ragged = w.get("kind") == "ragged"
    robust = w.get("kind") == "robust"
    if w.get("kind") == "serve":
        if args.impl == "ours":
            run_serve(args, w)
        else:
            print(json.dumps({"impl": args.impl, "unavailable": "serving trace: the reference has no server; "
                              "the per-request plain-launch arm is inside the default run"}), flush=True)
        return
    if robust:
        if args.impl == "reference-gpu":
            run_reference_gpu_robust(args, w)
        elif args.impl == "ours":
            run_ours_robust(args, w)
        else:
            print(json.dumps({"impl": "reference", "unavailable": "robust512 CPU arm: use the cpu_baseline of the "
                              "default run"}), flush=True)
        return
    if w.get("kind") == "grad" and args.impl != "ours":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"impl": args.impl, "unavailable": "the reference has no backward pass (its Numba "
                              "kernels end autograd); the oracle's adjoint is the cpu_baseline of the default run"}),
                  flush=True)
        return
    if args.impl == "reference":
        if ragged:
            if int(os.environ.get("RANK", "0")) == 0:
                run_reference_ragged(args, w)
            return
        run_reference(args, w, int(os.environ.get("RANK", "0")))
        return
    if args.impl == "reference-gpu":
        if int(os.environ.get("RANK", "0")) == 0:
            (run_reference_gpu_ragged if ragged else run_reference_gpu)(args, w)
        return
    if ragged:
        run_ours_ragged(args, w)
        return
    if w.get("kind") == "static":
        if int(os.environ.get("RANK", "0")) == 0:
            run_ours_static(args, w)
        return
    if w.get("kind") == "grad":
        if int(os.environ.get("RANK", "0")) == 0:
            run_ours_grad(args, w)
        return
    run_ours(args, w)


if __name__ == "__main__":
    main()
