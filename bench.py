"""Benchmark of the LLE-map hot path (one JSON line on stdout).

Workload (one "step" = one full map): Rossler largest-Lyapunov map dx=-y-z, dy=x+ay,
dz=b+z(x-c), a=0.2, b in [0.05, 2] x c in [2, 20] on an N x N grid (default 1024),
x0=(1,1,1), RK4 h=0.01, 10^4 transient steps, t_max=1000 with the tangent vector
renormalised every NT=0.1 (10 steps): 10^5 measured steps per trajectory. The step body
is the reference codegen's RK4 text for this system (tests/golden), passed through the
same C ABI a session would call. Inputs are the grid description (synthetic by
construction); no dataset is involved.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 1024]

`value` is the chosen form (FP32 state, tangent vector, FP64 norms and log sums) in
cells/s over all GPUs; `forms` also reports the plain FP64 form. The reference arm
(--impl reference) times the oracle's restatement of the reference's CPU path
(krs_cpu step + LLEKernelCUDA semantics, OpenMP over cells) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "u-cuda_b200"))
sys.path.insert(0, str(ROOT / "tests"))

METRIC = "RK4 steps/s; 1024² LLE-map cells/s, plain vs surrogate at ≤2e-3 LLE err"
L2_FLUSH_BYTES = 256 << 20


def rossler_body() -> str:
    cases = json.loads((ROOT / "tests" / "golden" / "codegen_cases.json").read_text())["cases"]
    return {c["name"]: c for c in cases}["rossler_config"]["schemes"]["RK4"]


def workload(n: int) -> dict:
    return dict(body=rossler_body(), nx=3, ic=(1.0, 1.0, 1.0), values=(0.0, 0.2, 0.2, 5.7), n_pts=n,
                param_index=2, param_index_2=3, param_lo=0.05, param_hi=2.0, param_lo_2=2.0, param_hi_2=20.0,
                h=0.01, transient_time=100.0, t_max=1000.0, NT=0.1, eps=1e-4, max_value=1e6)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.stop = threading.Event()
        self.t = threading.Thread(target=self.run, daemon=True)

    def run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                parts = [p.strip() for p in out.stdout.strip().split(",")]
                if len(parts) >= 8:
                    self.samples.append(parts)
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    import ucb
    from helpers import engine_request

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    # Weak scaling: every rank computes a full map of its own (independent replicas; the
    # path has no exchange step, so nothing crosses NVLink).
    c = workload(n)
    eng = ucb.Engine(local)
    forms = {
        "fp32": dict(precision=ucb.PREC_F32, mode=ucb.MODE_NATIVE),
        "plain_fp64": dict(precision=ucb.PREC_F64, mode=ucb.MODE_NATIVE),
    }
    cells = n * n
    d_values = torch.empty(cells, dtype=torch.float64, device=dev)
    d_flags = torch.empty(cells, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    results = {}
    clocks = None
    launches_timed = 0
    for name, opt in forms.items():
        req = engine_request(ucb, c, **opt)
        # warm-up (also compiles the kernel)
        for _ in range(args.warmup):
            eng.lle2d_device(req, d_values.data_ptr(), d_flags.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        l0 = eng.launches
        sampler = ClockSampler(local) if name == "fp32" else None
        ctx = sampler if sampler else _Null()
        with ctx:
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            for k in range(args.steps):
                flush.fill_(float(k))  # L2 flush between steps, outside the per-step events
                ev[k][0].record(stream)
                eng.lle2d_device(req, d_values.data_ptr(), d_flags.data_ptr(), stream.cuda_stream)
                ev[k][1].record(stream)
            torch.cuda.synchronize(dev)
            wall = time.perf_counter() - t0
        if sampler:
            clocks = sampler.summary()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        ms = float(np.mean(step_ms))
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        launches = eng.launches - l0
        if name == "fp32":
            launches_timed = launches
        # work and FLOPs of one map, read back through the host entry once
        _, flags, res = eng.run_lle2d(req)
        results[name] = dict(ms=ms, wall_s=wall, steps=res.steps, flops=res.flops, kernel_ms=res.kernel_ms,
                             valid_cells=int((flags == 1).sum()), launches=launches)
    # end-to-end through the public C ABI with host buffers (H2D of the request, D2H of
    # values + flags inside the timed region), chosen form
    req = engine_request(ucb, c, **forms["fp32"])
    hv = np.empty(cells, dtype=np.float64)
    hf = np.empty(cells, dtype=np.int32)
    e2e_ms = []
    e2e_kernel_ms = []
    for k in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _, _, r = eng.run_lle2d(req, hv, hf)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        e2e_kernel_ms.append(r.kernel_ms)
    e2e = float(np.mean(e2e_ms))
    results["e2e_detail"] = {"wall_ms": e2e_ms, "kernel_ms": e2e_kernel_ms}
    if world > 1:
        t = torch.tensor([e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = float(t.item())
    return results, clocks, launches_timed, e2e


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def cpu_sample_cells(n: int, stride: int):
    rows = np.arange(0, n, stride)
    cols = np.arange(0, n, stride)
    return (rows[:, None] * n + cols[None, :]).ravel().astype(np.int64)


def run_cpu_baseline(n: int, stride: int, nthreads: int = 0):
    from helpers import kernel_grid
    from oracle import oracle as O

    c = workload(n)
    k = O.Krs(c["body"], 3, "f64")
    cells = cpu_sample_cells(n, stride)
    t0 = time.perf_counter()
    v, f = O.lle2d(k, kernel_grid(c), cells=cells, nthreads=nthreads)
    dt = time.perf_counter() - t0
    cores = nthreads if nthreads > 0 else (os.cpu_count() or 1)
    steps_per_cell = (int(c["transient_time"] / c["h"]) + 1) + int(c["t_max"] / c["NT"]) * 2 * (
        int(c["NT"] / c["h"]) + 1)
    return dict(value=len(cells) / dt, unit="cells/s", cores=cores, kind="port",
                sample=f"{len(cells)} cells (every {stride}th row and column of the {n}x{n} map), "
                       f"{dt:.1f} s wall, FP64 krs_cpu restatement, OpenMP",
                steps_per_s=len(cells) * steps_per_cell / dt, seconds=dt)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--cpu-stride", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank, world, local = dist_env()
    cfg = {"workload": f"Rossler LLE map {args.n}x{args.n} (b in [0.05,2] x c in [2,20], a=0.2), RK4 h=0.01, "
                       f"1e4 transient + 1e5 measured steps, renormalised every 10 steps",
           "grid": args.n, "cells": args.n * args.n, "parallelism": f"replicas x{world}",
           "l2": "256 MiB buffer written between timed steps, outside the per-step events",
           "step_semantics": "reference (extra step after each loop call)"}

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        O.build() if not O.LIB_PATH.exists() else None
        vals = []
        info = None
        for k in range(args.warmup + args.steps):
            info = run_cpu_baseline(args.n, max(args.cpu_stride, 32), 0)
            if k >= args.warmup:
                vals.append(info["value"])
        v = float(np.mean(vals))
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cells/s", "n_gpus": 0,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * args.n * args.n / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic grid", "config": cfg,
                "cpu_baseline": {k2: info[k2] for k2 in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_baseline(args.n, args.cpu_stride, 0)
    results, clocks, launches, e2e_ms = run_ours(args, rank, world, local)
    import ucb
    peak64 = ucb.measure_fma_peak(ucb.PREC_F64)
    peak32 = ucb.measure_fma_peak(ucb.PREC_F32)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    cells = args.n * args.n
    r32, r64 = results["fp32"], results["plain_fp64"]
    value = world * cells / (r32["ms"] * 1e-3)
    forms = {}
    for name, r in results.items():
        if name == "e2e_detail":
            continue
        forms[name] = {"cells_per_s": world * cells / (r["ms"] * 1e-3),
                       "rk4_steps_per_s": world * r["steps"] / (r["ms"] * 1e-3), "ms_per_map": r["ms"],
                       "achieved_tflops": r["flops"] / (r["ms"] * 1e-3) / 1e12, "valid_cells": r["valid_cells"]}
    ach = r32["flops"] / (r32["ms"] * 1e-3) / 1e12
    ach64 = r64["flops"] / (r64["ms"] * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r32["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 state, f64 norms/log sums", "data": "synthetic grid (no dataset)",
        "config": cfg,
        "rk4_steps_per_s": world * r32["steps"] / (r32["ms"] * 1e-3),
        "forms": forms,
        "roofline": {"bound": "fp32", "achieved": ach, "peak": peak32, "unit": "TFLOP/s", "frac": ach / peak32,
                     "traffic": None,
                     "peak_source": "measured FMA probe (ucb_measure_fma_peak) on this GPU in this run",
                     "plain_fp64": {"bound": "fp64", "achieved": ach64, "peak": peak64, "frac": ach64 / peak64}},
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {"value": world * cells / (e2e_ms * 1e-3), "unit": "cells/s", "detail": results["e2e_detail"],
                "h2d_bytes_per_step": 2 * args.n * 4 + 3 * 8 + 4 * 8,
                "d2h_bytes_per_step": cells * (8 + 4) + 8},
    }
    if cpu:
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
