#!/usr/bin/env python
"""Benchmark: dose solves/s of the CSD-DLR energy loop on the B200 (plain FP64).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl titus|reference]
                    [--method bug|parallel|fixed]

Workload (default): the seeded water/lung/bone phantom on 200 x 200 cells,
P_29 (900 moments), rank cap 80, 5 MeV -> 1 keV electrons in 29 697 energy
steps, solved with the rank-adaptive BUG integrator (``--method parallel``:
the parallel integrator; ``--method fixed``: the fixed-rank integrator on the
100 x 100 water beam, P_21, r = 20).

A step is one complete dose solve (the whole energy sweep). ``value`` times the
device-resident solve (problem already uploaded, CUDA events on the launching
stream, L2 flushed between solves); ``e2e`` times the one-shot C-ABI call
``titus_solve_problem`` with host buffers (upload, solve, result copy-out,
free). Multi-GPU runs are independent replicas (one solve per GPU per step, no
data exchange), reported as weak scaling.

``--impl reference`` times the FP64 CPU oracle (numpy/scipy, all host
threads) on a bounded sample of energy steps of the same workload and
extrapolates to solves/s.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "bug": dict(name="csd_phantom_200x200_P29_cap80_bug", Nx=201, r=80, nPN=29, problem="csdPhantom", method="bug"),
    "parallel": dict(name="csd_phantom_200x200_P29_cap80_parallel", Nx=201, r=80, nPN=29, problem="csdPhantom",
                     method="parallel"),
    "fixed": dict(name="csd_water_beam_100x100_P21_r20_fixed", Nx=101, r=20, nPN=21, problem="csdWaterBeam",
                  method="fixed"),
}
WORKLOAD = WORKLOADS["bug"]
ORACLE_SAMPLE_STEPS = 40
# DRAM bytes (read + write) per energy step of each kernel on its workload, from
# one ncu capture of the first energy steps (see profiles/); the per-launch
# figure scales it to the launch's energy steps.
DRAM_BYTES_PER_STEP_NCU = {"fixed": (5.010176e6 + 0.218112e6) / 20,
                           "bug": (77.263616e6 + 193.732352e6) / 20, "parallel": None}


def algorithmic_bytes_per_step(n, r, q, w=8):
    """Per energy step with ideal fusion: w (15 n r + 4 n q) + 8 * 4 n (rho^-1 x2, dose RMW)."""
    return w * (15 * n * r + 4 * n * q) + 8 * 4 * n


def algorithmic_bytes_adaptive(n, ranks, q, w=8):
    """Adaptive integrators: the fixed-rank figure with r replaced by the
    augmented width 2r, summed over the ranks the solve actually ran at."""
    return sum(algorithmic_bytes_per_step(n, 2 * int(r), q, w) for r in ranks)


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = [r.split(",") for r in getattr(self, "out", "").strip().splitlines() if r.strip()]
        sm, reasons, mx = [], set(), None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def oracle_sample_seconds(steps):
    from oracle.settings import Settings as OSettings
    from oracle.solver import SolverCSD as OSolver
    from oracle.solver import solve_dlr_bug, solve_dlr_fixed, solve_dlr_parallel

    w = WORKLOAD
    s = OSettings(w["Nx"], w["Nx"], w["r"], w["problem"], nPN=w["nPN"])
    o = OSolver(s)
    fn = {"fixed": solve_dlr_fixed, "bug": solve_dlr_bug, "parallel": solve_dlr_parallel}[w["method"]]
    t0 = time.perf_counter()
    fn(o, max_steps=steps)
    return time.perf_counter() - t0, o.csd.eTrafo.size - 1


def run_reference(args, rank):
    if rank != 0:
        return
    cores = os.cpu_count()
    for _ in range(args.warmup):
        oracle_sample_seconds(ORACLE_SAMPLE_STEPS)
    ts = []
    total_steps = None
    for _ in range(args.steps):
        t, total_steps = oracle_sample_seconds(ORACLE_SAMPLE_STEPS)
        ts.append(t)
    t_solve = (sum(ts) / len(ts)) * total_steps / ORACLE_SAMPLE_STEPS
    v = 1.0 / t_solve
    line = {
        "impl": "reference", "metric": "dose solves/s", "value": v, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_solve * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD["name"], "energy_steps": total_steps, "parallelism": "replicas"},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"FP64 oracle, {WORKLOAD['method']} integrator, first {ORACLE_SAMPLE_STEPS} of "
                                   f"{total_steps} energy steps per step, extrapolated linearly"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_gpu(args, rank, world, local_rank):
    import numpy as np
    import torch

    from titus_b200 import Settings, SolverCSD
    from titus_b200 import _lib
    from titus_b200.replicas import replica_throughput

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    w = WORKLOAD
    method = {"fixed": _lib.TITUS_DLR_FIXED, "bug": _lib.TITUS_BUG_ADAPTIVE,
              "parallel": _lib.TITUS_PARALLEL_ADAPTIVE}[w["method"]]
    s = Settings(w["Nx"], w["Nx"], w["r"], w["problem"], nPN=w["nPN"])
    solver = SolverCSD(s, team_ctas=args.team)
    lib = _lib.load()
    h = solver.handle()
    opt = solver.options()
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def solve_once():
        _lib.check(lib.titus_solve_device(h, method, C.byref(opt), C.c_void_p(stream.cuda_stream)),
                   "titus_solve_device")

    for _ in range(args.warmup):
        solve_once()
    torch.cuda.synchronize()
    res, bufs = solver._result(s.r)
    _lib.check(lib.titus_fetch(h, C.byref(res)), "titus_fetch")
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    elapsed = 0.0
    # device-side time per kernel launch (the solve is one launch of the energy-loop kernel)
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solve_once()
            e1.record(stream)
            torch.cuda.synchronize()
            elapsed += e0.elapsed_time(e1) / 1e3
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    _lib.check(lib.titus_fetch(h, C.byref(res)), "titus_fetch")
    value, t_max = replica_throughput(args.steps, elapsed, world, device="cuda")
    ms_per_step = t_max / args.steps * 1e3

    # end-to-end: one-shot C-ABI call with host buffers (upload, solve, copy-out)
    p, keep = solver.problem_struct()
    h2d = sum(a.nbytes for a in keep)
    res2, bufs2 = solver._result(s.r)
    d2h = sum(b.nbytes for b in bufs2.values())
    e2e_steps = max(1, min(args.steps, 3))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        _lib.check(lib.titus_solve_problem(C.byref(p), method, C.byref(opt), C.byref(res2)),
                   "titus_solve_problem")
    t_e2e = time.perf_counter() - t0
    e2e_value, t_e2e = replica_throughput(e2e_steps, t_e2e, world, device="cuda")

    n, q = solver.n, solver.q
    steps_per_solve = int(res.steps_done)
    if w["method"] == "fixed":
        alg_bytes = algorithmic_bytes_per_step(n, s.r, q) * steps_per_solve
    else:
        hist = bufs["rank_history"]
        alg_bytes = algorithmic_bytes_adaptive(n, hist[hist >= 0], q)
    traffic_step = DRAM_BYTES_PER_STEP_NCU.get(w["method"])
    achieved = alg_bytes / (t_max / args.steps) / 1e9
    peak, peak_kind = read_peaks()
    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            t_s, total = oracle_sample_seconds(ORACLE_SAMPLE_STEPS)
            cv = 1.0 / (t_s * total / ORACLE_SAMPLE_STEPS)
            cpu = {"value": cv, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"FP64 oracle, first {ORACLE_SAMPLE_STEPS} of {total} energy steps, extrapolated"}
        line = {
            "metric": "dose solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w["name"], "energy_steps": steps_per_solve, "cells": n, "moments": solver.N,
                       "ordinates": q, "rank_cap" if w["method"] != "fixed" else "rank": s.r,
                       "method": w["method"], "team_ctas": args.team or "default", "parallelism": f"replicas{world}",
                       "l2": "flushed between solves (256 MB write)"},
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": traffic_step * steps_per_solve if traffic_step else None,
                         "traffic_note": "ncu capture of the first energy steps scaled to the launch's steps",
                         "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": (2 if w["method"] != "parallel" else 3) * args.steps,
            "rank_final": int(res.rank),
            "dose_max": float(np.max(bufs["dose"])),
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--method", default="bug", choices=sorted(WORKLOADS))
    ap.add_argument("--team", type=int, default=148, help="CTAs per solve (0 = library default)")
    ap.add_argument("--impl", default="titus", choices=["titus", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    global WORKLOAD
    WORKLOAD = WORKLOADS[args.method]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
