#!/usr/bin/env python
"""Benchmark: dose solves/s of the CSD-DLR energy loop on the B200 (plain FP64).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl titus|reference]
                    [--method bug|parallel|fixed|pn_full|pn3d|batched] [--no-batched] [--no-cpu-baseline]

Workload (default ``bug``): the seeded water/lung/bone phantom on 200 x 200
cells, P_29 (900 moments), rank cap 80, 5 MeV -> 1 keV electrons in 29 697
energy steps (29 695 loop iterations), solved with the rank-adaptive BUG
integrator. ``--method parallel`` runs the parallel integrator on it;
``--method fixed`` the fixed-rank integrator on the 100 x 100 water beam
(P_21, r = 20); ``--method pn_full`` the full-rank P_N solver on that water
beam; ``--method pn3d`` the full-rank P_N solver on the 3D proton problem (96^3
cells at 1 mm, seeded water / lung / bone spheres, P_13, 90 -> 1 MeV in 1336
energy steps); ``--method batched`` makes the batched pencil-beam plan below
the timed step.

A step is one complete dose solve (the whole energy sweep, one kernel
launch). ``value`` times the device-resident solve (problem already uploaded,
CUDA events on the launching stream, L2 flushed between solves by a 256 MB
write); ``e2e`` times the one-shot C-ABI call ``titus_solve_problem`` with
host buffers (upload, solve, result copy-out, free). After the timed steps the
same problem is run for its first 200 iterations and compared with the FP64
oracle's dose for them (``dose_rel_err_vs_oracle``, fixture
``tests/golden/phantom200_P29_bug200.npz``).

``batched``: 256 pencil beams on the seeded 128 x 128 phantom, P_21, rank cap
60, energies U(2, 8) MeV, entry y0 U(0.1, 0.9) (seed 3), all in one persistent
launch with small teams taking spots from a device work queue. Its ``plain``
companion is the same spots solved one at a time with all SMs, timed on the
shortest spots and scaled by iteration counts. The default run measures it
once after the timed steps on every spot's first 600 iterations
(``--no-batched`` skips it); ``--method batched`` times whole plans.

Multi-GPU (``--gpus N``; without WORLD_SIZE in the environment the script
re-launches itself under torch.distributed.run): the solve runs as N
independent replicas (a single dose solve does not shard) and reports weak
scaling with the max-over-ranks device time; the batched plan is sharded by
spot, and the weighted total dose is summed over ranks by an NCCL all-reduce.

``--impl reference`` times the FP64 CPU oracle (numpy/scipy, all host
threads) -- the Julia reference cannot run here -- on bounded windows of the
same workload and sums a per-iteration cost model over the GPU solve's rank
history (see ``cpu_cost_model``).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import socket
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
    "pn_full": dict(name="csd_water_beam_100x100_P21_full_rank", Nx=101, r=4, nPN=21, problem="csdWaterBeam",
                    method="pn_full"),
    # the 3D proton problem (96^3 cells at 1 mm, seeded spheres, P13) with the full-rank solver
    "pn3d": dict(name="csd_proton3d_96cube_P13_full_rank", Nx=97, r=40, nPN=13, problem="csdProton3D",
                 method="pn3d"),
    # the same 3D problem with the rank-adaptive BUG integrator (rank cap 40)
    "bug3d": dict(name="csd_proton3d_96cube_P13_cap40_bug", Nx=97, r=40, nPN=13, problem="csdProton3D",
                  method="bug3d"),
}
THREE_D = ("pn3d", "bug3d")


def three_d_workload(w, size):
    """`w` with `size` cells per axis (3D workloads; 0 keeps the workload's 96)."""
    if not size or w["method"] not in THREE_D:
        return w
    w = dict(w, Nx=size + 1)
    w["name"] = w["name"].replace("96cube", f"{size}cube")
    return w
BATCHED = dict(name="pencil_beams256_phantom_128x128_P21_cap60_bug", Nx=129, r=60, nPN=21, problem="csdPhantom",
               spots=256, seed=3, emin=2.0, emax=8.0, ymin=0.1, ymax=0.9)
# the batched plan measured beside the default solve: every spot's first
# BATCHED_SAMPLE_ITERS loop iterations (the whole plan takes minutes)
BATCHED_SAMPLE_ITERS = 600
FIXTURE = os.path.join(ROOT, "tests", "golden", "phantom200_P29_bug200.npz")
RANKS_FIXTURE = os.path.join(ROOT, "tests", "golden", "phantom200_P29_bug_ranks.npz")
# DRAM bytes (read + write) per energy step of each kernel on its workload, from
# one ncu capture of the first energy steps (profiles/); the per-launch figure
# scales it to the launch's energy steps.
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


def batched_spots(cfg=BATCHED, count=None):
    import numpy as np

    rng = np.random.default_rng(cfg["seed"])
    ns = cfg["spots"] if count is None else count
    e = rng.uniform(cfg["emin"], cfg["emax"], ns)
    y = rng.uniform(cfg["ymin"], cfg["ymax"], ns)
    return [(float(a), float(b)) for a, b in zip(e, y)]


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


# ------------------------------------------------------------ CPU baseline
def _oracle_setup(w):
    if w["method"] in THREE_D:
        from oracle.three_d import Settings3D as OSettings3D
        from oracle.three_d import SolverCSD3D as OSolver3D

        return lambda: OSolver3D(OSettings3D(w["Nx"], w["Nx"], w["Nx"], w["r"], w["problem"], nPN=w["nPN"]))
    from oracle.settings import Settings as OSettings
    from oracle.solver import SolverCSD as OSolver

    return lambda: OSolver(OSettings(w["Nx"], w["Nx"], w["r"], w["problem"], nPN=w["nPN"]))


class _IterClock:
    """Per-iteration wall times by the rank entering each iteration (the
    oracle's on_iter hook)."""

    def __init__(self):
        self.by_rank = {}
        self._t = None
        self._r = None

    def __call__(self, r):
        now = time.perf_counter()
        if self._r is not None:
            self.by_rank.setdefault(int(self._r), []).append(now - self._t)
        self._t, self._r = now, r


def _cost_of_history(by_rank, ranks):
    """Sum over the history of the mean measured time at each rank; ranks not
    measured take the linear interpolation between the nearest ranks measured
    at least twice (the nearest one outside their range). A rank met once --
    the first iteration, which also pays the loop's set-up -- is used where it
    occurs, never as an interpolation node: it would inflate every rank between
    it and the steady rank. Returns (seconds, share of the history's iterations
    at a directly measured rank)."""
    import numpy as np

    nodes = [r for r in sorted(by_rank) if len(by_rank[r]) >= 2] or sorted(by_rank)
    rs = np.array(nodes)
    cs = np.array([float(np.mean(by_rank[r])) for r in rs])
    vals, cnt = np.unique(np.asarray(ranks, dtype=np.int64), return_counts=True)
    per = np.interp(vals, rs, cs)
    for k, v in enumerate(vals):
        if int(v) in by_rank:
            per[k] = float(np.mean(by_rank[int(v)]))
    total = float(np.sum(per * cnt))
    direct = float(np.sum(cnt[np.isin(vals, np.array(sorted(by_rank)))]) / max(1, np.sum(cnt)))
    return total, direct


def _warm_oracle(w, mk):
    """A few untimed oracle iterations of the same problem, so that the timed
    windows do not pay first-call costs (thread pools, caches, lazy imports)."""
    if w["method"] in ("pn3d", "bug3d"):
        return
    from oracle.full_rank import solve_pn_full
    from oracle.solver import solve_dlr_bug, solve_dlr_fixed, solve_dlr_parallel

    fn = {"pn_full": solve_pn_full, "bug": solve_dlr_bug, "parallel": solve_dlr_parallel,
          "fixed": solve_dlr_fixed}[w["method"]]
    fn(mk(), max_steps=3)


def cpu_cost_model(w, ranks, state200=None, head=40, tail=20):
    """Estimated time of one whole solve by the FP64 oracle on this host's cores.

    The oracle is timed per loop iteration on two bounded windows of the same
    problem: iterations 1..`head` from the initial factors (the opening, ranks
    40 -> 3 on the 200 x 200 phantom) and `tail` iterations from the oracle's own
    state after 200 iterations (the steady rank of the sweep, about 8). The mean
    time per iteration at each rank, interpolated in the rank where a rank was
    not met, is summed over `ranks`, the rank entering every iteration of the
    GPU solve of the same problem (29 695 iterations). The fixed-rank
    integrator costs the same every step: its mean over `head` steps times the
    step count. Returns (seconds, sample description, state200) so a caller can
    reuse the 200-iteration state between repeats.
    """
    from oracle.solver import solve_dlr_bug, solve_dlr_fixed, solve_dlr_parallel

    mk = _oracle_setup(w)
    _warm_oracle(w, mk)
    if w["method"] == "pn_full":
        from oracle.full_rank import solve_pn_full

        o = mk()
        t0 = time.perf_counter()
        solve_pn_full(o, max_steps=head)
        per = (time.perf_counter() - t0) / head
        steps = o.csd.eTrafo.size - 1
        return per * steps, (f"FP64 oracle, full-rank P_N: {head} energy steps timed, x {steps} steps "
                             f"(constant cost per step)"), None
    if w["method"] == "pn3d":
        from oracle.csd import CSD
        from oracle.three_d import Settings3D as OSettings3D
        from oracle.three_d import SolverCSD3D as OSolver3D
        from oracle.three_d import solve_pn_full_3d

        # one oracle step on 96^3 cells takes minutes: time steps on the same problem
        # at half the resolution and scale by the cell count (the step's cost is
        # linear in the cells) and the full grid's step count
        nfull = w["Nx"] - 1
        nh = max(8, nfull // 2)
        o = OSolver3D(OSettings3D(nh + 1, nh + 1, nh + 1, w["r"], w["problem"], nPN=w["nPN"]))
        k = 2
        t0 = time.perf_counter()
        solve_pn_full_3d(o, max_steps=k)
        per = (time.perf_counter() - t0) / k * (nfull / nh) ** 3
        steps = CSD(OSettings3D(w["Nx"], w["Nx"], w["Nx"], w["r"], w["problem"], nPN=w["nPN"])).eTrafo.size - 1
        return per * steps, (f"FP64 oracle, 3D full-rank P_N: {k} energy steps timed on the {nh}^3 grid, "
                             f"x ({nfull}/{nh})^3 cells, x {steps} steps (cost linear in cells, constant per step)"), None
    fn = {"bug": solve_dlr_bug, "bug3d": solve_dlr_bug, "parallel": solve_dlr_parallel,
          "fixed": solve_dlr_fixed}[w["method"]]
    if w["method"] == "fixed":
        o = mk()
        t0 = time.perf_counter()
        fn(o, max_steps=head)
        per = (time.perf_counter() - t0) / head
        steps = o.csd.eTrafo.size - 1
        return per * steps, (f"FP64 oracle, fixed rank: {head} energy steps timed, x {steps} steps "
                             f"(constant cost per step)"), None
    clock = _IterClock()
    if w["method"] == "bug3d":
        # one oracle iteration on 96^3 cells takes tens of seconds: the opening
        # iterations only, their per-rank times carried over the GPU's rank history
        fn(mk(), max_steps=3, on_iter=clock)
        total, direct = _cost_of_history(clock.by_rank, ranks)
        measured = {r: len(v) for r, v in sorted(clock.by_rank.items())}
        return total, (f"FP64 oracle (BUG, 3D), per-iteration times of iterations 1-3 by rank ({measured}), "
                       f"summed over the {len(ranks)} iterations of the GPU solve's rank history; "
                       f"{100 * direct:.1f}% of those at a directly timed rank, the rest take the nearest "
                       f"timed rank's cost"), None
    fn(mk(), max_steps=head, on_iter=clock)
    if state200 is None:
        state200 = fn(mk(), max_steps=200, return_state=True)
    fn(mk(), max_steps=tail, state=state200, n_begin=state200["n_next"], on_iter=clock)
    total, direct = _cost_of_history(clock.by_rank, ranks)
    measured = {r: len(v) for r, v in sorted(clock.by_rank.items())}
    return total, (f"FP64 oracle ({w['method']}), per-iteration times at each rank measured on iterations "
                   f"1-{head} and 201-{200 + tail} (rank: iterations timed {measured}), summed over the "
                   f"{len(ranks)} iterations of the GPU solve's rank history; {100 * direct:.1f}% of those "
                   f"iterations at a directly timed rank, the rest interpolated in the rank"), state200


# ------------------------------------------------------------- GPU solve arm
def dose_error_vs_fixture(solver, lib, method_id):
    """Relative L2 error (interior cells) of the first 200 BUG iterations of the
    benchmark problem against the FP64 oracle's dose for them."""
    import numpy as np

    if not os.path.exists(FIXTURE):
        return None
    fx = np.load(FIXTURE)
    out = solver.run(method_id, max_steps=int(fx["iters"]))
    ref = fx["dose"]
    nx = int(fx["nx"]) - 1
    i, j = np.divmod(np.arange(nx * nx), nx)
    inner = (i > 0) & (j > 0) & (i < nx - 1) & (j < nx - 1)
    err = float(np.linalg.norm(out["dose"][inner] - ref[inner]) / np.linalg.norm(ref[inner]))
    same = bool(np.array_equal(out["rank_history"][:int(fx["iters"])], fx["ranks"]))
    return {"iterations": int(fx["iters"]), "dose_rel_l2_interior": err, "ranks_equal": same}


def run_gpu_solve(args, w, rank, world, local_rank, dist):
    import numpy as np
    import torch

    from titus_b200 import Settings, Settings3D, SolverCSD, SolverCSD3D
    from titus_b200 import _lib
    from titus_b200.replicas import replica_throughput

    method = {"fixed": _lib.TITUS_DLR_FIXED, "bug": _lib.TITUS_BUG_ADAPTIVE, "bug3d": _lib.TITUS_BUG_ADAPTIVE,
              "parallel": _lib.TITUS_PARALLEL_ADAPTIVE}[w["method"]]
    three_d = w["method"] == "bug3d"
    if three_d:
        s = Settings3D(w["Nx"], w["Nx"], w["Nx"], w["r"], w["problem"], nPN=w["nPN"])
        solver = SolverCSD3D(s, team_ctas=args.team)
    else:
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
    # device time of each solve (one launch of the energy-loop kernel plus its
    # state reset) on the launching stream
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
    ranks_hist = bufs["rank_history"][:int(res.steps_done)].copy()

    # end to end: one-shot C-ABI call with host buffers (upload, solve, copy-out, free)
    p, keep = solver.problem_struct()
    ext = None
    if three_d:
        ext = _lib.Problem3D()
        ext.nz, ext.dz = s.NCellsZ, s.dz
        for d, (rp, ci, v) in enumerate(solver.ops3):
            keep += [rp, ci, v]
            ext.op_rowptr[d], ext.op_col[d], ext.op_val[d] = _lib.as_ip(rp), _lib.as_ip(ci), _lib.as_dp(v)
    h2d = sum(a.nbytes for a in keep)
    res2, bufs2 = solver._result(s.r)
    d2h = sum(b.nbytes for b in bufs2.values())
    e2e_steps = max(1, min(args.steps, 3))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        if three_d:
            # one-shot: titus_create_3d, titus_solve, titus_destroy
            h2 = C.c_void_p()
            _lib.check(lib.titus_create_3d(C.byref(p), C.byref(ext), C.byref(h2)), "titus_create_3d")
            rc = lib.titus_solve(h2, method, C.byref(opt), C.byref(res2))
            lib.titus_destroy(h2)
            _lib.check(rc, "titus_solve")
        else:
            _lib.check(lib.titus_solve_problem(C.byref(p), method, C.byref(opt), C.byref(res2)),
                       "titus_solve_problem")
    t_e2e = time.perf_counter() - t0
    e2e_value, t_e2e = replica_throughput(e2e_steps, t_e2e, world, device="cuda")

    n, q = solver.n, solver.q
    steps_per_solve = int(res.steps_done)
    if w["method"] == "fixed":
        alg_bytes = algorithmic_bytes_per_step(n, s.r, q) * steps_per_solve
    else:
        alg_bytes = algorithmic_bytes_adaptive(n, ranks_hist[ranks_hist >= 0], q)
    traffic_step = DRAM_BYTES_PER_STEP_NCU.get(w["method"])
    achieved = alg_bytes / (t_max / args.steps) / 1e9
    peak, peak_kind = read_peaks()
    acc = dose_error_vs_fixture(solver, lib, method) if w["method"] == "bug" else None
    info = dict(value=value, ms_per_step=ms_per_step, e2e_value=e2e_value, h2d=h2d, d2h=d2h, n=n, q=q,
                N=solver.N, steps_per_solve=steps_per_solve, alg_bytes=alg_bytes, achieved=achieved,
                peak=peak, peak_kind=peak_kind, traffic_step=traffic_step, clocks=clk.summary(),
                rank_final=int(res.rank), dose_max=float(np.max(bufs["dose"])), accuracy=acc,
                ranks=ranks_hist, r=s.r)
    solver.close()
    return info


# ------------------------------------------------------- full-rank P_N arm
def run_gpu_pn_full(args, w, rank, world, local_rank, dist):
    """Full-rank P_N solve (SolveFirstCollisionSource): one captured graph of
    three kernels per energy step; value times the graph launch with CUDA events."""
    import numpy as np
    import torch

    from titus_b200 import Settings, Settings3D, SolverCSD, SolverCSD3D, _lib
    from titus_b200.replicas import replica_throughput

    three_d = w["method"] == "pn3d"
    if three_d:
        solver = SolverCSD3D(Settings3D(w["Nx"], w["Nx"], w["Nx"], w["r"], w["problem"], nPN=w["nPN"]))
    else:
        solver = SolverCSD(Settings(w["Nx"], w["Nx"], w["r"], w["problem"], nPN=w["nPN"]))
    lib = _lib.load()
    h = solver.handle()
    opt = solver.options()
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def solve_once():
        _lib.check(lib.titus_pn_full_solve_device(h, C.byref(opt), C.c_void_p(stream.cuda_stream)),
                   "titus_pn_full_solve_device")

    for _ in range(args.warmup):
        solve_once()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    elapsed = 0.0
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
    value, t_max = replica_throughput(args.steps, elapsed, world, device="cuda")
    dose = np.zeros(solver.n)
    _lib.check(lib.titus_pn_full_fetch(h, None, _lib.as_dp(dose), None), "titus_pn_full_fetch")
    # end to end: upload, solve, u/dose/psi copy-out, free
    p, keep = solver.problem_struct()
    ext = None
    if three_d:
        ext = _lib.Problem3D()
        ext.nz, ext.dz = solver.settings.NCellsZ, solver.settings.dz
        for d, (rp, ci, v) in enumerate(solver.ops3):
            keep += [rp, ci, v]
            ext.op_rowptr[d], ext.op_col[d], ext.op_val[d] = _lib.as_ip(rp), _lib.as_ip(ci), _lib.as_dp(v)
    h2d = sum(a.nbytes for a in keep)
    u = np.zeros((solver.n, solver.N))
    psi = np.zeros((solver.n, solver.q))
    d2h = u.nbytes + dose.nbytes + psi.nbytes
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h2 = C.c_void_p()
    if three_d:
        _lib.check(lib.titus_create_3d(C.byref(p), C.byref(ext), C.byref(h2)), "titus_create_3d")
    else:
        _lib.check(lib.titus_create(C.byref(p), C.byref(h2)), "titus_create")
    rc = lib.titus_pn_full_solve(h2, C.byref(opt), _lib.as_dp(u), _lib.as_dp(dose), _lib.as_dp(psi))
    lib.titus_destroy(h2)
    _lib.check(rc, "titus_pn_full_solve")
    e2e_value, _ = replica_throughput(1, time.perf_counter() - t0, world, device="cuda")
    steps = solver.nE - 1
    nN = solver.n * solver.N
    if three_d:
        # per step, the fused stencil + moment kernel reads u and writes u' (2 nN); psi is
        # written by the sweep and read by the sweep and the stream kernel (3 n q); the
        # dose is read and written and 1/rho read once (3 n)
        alg = steps * 8 * (2 * nN + 3 * solver.n * solver.q + 3 * solver.n)
    else:
        # per step: moments read u, write W (5 nN); stream reads u, W (4 nN), writes u' (6 nN);
        # psi read + write (2 n q), dose read + write (2 n)
        alg = steps * 8 * (11 * nN + 2 * solver.n * solver.q + 2 * solver.n)
    peak, peak_kind = read_peaks()
    achieved = alg / (t_max / args.steps) / 1e9
    info = dict(value=value, ms_per_step=t_max / args.steps * 1e3, e2e_value=e2e_value, h2d=h2d, d2h=d2h,
                alg=alg, achieved=achieved, peak=peak, peak_kind=peak_kind, clocks=clk.summary(),
                dose_max=float(dose.max()), steps_per_solve=steps, q=solver.q, n=solver.n, N=solver.N)
    solver.close()
    return info


# ------------------------------------------------------------ batched plan
def batched_team(args, solver):
    """Team size (CTAs per spot) of the batched plan: --team-batched if given,
    else the tuned choice for this problem shape (titus_b200.autotune), else 1."""
    if args.team_batched > 0:
        return args.team_batched, "argument"
    try:
        from titus_b200.autotune import lookup

        t = lookup(solver)
        if t:
            return t, "tuned table"
    except ImportError:
        pass
    return 1, "default"


def run_gpu_batched(args, rank, world, local_rank, dist, steps, warmup, short_warmup=False, iters=0):
    """The 256-spot pencil-beam plan sharded by spot over the ranks: each step is
    one persistent launch of this rank's spots (device-resident tables), timed
    with CUDA events; e2e adds the host tables, upload, dose copy-back and the
    SUM all-reduce of the weighted total dose (spots.plan_dose). `iters` > 0
    bounds every spot to its first `iters` loop iterations (the same bound for
    batched and plain, so their ratio compares equal work)."""
    import numpy as np
    import torch

    from titus_b200 import Settings, SolverCSD, _lib
    from titus_b200.replicas import max_over_ranks
    from titus_b200.spots import partition, plan_dose

    cfg = BATCHED
    s = Settings(cfg["Nx"], cfg["Nx"], cfg["r"], cfg["problem"], nPN=cfg["nPN"])
    solver = SolverCSD(s)
    spots = batched_spots(cfg)
    idx = partition(len(spots), world, rank)
    local = [spots[i] for i in idx]
    team, team_src = batched_team(args, solver)
    batch = solver.batch(local)
    stream = torch.cuda.current_stream()
    for i in range(warmup):
        batch.solve_device(_lib.TITUS_BUG_ADAPTIVE, team, max_steps=50 if short_warmup else 0,
                           stream=stream.cuda_stream)
        batch.fetch(want_dose=False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    elapsed = 0.0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(steps, 1)):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.solve_device(_lib.TITUS_BUG_ADAPTIVE, team, max_steps=iters, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        elapsed += e0.elapsed_time(e1) / 1e3
    nsteps = max(steps, 1)
    t_max = max_over_ranks(elapsed / nsteps, device="cuda")
    dose_b, rank_b, it_b = batch.fetch()
    rsum = batch.rank_sums()
    value = len(spots) / t_max
    # plain companion: this rank's two shortest spots solved one at a time on all SMs
    order = np.argsort(batch.n_energies)[:2]
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    t0 = time.perf_counter()
    plain_it = 0
    max_rel = 0.0
    for i in order:
        d, _, it = solver.solve_batched([local[i]], _lib.TITUS_BUG_ADAPTIVE, team_ctas=sms, max_steps=iters)
        plain_it += int(it[0])
        max_rel = max(max_rel, float(np.linalg.norm(d[0] - dose_b[i]) / np.linalg.norm(dose_b[i])))
    t_plain_sample = time.perf_counter() - t0
    per_it = t_plain_sample / plain_it
    tot_it = float(np.sum(it_b))
    if dist:
        t = torch.tensor([tot_it, per_it], dtype=torch.float64, device="cuda")
        dist.all_reduce(t[:1])
        tot_it = float(t[0].item())
        per_it = max_over_ranks(per_it, device="cuda")
    t_plain = per_it * tot_it
    # end to end: host tables, upload, solve, dose copy-back, SUM all-reduce of the total dose
    weights = np.ones(len(spots))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    total, _, _ = plan_dose(solver, spots, weights, "bug", team, max_steps=iters, device="cuda")
    t_e2e = max_over_ranks(time.perf_counter() - t0, device="cuda")
    n, q = solver.n, solver.q
    alg = float(sum(algorithmic_bytes_per_step(n, 2.0 * rs / max(1, it), q) * it for rs, it in zip(rsum, it_b)))
    if dist:
        t = torch.tensor([alg], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        alg = float(t.item())
    peak, peak_kind = read_peaks()
    achieved = alg / t_max / 1e9
    out = {
        "workload": cfg["name"] + (f"_first{iters}iters" if iters else ""), "spots": len(spots),
        "iterations_per_spot_bound": iters or None, "team_ctas": team, "team_source": team_src,
        "value": value, "unit": "solves/s", "seconds": t_max, "steps": nsteps,
        "iterations_total": int(tot_it), "spot_steps_per_s": tot_it / t_max,
        "plain": {"value": len(spots) / t_plain, "seconds_estimated": t_plain, "seconds_per_iteration": per_it,
                  "team_ctas": sms, "sample": f"{len(order)} shortest spots of each rank solved one at a time "
                                              f"({plain_it} iterations, same bound), scaled by the plan's "
                                              f"iterations"},
        "batched_over_plain": t_plain / t_max,
        "max_rel_dose_diff_batched_vs_plain": max_rel,
        "e2e": {"value": len(spots) / t_e2e, "unit": "solves/s", "seconds": t_e2e,
                "includes": "host tables, upload, solve, dose copy-back, total-dose SUM all-reduce"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg},
        "total_dose_max": float(np.max(total)),
    }
    batch.close()
    solver.close()
    return out


# --------------------------------------------------------- reference arm
def _ranks_for(w):
    """The GPU solve's rank per iteration (fixture written by
    tests/golden/make_rank_history.py), for the CPU cost model."""
    import numpy as np

    if w["method"] in ("bug", "parallel") and os.path.exists(RANKS_FIXTURE):
        return np.load(RANKS_FIXTURE)["ranks"].astype(np.int64)
    return None


def batched_reference_seconds(cfg=BATCHED, head=40, tail=20):
    """FP64 oracle time of the whole 256-spot plan: one spot of median energy
    timed on iterations 1..head and on `tail` iterations from its state after
    200; each spot is then charged the opening window plus the tail's mean
    time per iteration for the rest of its energy grid (nE - 2 iterations,
    rejections not counted)."""
    import numpy as np

    from oracle.settings import Settings as OSettings
    from oracle.solver import SolverCSD as OSolver
    from oracle.solver import solve_dlr_bug
    from titus_b200.physics import energy_grid

    spots = batched_spots(cfg)
    e_med = float(np.median([e for e, _ in spots]))

    def mk(e=e_med, y=0.5):
        s = OSettings(cfg["Nx"], cfg["Nx"], cfg["r"], cfg["problem"], nPN=cfg["nPN"])
        s.eMax, s.y0 = e, y
        return s

    solve_dlr_bug(OSolver(mk()), max_steps=3)   # untimed: first-call costs
    t0 = time.perf_counter()
    solve_dlr_bug(OSolver(mk()), max_steps=head)
    t_head = time.perf_counter() - t0
    st = solve_dlr_bug(OSolver(mk()), max_steps=200, return_state=True)
    t0 = time.perf_counter()
    solve_dlr_bug(OSolver(mk()), max_steps=tail, state=st, n_begin=st["n_next"])
    per = (time.perf_counter() - t0) / tail
    total = 0.0
    for e, y in spots:
        s = mk(e, y)
        nE = energy_grid(s)[1].size
        total += t_head + per * max(0, nE - 2 - head)
    return total, (f"FP64 oracle, one {e_med:.2f} MeV spot: iterations 1-{head} ({t_head:.2f} s) and "
                   f"{tail} iterations after 200 ({per * 1e3:.1f} ms each); every spot charged the opening "
                   f"plus nE-2-{head} iterations at that rate")


def host_threads():
    """Use every host core for the oracle's BLAS/LAPACK calls (a launcher such as
    torch.distributed.run sets OMP_NUM_THREADS=1 for its ranks)."""
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    try:
        from threadpoolctl import threadpool_limits

        threadpool_limits(limits=cores)
    except ImportError:
        pass
    return cores


def run_reference(args, w, rank):
    if rank != 0:
        return
    cores = host_threads()
    line = {"impl": "reference", "metric": "dose solves/s", "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    if args.method == "batched":
        cfg = BATCHED
        for _ in range(args.warmup):
            batched_reference_seconds(cfg)
        ts = []
        for _ in range(args.steps):
            t, sample = batched_reference_seconds(cfg)
            ts.append(t)
        t_plan = sum(ts) / len(ts)
        v = cfg["spots"] / t_plan
        line.update({"value": v, "ms_per_step": t_plan * 1e3,
                     "config": batched_config(cfg, world=args.gpus)})
    else:
        ranks = _ranks_for(w)
        if ranks is None and w["method"] not in ("fixed", "pn_full", "pn3d"):
            print(json.dumps({"impl": "reference", "unavailable": "rank-history fixture missing: run "
                              "tests/golden/make_rank_history.py on a GPU"}), flush=True)
            return
        state = None
        for _ in range(args.warmup):
            _, _, state = cpu_cost_model(w, ranks, state)
        ts = []
        for _ in range(args.steps):
            t, sample, state = cpu_cost_model(w, ranks, state)
            ts.append(t)
        t_solve = sum(ts) / len(ts)
        v = 1.0 / t_solve
        line.update({"value": v, "ms_per_step": t_solve * 1e3,
                     "config": solve_config(w, iterations=len(ranks) if ranks is not None else None,
                                            world=args.gpus)})
    line["cpu_baseline"] = {"value": v, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample}
    line["e2e"] = {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line), flush=True)


def solve_config(w, iterations=None, world=1, team=148):
    """The `config` dict both arms print for a single-solve workload."""
    cells = (w["Nx"] - 1) ** (3 if w["method"] == "pn3d" else 2)
    cfg = {"workload": w["name"], "cells": cells, "moments": (w["nPN"] + 1) ** 2, "method": w["method"],
           "parallelism": f"replicas{world}", "l2": "flushed between solves (256 MB write)"}
    if w["method"] not in ("pn_full", "pn3d"):
        cfg["rank_cap" if w["method"] != "fixed" else "rank"] = w["r"]
    if iterations is not None:
        cfg["loop_iterations"] = int(iterations)
    return cfg


def batched_config(cfg, world=1):
    return {"workload": cfg["name"], "spots": cfg["spots"], "cells": (cfg["Nx"] - 1) ** 2,
            "moments": (cfg["nPN"] + 1) ** 2, "rank_cap": cfg["r"], "method": "bug",
            "energies_MeV": f"U({cfg['emin']},{cfg['emax']})", "y0": f"U({cfg['ymin']},{cfg['ymax']})",
            "seed": cfg["seed"], "parallelism": f"spots sharded over {world} rank(s)",
            "l2": "flushed between launches (256 MB write)"}


# ------------------------------------------------------------------ driver
def run_gpu(args, w, rank, world, local_rank):
    import datetime

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    line = None
    if args.method == "batched":
        b = run_gpu_batched(args, rank, world, local_rank, dist, args.steps, args.warmup)
        if rank == 0:
            line = {"metric": "dose solves/s", "value": b["value"], "unit": "solves/s", "n_gpus": world,
                    "steps": b["steps"], "warmup": args.warmup, "ms_per_step": b["seconds"] * 1e3,
                    "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic", "config": batched_config(BATCHED, world),
                    "e2e": {"value": b["e2e"]["value"], "unit": "solves/s", "h2d_bytes_per_step": None,
                            "d2h_bytes_per_step": None},
                    "roofline": b["roofline"], "batched": b, "gpu_launches": args.steps}
            if world == 1 and not args.no_cpu_baseline:
                cores = host_threads()
                t, sample = batched_reference_seconds(BATCHED)
                line["cpu_baseline"] = {"value": BATCHED["spots"] / t, "unit": "solves/s",
                                        "cores": cores, "kind": "port", "sample": sample}
    elif args.method in ("pn_full", "pn3d"):
        info = run_gpu_pn_full(args, w, rank, world, local_rank, dist)
        if rank == 0:
            line = {"metric": "dose solves/s", "value": info["value"], "unit": "solves/s", "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": info["ms_per_step"],
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic",
                    "config": dict(solve_config(w, info["steps_per_solve"], world), ordinates=info["q"]),
                    "e2e": {"value": info["e2e_value"], "unit": "solves/s", "h2d_bytes_per_step": int(info["h2d"]),
                            "d2h_bytes_per_step": int(info["d2h"])},
                    "roofline": {"bound": "hbm", "achieved": info["achieved"], "peak": info["peak"], "unit": "GB/s",
                                 "frac": info["achieved"] / info["peak"], "traffic": None,
                                 "peak_kind": info["peak_kind"], "algorithmic_bytes_per_launch": info["alg"],
                                 "note": "all kernels of every energy step (one graph launch)"},
                    "clocks": info["clocks"],
                    "gpu_launches": (2 if args.method == "pn3d" else 3) * info["steps_per_solve"] * args.steps,
                    "dose_max": info["dose_max"], "cpu_baseline": None}
            if world == 1 and not args.no_cpu_baseline:
                cores = host_threads()
                t, sample, _ = cpu_cost_model(w, None)
                line["cpu_baseline"] = {"value": 1.0 / t, "unit": "solves/s", "cores": cores, "kind": "port",
                                        "sample": sample}
    else:
        info = run_gpu_solve(args, w, rank, world, local_rank, dist)
        batched = None
        if not args.no_batched:
            batched = run_gpu_batched(args, rank, world, local_rank, dist, 1, 1, short_warmup=True,
                                      iters=BATCHED_SAMPLE_ITERS)
        if rank == 0:
            peak = info["peak"]
            line = {
                "metric": "dose solves/s", "value": info["value"], "unit": "solves/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": info["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": dict(solve_config(w, info["steps_per_solve"], world), ordinates=info["q"],
                               team_ctas=args.team or "default"),
                "e2e": {"value": info["e2e_value"], "unit": "solves/s", "h2d_bytes_per_step": int(info["h2d"]),
                        "d2h_bytes_per_step": int(info["d2h"])},
                "roofline": {"bound": "hbm", "achieved": info["achieved"], "peak": peak, "unit": "GB/s",
                             "frac": info["achieved"] / peak,
                             "traffic": (info["traffic_step"] * info["steps_per_solve"]
                                         if info["traffic_step"] else None),
                             "traffic_note": "ncu capture of the first energy steps scaled to the launch's steps",
                             "peak_kind": info["peak_kind"], "algorithmic_bytes_per_launch": info["alg_bytes"]},
                "cpu_baseline": None,
                "clocks": info["clocks"],
                # per solve: the state-reset kernel(s) and the energy-loop kernel
                "gpu_launches": (2 if w["method"] != "parallel" else 3) * args.steps,
                "rank_final": info["rank_final"], "dose_max": info["dose_max"],
                "dose_rel_err_vs_oracle": info["accuracy"],
            }
            if batched is not None:
                line["batched"] = batched
            if world == 1 and not args.no_cpu_baseline:
                cores = host_threads()
                t, sample, _ = cpu_cost_model(w, info["ranks"])
                line["cpu_baseline"] = {"value": 1.0 / t, "unit": "solves/s", "cores": cores, "kind": "port",
                                        "sample": sample}
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def relaunch(args_list, n):
    """Re-run this script as n ranks under torch.distributed.run (one per GPU)."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__), *args_list]
    return subprocess.call(cmd)


def run_dry(args, rank, world):
    """CPU stand-in of the multi-rank path (gloo): each rank 'solves' its spots
    with a synthetic dose, the total goes through the same SUM all-reduce and
    max-over-ranks timing, and rank 0 prints the line shape."""
    import datetime

    import numpy as np
    import torch.distributed as dist

    from titus_b200.replicas import replica_throughput
    from titus_b200.spots import plan_dose

    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))

    class Stand:
        n = 64

    def fake(sv, sp, m, t, k):
        c = np.arange(sv.n)
        return np.array([e * np.exp(-((c - y * sv.n) / 5.0) ** 2) for e, y in sp])

    t0 = time.perf_counter()
    total, idx, _ = plan_dose(Stand(), batched_spots(BATCHED, 16), None, solve=fake)
    value, t = replica_throughput(args.steps, time.perf_counter() - t0, world)
    if rank == 0:
        print(json.dumps({"metric": "dose solves/s", "value": value, "unit": "solves/s", "n_gpus": world,
                          "steps": args.steps, "dry_run": True, "total_dose_sum": float(total.sum()),
                          "spots_rank0": int(idx.size)}), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--method", default="bug", choices=sorted(WORKLOADS) + ["batched"])
    ap.add_argument("--team", type=int, default=148, help="CTAs per solve (0 = library default)")
    ap.add_argument("--size", type=int, default=0, help="cells per axis of the 3D workloads (default 96)")
    ap.add_argument("--team-batched", type=int, default=0, help="CTAs per spot of the batched plan (0 = tuned)")
    ap.add_argument("--impl", default="titus", choices=["titus", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-plan measurement")
    ap.add_argument("--dry-run", action="store_true", help="CPU stand-in of the multi-rank path (gloo)")
    args = ap.parse_args()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(relaunch(sys.argv[1:], args.gpus))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    w = three_d_workload(WORKLOADS.get(args.method, WORKLOADS["bug"]), args.size)
    if args.dry_run:
        run_dry(args, rank, world)
    elif args.impl == "reference":
        run_reference(args, w, rank)
    else:
        run_gpu(args, w, rank, world, local_rank)


if __name__ == "__main__":
    main()
