"""Per-phase device timer breakdown of one solve of a benchmark workload.

    python -m titus_b200.profile_phases [--nx 101] [--npn 21] [--r 20] [--steps 200] [--team 0]
                                        [--method fixed|parallel|bug] [--problem csdWaterBeam]
                                        [--precision fp64|mixed] [--theta 1e-2]

Timers are exclusive (each cycle is charged to the innermost open phase) and
recorded on the first CTA; "total" is their sum.
"""
from __future__ import annotations

import argparse
import json
import time

from . import _lib
from .settings import Settings
from .solver import SolverCSD


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=101)
    ap.add_argument("--npn", type=int, default=21)
    ap.add_argument("--r", type=int, default=20)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--team", type=int, default=0)
    ap.add_argument("--problem", default="csdWaterBeam")
    ap.add_argument("--method", default="fixed", choices=["fixed", "parallel", "bug"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--theta", type=float, default=None, help="truncation tolerance (problem default if unset)")
    a = ap.parse_args()
    method = {"fixed": _lib.TITUS_DLR_FIXED, "parallel": _lib.TITUS_PARALLEL_ADAPTIVE,
              "bug": _lib.TITUS_BUG_ADAPTIVE}[a.method]
    s = Settings(a.nx, a.nx, a.r, a.problem, nPN=a.npn)
    if a.theta is not None:
        s.theta = a.theta
    prec = {"fp64": _lib.TITUS_PRECISION_FP64, "mixed": _lib.TITUS_PRECISION_MIXED}[a.precision]
    g = SolverCSD(s, team_ctas=a.team, precision=prec)
    g.run(method, max_steps=5)
    t0 = time.perf_counter()
    out = g.run(method, max_steps=a.steps, profile=True)
    wall = time.perf_counter() - t0
    prof = g.profile()
    steps = max(out["steps"], 1)
    counters = {k: prof.pop(k) for k in _lib.PROFILE_COUNTERS if k in prof}
    per_step = {k: v / steps / 1e3 for k, v in prof.items()}
    events = {k: v / steps for k, v in counters.items()}
    if counters.get("svd_calls"):
        events["svd_sweeps_per_call"] = counters["svd_sweeps"] / counters["svd_calls"]
    if counters.get("eig_calls"):
        events["eig_sweeps_per_call"] = counters["eig_sweeps"] / counters["eig_calls"]
    if counters.get("barriers") and "barrier" in prof:
        events["us_per_barrier_wait"] = prof["barrier"] / 1e3 / counters["barriers"]
    hist = out["rank_history"]
    print(json.dumps({"workload": vars(a), "steps": out["steps"], "rank": out["rank"],
                      "rank_max": int(hist.max()), "wall_s": wall, "us_per_step": per_step,
                      "events_per_step": events}))


if __name__ == "__main__":
    main()
