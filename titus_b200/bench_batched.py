"""Batched against plain pencil-beam solves on one GPU.

    python -m titus_b200.bench_batched [--nx 129 --npn 21 --cap 60 --spots 16 --team 9 --seed 3]

Spots are seeded: energies uniform in [2, 8] MeV, entry y0 uniform in
[0.1, 0.9] at x = 0, on the seeded 128 x 128 phantom (adaptive BUG, theta
1e-2, rank cap 60, P21): the pattern of 256-spot plans, on a subset of spots
that runs in minutes. "batched" is one ``titus_solve_batched`` launch in which
teams of ``--team`` CTAs take the spots; "plain" solves the same spots one
after the other, each with all SMs (one team). Both are timed end to end
through the Python API (host tables, upload, solve, dose copy back); the
solve kernels dominate. Prints one JSON line with both throughputs and the
largest relative difference between a spot's batched and plain dose.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _lib
from .settings import Settings
from .solver import SolverCSD


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=129)
    ap.add_argument("--npn", type=int, default=21)
    ap.add_argument("--cap", type=int, default=60)
    ap.add_argument("--spots", type=int, default=16)
    ap.add_argument("--team", type=int, default=9)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--skip-plain", action="store_true")
    a = ap.parse_args()
    rng = np.random.default_rng(a.seed)
    spots = [(float(e), float(y)) for e, y in zip(rng.uniform(2.0, 8.0, a.spots), rng.uniform(0.1, 0.9, a.spots))]
    sv = SolverCSD(Settings(a.nx, a.nx, a.cap, "csdPhantom", nPN=a.npn))
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    # warm-up: one short batched launch (module load, allocation)
    sv.solve_batched(spots[:1], _lib.TITUS_BUG_ADAPTIVE, team_ctas=a.team, max_steps=5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dose_b, rank_b, it_b = sv.solve_batched(spots, _lib.TITUS_BUG_ADAPTIVE, team_ctas=a.team)
    torch.cuda.synchronize()
    t_batched = time.perf_counter() - t0
    out = {"metric": "pencil-beam dose solves/s", "unit": "solves/s", "dtype": "f64",
           "config": {"workload": f"spots{a.spots}_phantom_{a.nx - 1}x{a.nx - 1}_P{a.npn}_cap{a.cap}_bug",
                      "energies_MeV": "U(2,8)", "y0": "U(0.1,0.9)", "seed": a.seed, "team_ctas": a.team,
                      "teams": max(1, sms // a.team)},
           "batched": {"seconds": t_batched, "value": a.spots / t_batched},
           "iterations_per_spot": [int(v) for v in it_b], "final_rank": [int(v) for v in rank_b]}
    if not a.skip_plain:
        t0 = time.perf_counter()
        dose_p = []
        for s in spots:
            d, _, _ = sv.solve_batched([s], _lib.TITUS_BUG_ADAPTIVE, team_ctas=sms)
            dose_p.append(d[0])
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
        dose_p = np.array(dose_p)
        rel = [float(np.linalg.norm(dose_b[i] - dose_p[i]) / np.linalg.norm(dose_p[i])) for i in range(a.spots)]
        out["plain"] = {"seconds": t_plain, "value": a.spots / t_plain, "team_ctas": sms}
        out["batched_over_plain"] = t_plain / t_batched
        out["max_rel_dose_diff_batched_vs_plain"] = max(rel)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
