"""Per-phase device timer breakdown of one solve of a benchmark workload.

    python -m titus_b200.profile_phases [--nx 101] [--npn 21] [--r 20] [--steps 200] [--team 0]
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
    a = ap.parse_args()
    s = Settings(a.nx, a.nx, a.r, a.problem, nPN=a.npn)
    g = SolverCSD(s, team_ctas=a.team)
    g.run(_lib.TITUS_DLR_FIXED, max_steps=5)
    t0 = time.perf_counter()
    g.run(_lib.TITUS_DLR_FIXED, max_steps=a.steps, profile=True)
    wall = time.perf_counter() - t0
    prof = g.profile()
    per_step = {k: v / a.steps / 1e3 for k, v in prof.items()}
    print(json.dumps({"workload": vars(a), "wall_s": wall, "us_per_step": per_step}))


if __name__ == "__main__":
    main()
