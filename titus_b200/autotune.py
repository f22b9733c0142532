"""Team-size tuner for batched pencil-beam solves.

    python -m titus_b200.autotune [--nx 129 --npn 21 --cap 60 --spots 148 --steps 300]

A batched launch runs T teams of G CTAs (G CTAs per spot, T = SMs / G teams at
a time, one CTA per SM because of the kernel's shared memory). Small teams run
more spots at once but each spot's energy step takes longer; which G gives the
most spot-steps per second depends on the grid, the moment count and the
ranks the spots reach. The tuner launches the first `steps` loop iterations of
`spots` seeded spots (energies U(2, 8) MeV) for each candidate G, measures
spot-iterations per second, and records the best G in
``tuning/batched.json`` keyed by the problem shape and the GPU name.
``lookup`` returns the recorded choice (None if the shape was never tuned).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning", "batched.json")
CANDIDATES = (1, 2, 4, 8)


def shape_key(solver, gpu_name: str | None = None) -> str:
    if gpu_name is None:
        import torch

        gpu_name = torch.cuda.get_device_name(0) if torch.cuda.is_available() else "cpu"
    s = solver.settings
    return f"{s.NCellsX}x{s.NCellsY}_N{solver.N}_q{solver.q}_cap{s.r}|{gpu_name}"


def load_table(path: str = TABLE) -> dict:
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def lookup(solver, path: str = TABLE, gpu_name: str | None = None):
    """Recorded team size for this solver's shape on this GPU, or None."""
    ent = load_table(path).get(shape_key(solver, gpu_name))
    return int(ent["team_ctas"]) if ent else None


def tune(solver, spots, steps: int = 300, candidates=CANDIDATES, method=None):
    """Measure spot-iterations/s of a `steps`-iteration batched launch of
    `spots` for each team size; returns (best G, {G: rate})."""
    import torch

    from . import _lib

    method = _lib.TITUS_BUG_ADAPTIVE if method is None else method
    batch = solver.batch(spots)
    rates = {}
    batch.solve_device(method, 1, max_steps=5)   # module load, allocations
    batch.fetch(want_dose=False)
    for g in candidates:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        batch.solve_device(method, g, max_steps=steps)
        _, _, it = batch.fetch(want_dose=False)
        torch.cuda.synchronize()
        rates[g] = float(np.sum(it)) / (time.perf_counter() - t0)
    batch.close()
    best = max(rates, key=rates.get)
    return best, rates


def record(solver, best: int, rates: dict, steps: int, nspots: int, path: str = TABLE) -> None:
    tab = load_table(path)
    tab[shape_key(solver)] = {"team_ctas": int(best), "spot_iterations_per_s": {str(k): v for k, v in rates.items()},
                              "probe": f"{nspots} spots x {steps} iterations"}
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(tab, f, indent=1, sort_keys=True)


def main():
    from .settings import Settings
    from .solver import SolverCSD

    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=129)
    ap.add_argument("--npn", type=int, default=21)
    ap.add_argument("--cap", type=int, default=60)
    ap.add_argument("--spots", type=int, default=148)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--out", default=TABLE)
    a = ap.parse_args()
    rng = np.random.default_rng(a.seed)
    spots = [(float(e), float(y)) for e, y in zip(rng.uniform(2.0, 8.0, a.spots), rng.uniform(0.1, 0.9, a.spots))]
    sv = SolverCSD(Settings(a.nx, a.nx, a.cap, "csdPhantom", nPN=a.npn))
    best, rates = tune(sv, spots, a.steps)
    record(sv, best, rates, a.steps, a.spots, a.out)
    print(json.dumps({"key": shape_key(sv), "team_ctas": best, "spot_iterations_per_s": rates}))


if __name__ == "__main__":
    main()
