"""Timing of the limited-flux operator ``titus_limited_flux`` (solveFlux!).

    python -m titus_b200.bench_flux [--nx 2048 --ny 2048 --q 16 --steps 20 --warmup 3]

Prints one JSON line. ``value``: device bandwidth over ``steps`` back-to-back
launches, timed with CUDA events on the launching stream (phi and flux are each
larger than the 126 MB L2, so no flush is needed between launches).
Algorithmic bytes per launch: phi read once (8 nx ny q) and the interior flux
written once (8 (nx-4)(ny-4) q). ``e2e``: the host-array path, i.e. pinned
phi copied to the device, the flux computed and copied back, every step.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import _lib
from .flux import limited_flux_device

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f).get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--q", type=int, default=16)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args()
    _lib.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(7)
    shape = (a.nx, a.ny, a.q)
    phi = torch.rand(shape, dtype=torch.float64, device=dev, generator=g)
    flux = torch.zeros(shape, dtype=torch.float64, device=dev)
    ang = torch.linspace(0.1, 6.2, a.q, dtype=torch.float64, device=dev)
    ox, oz = torch.cos(ang), torch.sin(ang)   # all four sign quadrants
    dx = dy = 1.0 / (a.nx - 1)
    stream = torch.cuda.current_stream()
    for _ in range(a.warmup):
        limited_flux_device(phi, flux, ox, oz, dx, dy)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(a.steps):
        limited_flux_device(phi, flux, ox, oz, dx, dy)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / a.steps
    alg = 8.0 * a.nx * a.ny * a.q + 8.0 * max(a.nx - 4, 0) * max(a.ny - 4, 0) * a.q
    gbs = alg / (ms * 1e-3) / 1e9
    peak, kind = _peak()
    # end to end through host memory
    h_phi = phi.cpu().pin_memory()
    h_flux = torch.empty(shape, dtype=torch.float64).pin_memory()
    for _ in range(2):
        phi.copy_(h_phi, non_blocking=True)
        limited_flux_device(phi, flux, ox, oz, dx, dy)
        h_flux.copy_(flux, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        phi.copy_(h_phi, non_blocking=True)
        limited_flux_device(phi, flux, ox, oz, dx, dy)
        h_flux.copy_(flux, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / a.steps
    cells = a.nx * a.ny * a.q
    print(json.dumps({
        "metric": "limited-flux cell-ordinates/s", "value": cells / (ms * 1e-3), "unit": "cell-ordinates/s",
        "ms_per_step": ms, "steps": a.steps, "warmup": a.warmup, "dtype": "f64",
        "config": {"workload": f"limited_flux_{a.nx}x{a.ny}_q{a.q}", "l2": "inputs larger than L2"},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                     "peak_kind": kind, "algorithmic_bytes_per_launch": alg},
        "e2e": {"value": cells / (ms_e2e * 1e-3), "unit": "cell-ordinates/s", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": 8 * cells, "d2h_bytes_per_step": 8 * cells},
        "gpu_launches": a.steps,
    }))


if __name__ == "__main__":
    main()
