"""``Settings`` of the benchmark problems (mirror of ``code/settings.jl:5-338``).

Field names follow the reference struct; callers may overwrite fields after
construction exactly as the reference's drivers do (``runLungParallel.jl:23``).
The problems are the analytic-physics benchmark cases:

* ``"csdWaterBeam"`` -- 2D water slab [0,1]^2 cm, pencil beam along +x entering
  at x = 0, y0 = 0.5, spatial sigma 0.05 cm, angular sigma 0.01 rad, 5 MeV
  electrons, S(E) = 0.2/E ln(1 + 10 E), Henyey-Greenstein sigma_l = 100 * 0.9^l.
* ``"csdPhantom"`` -- the same beam on a seeded water / lung / bone phantom.

The energy-step count follows the explicit scheme's stability bound in
transformed energy (``tau_cfl``), see ``titus_b200.physics.energy_grid``.
"""
from __future__ import annotations

import math

import numpy as np

BENCHMARK_PROBLEMS = ("csdWaterBeam", "csdPhantom")


def seeded_phantom(ncx, ncy, a, b, c, d, seed, n_lung=3, n_bone=1, rho_water=1.0, rho_lung=0.25,
                   rho_bone=1.85, rmin=0.05, rmax=0.2):
    """Water background with random lung and bone ellipses from ``default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    X, Y = np.meshgrid(np.linspace(a, b, ncx), np.linspace(c, d, ncy), indexing="ij")
    rho = np.full((ncx, ncy), rho_water)
    for val in [rho_lung] * n_lung + [rho_bone] * n_bone:
        cx = rng.uniform(a + 0.1 * (b - a), b - 0.1 * (b - a))
        cy = rng.uniform(c + 0.1 * (d - c), d - 0.1 * (d - c))
        ra, rb = rng.uniform(rmin, rmax), rng.uniform(rmin, rmax)
        th = rng.uniform(0.0, math.pi)
        u = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
        v = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
        rho[(u / ra) ** 2 + (v / rb) ** 2 <= 1.0] = val
    return rho


class Settings:
    """``Settings(Nx, Ny, r, problem, particle)`` (``settings.jl:67``)."""

    def __init__(self, Nx: int = 101, Ny: int = 101, r: int = 20, problem: str = "csdWaterBeam",
                 particle: str = "Electrons", nPN: int | None = None, nEnergies: int = 0,
                 seed: int = 20240601, tau_cfl: float = 0.5):
        if problem not in BENCHMARK_PROBLEMS:
            raise ValueError(f"problem {problem!r} not available; choose one of {BENCHMARK_PROBLEMS}")
        self.Nx, self.Ny = Nx, Ny
        self.NCellsX, self.NCellsY = Nx - 1, Ny - 1
        self.a, self.b, self.c, self.d = 0.0, 1.0, 0.0, 1.0
        self.problem, self.particle = problem, particle
        self.eRest = 938.26 if particle == "Protons" else 0.5
        self.eMax, self.eMin = 5.0, 0.001
        self.x0, self.y0 = 0.0, 0.5
        self.Omega1, self.Omega3 = 1.0, 0.0
        self.densityMin = 1.0
        self.sigmaXInv = self.sigmaYInv = 1.0 / (2 * 0.05**2)
        self.sigmaO1Inv = self.sigmaO3Inv = 1.0 / (2 * 0.01**2)
        self.sigmaEInv = 100.0
        self.psi_scale = 1e5
        self.beam_peak_normalized = True
        self.stopping = "electron_log"
        self.hg_g, self.sigmaT_hg = 0.9, 100.0
        self.seed = seed
        self.r = r
        self.theta, self.thetaIndex, self.c_eta = 1e-2, 1.0, 5.0
        self.nPN = 21 if nPN is None else nPN
        self.nEnergies = nEnergies
        self.tau_cfl = tau_cfl
        self.cfl = 0.5
        ncx, ncy = self.NCellsX, self.NCellsY
        if problem == "csdPhantom":
            self.density = seeded_phantom(ncx, ncy, self.a, self.b, self.c, self.d, seed)
        else:
            self.density = np.ones((ncx, ncy))
        # grid with ghost shift, settings.jl:315-325 (xMid spans [a, b])
        x = np.linspace(self.a, self.b, ncx)
        self.dx = x[1] - x[0]
        x = np.concatenate([[x[0] - self.dx], x]) + self.dx / 2
        self.x, self.xMid = x, x[:-1] + 0.5 * self.dx
        y = np.linspace(self.c, self.d, ncy)
        self.dy = y[1] - y[0]
        y = np.concatenate([[y[0] - self.dy], y]) + self.dy / 2
        self.y, self.yMid = y, y[:-1] + 0.5 * self.dy
        self.dE = self.cfl * min(self.dx, self.dy) * self.density.min()
