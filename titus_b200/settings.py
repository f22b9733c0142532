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


def seeded_spheres(ncx, ncy, ncz, L, seed, n_lung=3, n_bone=1, rho_water=1.0, rho_lung=0.25, rho_bone=1.85,
                   rmin=0.5, rmax=2.0):
    """Water cube [0, L]^3 with random lung, then bone spheres from ``default_rng(seed)``
    (centres uniform in the inner 80 %, radii U(rmin, rmax) cm); indexed [k, i, j] = (z, x, y)."""
    rng = np.random.default_rng(seed)
    Z, X, Y = np.meshgrid(np.linspace(0.0, L, ncz), np.linspace(0.0, L, ncx), np.linspace(0.0, L, ncy),
                          indexing="ij")
    rho = np.full((ncz, ncx, ncy), rho_water)
    for val in [rho_lung] * n_lung + [rho_bone] * n_bone:
        c = rng.uniform(0.1 * L, 0.9 * L, 3)
        rad = rng.uniform(rmin, rmax)
        rho[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= rad * rad] = val
    return rho


def _ghost_axis(a, b, ncells):
    """Cell centres spanning [a, b] with the reference's ghost shift (settings.jl:315-325)."""
    x = np.linspace(a, b, ncells)
    dx = x[1] - x[0]
    x = np.concatenate([[x[0] - dx], x]) + dx / 2
    return x, x[:-1] + 0.5 * dx, dx


class Settings3D:
    """Settings of the 3D proton problem ``"csdProton3D"`` (no counterpart in
    the reference, which is 2D): a 96^3 grid at 1 mm ([0, 9.5]^3 cm with the
    ghost-cell grid), seeded water / lung / bone spheres, a pencil beam along +x
    entering at x = 0 centred at (y0, z0) = (4.75, 4.75) cm (spatial sigma
    0.3 cm, angular sigma 0.01 rad about +x), protons 90 -> 1 MeV with
    S(E) = (250 / E) ln(1 + 0.07 E) MeV cm^2/g (the Bethe-like (a/E) ln(b E)
    is negative below 1/b = 14.3 MeV), Henyey-Greenstein sigma_l =
    100 * 0.95^l cm^-1, P_13 (196 moments), rank cap 40. The energy step is
    the stability bound dtau = tau_cfl min(dx, dy, dz) min(rho) with
    tau_cfl = 1/3 (1336 steps)."""

    def __init__(self, Nx: int = 97, Ny: int = 97, Nz: int = 97, r: int = 40, problem: str = "csdProton3D",
                 nPN: int = 13, seed: int = 20240605, nEnergies: int = 0, tau_cfl: float = 1.0 / 3.0,
                 L: float = 9.5):
        if problem != "csdProton3D":
            raise ValueError(f"3D problem {problem!r} not available; choose 'csdProton3D'")
        self.problem, self.particle = problem, "Protons"
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.NCellsX, self.NCellsY, self.NCellsZ = Nx - 1, Ny - 1, Nz - 1
        self.x, self.xMid, self.dx = _ghost_axis(0.0, L, self.NCellsX)
        self.y, self.yMid, self.dy = _ghost_axis(0.0, L, self.NCellsY)
        self.z, self.zMid, self.dz = _ghost_axis(0.0, L, self.NCellsZ)
        self.eRest = 938.26
        self.eMax, self.eMin = 90.0, 1.0
        self.stopping = "proton_log1p"
        self.hg_g, self.sigmaT_hg = 0.95, 100.0
        self.x0, self.y0, self.z0 = 0.0, 0.5 * L, 0.5 * L
        self.Omega1, self.Omega2, self.Omega3 = 1.0, 0.0, 0.0
        self.densityMin = 1.0
        self.sigmaXInv = self.sigmaYInv = self.sigmaZInv = 1.0 / (2 * 0.3**2)
        self.sigmaO1Inv = self.sigmaO2Inv = self.sigmaO3Inv = 1.0 / (2 * 0.01**2)
        self.sigmaEInv = 1.0
        self.psi_scale = 1e5
        self.beam_peak_normalized = True
        self.seed = seed
        self.density = seeded_spheres(self.NCellsX, self.NCellsY, self.NCellsZ, L, seed)
        self.r = r
        self.theta, self.thetaIndex, self.c_eta = 1e-2, 1.0, 5.0
        self.nPN = nPN
        self.nEnergies = nEnergies
        self.tau_cfl = tau_cfl
        self.cfl = tau_cfl
        self.dE = tau_cfl * min(self.dx, self.dy, self.dz) * self.density.min()
