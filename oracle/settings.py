"""``mutable struct Settings`` (oracle restatement of ``code/settings.jl:5-338``).

Only problems whose physics does not come from the reference's material tables
or image phantoms are restated. The reference problems kept are the
analytic-source ones; the benchmark problems are new names that plug analytic
S(E), Henyey-Greenstein sigma_l and seeded phantoms into the same struct.
"""
from __future__ import annotations

import math

import numpy as np


def seeded_phantom(ncx: int, ncy: int, a: float, b: float, c: float, d: float, seed: int,
                   n_lung: int = 3, n_bone: int = 1, rho_water: float = 1.0,
                   rho_lung: float = 0.25, rho_bone: float = 1.85,
                   rmin: float = 0.05, rmax: float = 0.2) -> np.ndarray:
    """Water background with random ellipses (lung, then bone) from ``default_rng(seed)``.

    Ellipse centres are uniform in the inner 80 % of the domain, semi-axes are
    U(rmin, rmax) cm, orientation U(0, pi). Density is indexed [i, j] = (x, y).
    """
    rng = np.random.default_rng(seed)
    xs = np.linspace(a, b, ncx)
    ys = np.linspace(c, d, ncy)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    rho = np.full((ncx, ncy), rho_water)
    kinds = [rho_lung] * n_lung + [rho_bone] * n_bone
    for val in kinds:
        cx = rng.uniform(a + 0.1 * (b - a), b - 0.1 * (b - a))
        cy = rng.uniform(c + 0.1 * (d - c), d - 0.1 * (d - c))
        ra = rng.uniform(rmin, rmax)
        rb = rng.uniform(rmin, rmax)
        th = rng.uniform(0.0, math.pi)
        dxx = X - cx
        dyy = Y - cy
        u = dxx * math.cos(th) + dyy * math.sin(th)
        v = -dxx * math.sin(th) + dyy * math.cos(th)
        rho[(u / ra) ** 2 + (v / rb) ** 2 <= 1.0] = val
    return rho


class Settings:
    """Settings(Nx, Ny, r, problem, particle) -- ``settings.jl:67``.

    Fields keep the reference names. Added fields (defaults keep the reference
    behaviour): ``stopping`` (analytic S(E) model), ``eMin``, ``hg_g``,
    ``sigmaT_hg`` (HG sigma_l = sigmaT_hg g^l), ``nEnergies`` (0 = reference
    rule ceil(eMax/dE)), the PsiBeam widths ``sigmaO1Inv .. sigmaEInv``,
    ``psi_scale`` (the 10^5 prefactor) and ``seed``.
    """

    def __init__(self, Nx: int = 102, Ny: int = 102, r: int = 15, problem: str = "LineSource",
                 particle: str = "Electrons", nPN: int | None = None, nEnergies: int = 0,
                 seed: int = 20240601, cfl: float | None = None,
                 tau_cfl: float | None = None):
        # settings.jl:69-73
        eRest = 938.26 if particle == "Protons" else 0.5
        NCellsX = Nx - 1
        NCellsY = Ny - 1
        a, b, c, d = 0.0, 14.5, 0.0, 14.5
        density = np.ones((NCellsX, NCellsY))
        sigmaS = 0.0
        sigmaA = 0.0
        eMax = 1.0
        x0 = 0.5 * b
        y0 = 1.0 * d
        Omega1 = -1.0
        Omega3 = -1.0
        densityMin = 0.2
        thetaIndex = 1.0
        theta = 1e-2
        cfl_ = 1.5
        # analytic-physics extensions
        self.stopping = "electron_log"
        self.eMin = 0.001
        self.hg_g = 0.9
        self.sigmaT_hg = 100.0
        self.sigmaO1Inv = 0.0
        self.sigmaO3Inv = 75.0
        self.sigmaXInv = 20.0
        self.sigmaYInv = 20.0
        self.sigmaEInv = 100.0
        self.psi_scale = 1e5
        self.beam_peak_normalized = problem in ("csdWaterBeam", "csdPhantom")
        self.seed = seed
        if problem == "csdWaterBeam":
            # Benchmark problem 1: 100x100 cells on [0,1]^2, water, beam along +x
            # entering at x = 0, y0 = 0.5, sigma_x = 0.05 cm, sigma_Omega = 0.01 rad.
            a, b, c, d = 0.0, 1.0, 0.0, 1.0
            eMax = 5.0
            x0, y0 = 0.0, 0.5
            Omega1, Omega3 = 1.0, 0.0
            densityMin = 1.0
            self.sigmaXInv = self.sigmaYInv = 1.0 / (2 * 0.05**2)
            self.sigmaO1Inv = self.sigmaO3Inv = 1.0 / (2 * 0.01**2)
            self.sigmaEInv = 100.0
            cfl_ = 0.5
        elif problem == "csdPhantom":
            # Benchmark problem 2: seeded water/lung/bone phantom on [0,1]^2.
            a, b, c, d = 0.0, 1.0, 0.0, 1.0
            eMax = 5.0
            x0, y0 = 0.0, 0.5
            Omega1, Omega3 = 1.0, 0.0
            densityMin = 1.0
            self.sigmaXInv = self.sigmaYInv = 1.0 / (2 * 0.05**2)
            self.sigmaO1Inv = self.sigmaO3Inv = 1.0 / (2 * 0.01**2)
            self.sigmaEInv = 100.0
            density = seeded_phantom(NCellsX, NCellsY, a, b, c, d, seed)
            cfl_ = 0.5
        else:
            raise ValueError(f"problem {problem!r} is not restated in the oracle")
        if cfl is not None:
            cfl_ = cfl
        sigmaT = sigmaA + sigmaS

        # settings.jl:315-325 (grid with ghost shift; xMid spans [a, b])
        x = np.linspace(a, b, NCellsX)
        dx = x[1] - x[0]
        x = np.concatenate([[x[0] - dx], x]) + dx / 2
        xMid = x[:-1] + 0.5 * dx
        y = np.linspace(c, d, NCellsY)
        dy = y[1] - y[0]
        y = np.concatenate([[y[0] - dy], y]) + dy / 2
        yMid = y[:-1] + 0.5 * dy
        # settings.jl:329
        dE = cfl_ * min(dx, dy) * density.min()

        self.Nx, self.Ny = Nx, Ny
        self.NCellsX, self.NCellsY = NCellsX, NCellsY
        self.a, self.b, self.c, self.d = a, b, c, d
        self.dx, self.dy = dx, dy
        self.eMax, self.eRest, self.dE, self.cfl = eMax, eRest, dE, cfl_
        self.nPN = 21 if nPN is None else nPN  # settings.jl:332
        self.x, self.xMid, self.y, self.yMid = x, xMid, y, yMid
        self.problem, self.particle = problem, particle
        self.x0, self.y0, self.Omega1, self.Omega3 = x0, y0, Omega1, Omega3
        self.densityMin = densityMin
        self.sigmaT, self.sigmaS = sigmaT, sigmaS
        self.density = density
        self.r = r
        self.theta = theta  # reference field name: ϑ
        self.thetaIndex = thetaIndex  # ϑIndex
        self.c_eta = 5.0  # cη, settings.jl:334
        self.nEnergies = nEnergies
        self.tau_cfl = tau_cfl if tau_cfl is not None else (0.5 if problem in ("csdWaterBeam", "csdPhantom") else 0.0)
