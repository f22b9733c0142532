"""CSD energy grid and cross sections (oracle restatement of ``code/CSD.jl``).

The reference reads tabulated stopping powers and Legendre moments of the
elastic cross section (``MaterialParameters.jl``). The benchmark problems use
an analytic stopping power S(E) and Henyey-Greenstein moments instead; the
analytic S(E) is sampled on a fixed logarithmic table and then goes through
exactly the reference's transformed-energy construction (``CSD.jl:47-89``):
trapezoidal tau(E) = int dE/S, a uniform tau grid, and piecewise-linear
interpolation back to E.
"""
from __future__ import annotations

import math

import numpy as np


def linear_interp(xt: np.ndarray, yt: np.ndarray, x):
    """Interpolations.jl ``LinearInterpolation(xt, yt; extrapolation_bc=Throw())``.

    Piecewise linear on the (strictly monotone increasing) knots ``xt``; raises
    outside [xt[0], xt[-1]] like ``Throw()``. Interval search uses the left
    knot (``searchsorted`` semantics of Interpolations 0.14 gridded BSpline(Linear)).
    """
    x = np.asarray(x, dtype=np.float64)
    if np.any(x < xt[0]) or np.any(x > xt[-1]):
        raise ValueError("linear_interp: argument outside the table (Throw())")
    i = np.searchsorted(xt, x, side="right") - 1
    i = np.clip(i, 0, xt.size - 2)
    t = (x - xt[i]) / (xt[i + 1] - xt[i])
    return yt[i] * (1.0 - t) + yt[i + 1] * t


def analytic_stopping_power(kind: str, E):
    """Analytic stopping powers (MeV cm^2/g) of the benchmark problems."""
    E = np.asarray(E, dtype=np.float64)
    if kind == "electron_log":  # S(E) = 0.2/E ln(1 + 10 E)
        return 0.2 / E * np.log1p(10.0 * E)
    if kind == "proton_bethe":  # S(E) = (a/E) ln(b E), a = 250, b = 0.07
        return 250.0 / E * np.log(0.07 * E)
    if kind == "proton_log1p":  # S(E) = (a/E) ln(1 + b E): the form above kept positive below 1/b
        return 250.0 / E * np.log1p(0.07 * E)
    raise ValueError(f"unknown stopping power model {kind!r}")


def analytic_table(kind: str, e_min: float, e_max: float, n_tab: int = 4001):
    """Fixed log-spaced table [e_min/2, 2 e_max] of the analytic S(E)."""
    E = np.geomspace(0.5 * e_min, 2.0 * e_max, n_tab)
    return E, analytic_stopping_power(kind, E)


class CSD:
    """``struct CSD`` + constructor (``CSD.jl:6-95``) for analytic physics.

    Attributes follow the reference: ``eGrid``, ``eTrafo``, ``S``, ``SMid``;
    ``sigma_l`` holds the (energy independent) Legendre moments sigma_l,
    l = 0..nPN, used by ``SigmaAtEnergy``.
    """

    def __init__(self, settings):
        s = settings
        E_tab, S_tab = analytic_table(s.stopping, s.eMin, s.eMax)
        n_tab = E_tab.size
        # CSD.jl:47-51 trapezoid for tau(E)
        E_tr = np.zeros(n_tab)
        for i in range(1, n_tab):
            E_tr[i] = E_tr[i - 1] + (E_tab[i] - E_tab[i - 1]) / 2 * (1.0 / S_tab[i] + 1.0 / S_tab[i - 1])
        minE = s.eMin
        maxE = s.eMax
        eMaxTrafo = float(linear_interp(E_tab, E_tr, maxE))
        eMinTrafo = float(linear_interp(E_tab, E_tr, minE))
        # CSD.jl:68-70. New problems may pin the grid size through
        # settings.nEnergies; otherwise the reference rule ceil(maxE/dE).
        if s.nEnergies > 0:
            nE = s.nEnergies
        elif s.tau_cfl > 0:
            # benchmark problems: step count from the explicit scheme's
            # stability bound in transformed energy, dtau = cfl min(dx,dy) min(rho)
            dtau = s.tau_cfl * min(s.dx, s.dy) * float(s.density.min())
            nE = int(math.ceil((eMaxTrafo - eMinTrafo) / dtau)) + 1
        else:
            nE = int(math.ceil(maxE / s.dE))
        eTrafo = np.linspace(eMaxTrafo - eMaxTrafo, eMaxTrafo - eMinTrafo, nE)
        eGrid = linear_interp(E_tr, E_tab, eMaxTrafo - eTrafo)
        S = linear_interp(E_tab, S_tab, eGrid)
        dE = eTrafo[1:] - eTrafo[:-1]
        eGridMid = linear_interp(E_tr, E_tab, eMaxTrafo - (eTrafo[:-1] + 0.5 * dE))
        SMid = linear_interp(E_tab, S_tab, eGridMid)
        self.eGrid = eGrid
        self.eTrafo = eTrafo
        self.S = S
        self.SMid = SMid
        self.settings = s
        g = s.hg_g
        self.sigma_l = np.array([s.sigmaT_hg * g**l for l in range(s.nPN + 1)])

    def sigma_at_energy(self, energy: float) -> np.ndarray:
        """``SigmaAtEnergy`` (``CSD.jl:97-127``): per-Legendre-order sigma_l(E).

        Henyey-Greenstein moments sigma_l = sigma_t g^l do not depend on E.
        """
        return self.sigma_l.copy()
