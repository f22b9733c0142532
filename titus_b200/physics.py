"""Host-side setup of the CSD energy step (the work of ``SolverCSD(settings)``).

Builds the arrays the device energy loop reads, following the reference's
constructor (``code/SolverCSD.jl:63-146``) and the files it uses:
P_N flux matrices (``code/PNSystem.jl:196-250``), Roe matrices |A|
(``SolverCSD.jl:83-97``), the tensorised quadrature and SH transforms
(``code/quadratures/Quadrature.jl:173-208``, ``code/utils.jl:1-41``), the CSD
transformed-energy grid (``code/CSD.jl:27-95``) and the separable boundary
source ``PsiBeam`` (``SolverCSD.jl:240-276``). Vectorised numpy; runs once per
solver, not per energy step.
"""
from __future__ import annotations

import math

import numpy as np


# ----------------------------------------------------------------- P_N ------
def moment_index(l, k):
    return l * l + k + l


def flux_matrices(npn: int):
    """Dense Ax, Az of the real-SH P_N system (``PNSystem.jl:142-194``)."""
    N = (npn + 1) ** 2
    Ax = np.zeros((N, N))
    Az = np.zeros((N, N))

    def A_(l, k):
        return math.sqrt(((l - k + 1) * (l + k + 1)) / ((2 * l + 3) * (2 * l + 1)))

    def B_(l, k):
        return math.sqrt(((l - k) * (l + k)) / ((2 * l + 1) * (2 * l - 1)))

    def C_(l, k):
        return math.sqrt(((l + k + 1) * (l + k + 2)) / ((2 * l + 3) * (2 * l + 1)))

    def D_(l, k):
        return math.sqrt(((l - k) * (l - k - 1)) / ((2 * l + 1) * (2 * l - 1)))

    def E_(l, k):
        return math.sqrt(((l - k + 1) * (l - k + 2)) / ((2 * l + 3) * (2 * l + 1)))

    def F_(l, k):
        return math.sqrt(((l + k) * (l + k - 1)) / ((2 * l + 1) * (2 * l - 1)))

    r2 = math.sqrt(2.0)

    def Ct(l, k):
        return 0.0 if k < 0 else (r2 * C_(l, k) if k == 0 else C_(l, k))

    def Dt(l, k):
        return 0.0 if k < 0 else (r2 * D_(l, k) if k == 0 else D_(l, k))

    def Et(l, k):
        return r2 * E_(l, k) if k == 1 else E_(l, k)

    def Ft(l, k):
        return r2 * F_(l, k) if k == 1 else F_(l, k)

    sgn = lambda k: 1 if k >= 0 else -1  # noqa: E731
    for l in range(npn + 1):
        for k in range(-l, l + 1):
            i = moment_index(l, k)
            kp, km = k + sgn(k), k - sgn(k)
            # same visiting order as the reference, so later writes win identically
            ent = []
            if k != -1:
                ent.append((moment_index(l - 1, km), 0.5 * Ct(l - 1, abs(k) - 1)))
                ent.append((moment_index(l + 1, km), -0.5 * Dt(l + 1, abs(k) - 1)))
            ent.append((moment_index(l - 1, kp), -0.5 * Et(l - 1, abs(k) + 1)))
            ent.append((moment_index(l + 1, kp), 0.5 * Ft(l + 1, abs(k) + 1)))
            for j, v in ent:
                if 0 <= j < N:
                    Ax[i, j] = v
            j = moment_index(l - 1, k)
            if 0 <= j < N:
                Az[i, j] = A_(l - 1, k)
            j = moment_index(l + 1, k)
            if 0 <= j < N:
                Az[i, j] = B_(l + 1, k)
    return Ax, Az


def flux_matrix_y(npn: int):
    """Dense Ay of the real-SH P_N system (``PNSystem.jl:142-194``; unused by
    the reference's 2D solvers, the z direction of the 3D problems). It is the
    moment matrix of Omega_y: M diag(Omega_y) O."""
    N = (npn + 1) ** 2
    Ay = np.zeros((N, N))
    r2 = math.sqrt(2.0)

    def frac(a, b):
        return math.sqrt(a / b)

    def C_(l, k):
        return frac((l + k + 1) * (l + k + 2), (2 * l + 3) * (2 * l + 1))

    def D_(l, k):
        return frac((l - k) * (l - k - 1), (2 * l + 1) * (2 * l - 1))

    def E_(l, k):
        return frac((l - k + 1) * (l - k + 2), (2 * l + 3) * (2 * l + 1))

    def F_(l, k):
        return frac((l + k) * (l + k - 1), (2 * l + 1) * (2 * l - 1))

    def Ct(l, k):
        return 0.0 if k < 0 else (r2 * C_(l, k) if k == 0 else C_(l, k))

    def Dt(l, k):
        return 0.0 if k < 0 else (r2 * D_(l, k) if k == 0 else D_(l, k))

    def Et(l, k):
        return r2 * E_(l, k) if k == 1 else E_(l, k)

    def Ft(l, k):
        return r2 * F_(l, k) if k == 1 else F_(l, k)

    sgn = lambda k: 1 if k >= 0 else -1  # noqa: E731
    for l in range(npn + 1):
        for k in range(-l, l + 1):
            i = moment_index(l, k)
            kp, km, s = k + sgn(k), k - sgn(k), sgn(k)
            ent = []
            if k != 1:
                ent.append((moment_index(l - 1, -km), -0.5 * s * Ct(l - 1, abs(k) - 1)))
                ent.append((moment_index(l + 1, -km), 0.5 * s * Dt(l + 1, abs(k) - 1)))
            ent.append((moment_index(l - 1, -kp), -0.5 * s * Et(l - 1, abs(k) + 1)))
            ent.append((moment_index(l + 1, -kp), 0.5 * s * Ft(l + 1, abs(k) + 1)))
            for j, v in ent:
                if 0 <= j < N:
                    Ay[i, j] = v
    return Ay


def roe(A: np.ndarray, drop: float = 1e-10) -> np.ndarray:
    """|A| = V |Lambda| V^-1 with |entries| <= drop removed (``SolverCSD.jl:83-97``)."""
    lam, V = np.linalg.eigh(0.5 * (A + A.T))
    R = (V * np.abs(lam)) @ V.T
    R[np.abs(R) <= drop] = 0.0
    return R


def to_csr(A: np.ndarray):
    rows, cols = np.nonzero(A)
    order = np.lexsort((cols, rows))
    rows, cols = rows[order], cols[order]
    rowptr = np.zeros(A.shape[0] + 1, dtype=np.int32)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr).astype(np.int32)
    return rowptr, cols.astype(np.int32), np.ascontiguousarray(A[rows, cols], dtype=np.float64)


# ---------------------------------------------------------- quadrature -----
def assoc_legendre_table(x: np.ndarray, lmax: int) -> np.ndarray:
    """P_l^m(x) without Condon-Shortley phase, shape (len(x), lmax+1, lmax+1) [.., l, m]."""
    x = np.asarray(x, dtype=np.float64)
    P = np.zeros((x.size, lmax + 1, lmax + 1))
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    pmm = np.ones_like(x)
    for m in range(lmax + 1):
        if m > 0:
            pmm = pmm * (2 * m - 1) * s
        P[:, m, m] = pmm
        if m + 1 <= lmax:
            P[:, m + 1, m] = x * (2 * m + 1) * pmm
        for l in range(m + 2, lmax + 1):
            P[:, l, m] = (x * (2 * l - 1) * P[:, l - 1, m] - (l + m - 1) * P[:, l - 2, m]) / (l - m)
    return P


def quadrature(q: int, npn: int):
    """Points (2q^2 x 3), weights, O (2q^2 x N), M (N x 2q^2); point (j, k) at row j*q + k."""
    mu, gw = np.polynomial.legendre.leggauss(q)
    phi = (np.arange(2 * q) + 0.5) * math.pi / q
    MU = np.tile(mu, 2 * q)                 # row j*q + k -> mu_k
    PHI = np.repeat(phi, q)                 # -> phi_j
    st = np.sqrt(1.0 - MU * MU)
    pts = np.stack([st * np.cos(PHI), st * np.sin(PHI), MU], axis=1)
    w = 2.0 * math.pi / q * np.tile(gw, 2 * q) * 0.5
    Pl = assoc_legendre_table(mu, npn)      # (q, l, m)
    N = (npn + 1) ** 2
    O = np.zeros((2 * q * q, N))
    kidx = np.tile(np.arange(q), 2 * q)
    for l in range(npn + 1):
        for m in range(-l, l + 1):
            ma = abs(m)
            nrm = math.sqrt((2 * l + 1) / (4 * math.pi) * (math.factorial(l - ma) / math.factorial(l + ma)))
            p = Pl[kidx, l, ma]
            if m > 0:
                col = math.sqrt(2.0) * nrm * p * np.cos(m * PHI)
            elif m < 0:
                col = math.sqrt(2.0) * nrm * p * np.sin(ma * PHI)
            else:
                col = nrm * p
            O[:, moment_index(l, m)] = col
    M = (O * w[:, None]).T.copy()
    return pts, w, O, M


# ----------------------------------------------------------------- CSD ------
def stopping_power(kind: str, E):
    E = np.asarray(E, dtype=np.float64)
    if kind == "electron_log":
        return 0.2 / E * np.log1p(10.0 * E)
    if kind == "proton_bethe":
        return 250.0 / E * np.log(0.07 * E)
    if kind == "proton_log1p":
        # (a / E) ln(1 + b E), a = 250 MeV^2 cm^2/g, b = 0.07 / MeV: the Bethe-like
        # form (a / E) ln(b E) is negative below 1/b = 14.3 MeV
        return 250.0 / E * np.log1p(0.07 * E)
    raise ValueError(f"unknown stopping power {kind!r}")


def _interp(xt, yt, x):
    x = np.asarray(x, dtype=np.float64)
    if np.any(x < xt[0]) or np.any(x > xt[-1]):
        raise ValueError("energy outside the stopping-power table")
    i = np.clip(np.searchsorted(xt, x, side="right") - 1, 0, xt.size - 2)
    t = (x - xt[i]) / (xt[i + 1] - xt[i])
    return yt[i] * (1.0 - t) + yt[i + 1] * t


def energy_grid(settings, with_mid: bool = False):
    """(eGrid, eTrafo, S) of ``CSD(settings)`` (``CSD.jl:47-89``) for analytic S(E);
    with ``with_mid`` also SMid, the stopping power at the midpoints of the
    transformed-energy steps (``CSD.jl:82-89``)."""
    s = settings
    E_tab = np.geomspace(0.5 * s.eMin, 2.0 * s.eMax, 4001)
    S_tab = stopping_power(s.stopping, E_tab)
    inc = np.diff(E_tab) / 2 * (1.0 / S_tab[1:] + 1.0 / S_tab[:-1])
    E_tr = np.concatenate([[0.0], np.cumsum(inc)])
    # sequential accumulation like the reference's loop (bitwise identical sums)
    acc = 0.0
    for i in range(1, E_tab.size):
        acc = acc + inc[i - 1]
        E_tr[i] = acc
    eMaxT = float(_interp(E_tab, E_tr, s.eMax))
    eMinT = float(_interp(E_tab, E_tr, s.eMin))
    if s.nEnergies > 0:
        nE = s.nEnergies
    elif s.tau_cfl > 0:
        dtau = s.tau_cfl * min(s.dx, s.dy) * float(np.min(s.density))
        nE = int(math.ceil((eMaxT - eMinT) / dtau)) + 1
    else:
        nE = int(math.ceil(s.eMax / s.dE))
    eTrafo = np.linspace(0.0, eMaxT - eMinT, nE)
    eGrid = _interp(E_tr, E_tab, eMaxT - eTrafo)
    S = _interp(E_tab, S_tab, eGrid)
    if not with_mid:
        return eGrid, eTrafo, S
    dE = eTrafo[1:] - eTrafo[:-1]
    SMid = _interp(E_tab, S_tab, _interp(E_tr, E_tab, eMaxT - (eTrafo[:-1] + 0.5 * dE)))
    return eGrid, eTrafo, S, SMid
