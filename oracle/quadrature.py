"""Tensorised Gauss-Legendre x equispaced-phi quadrature and SH transforms (oracle).

Follows ``code/quadratures/standardQuadrature.jl:7-37`` (points and weights),
``code/quadratures/Quadrature.jl:173-208`` (``ComputeTrafoMatrices``) and
``code/utils.jl:1-41`` (``sph_cc`` / ``real_sph``).
"""
from __future__ import annotations

import math

import numpy as np

from .pn import n_moments


def gauss_legendre(n: int):
    """FastGaussQuadrature.jl ``gausslegendre(n)``: ascending nodes and weights."""
    mu, w = np.polynomial.legendre.leggauss(n)
    return mu, w


def standard_points(q: int):
    """``computeXYZandWeights(q)`` (``standardQuadrature.jl:7-37``).

    Returns (pointsxyz (2q^2, 3), weights (2q^2,)). Point ``(j-1)*q + k`` (1-based)
    holds mu_k and phi_j = (j - 1/2) pi / q (column-major flattening of the q x 2q
    grids).
    """
    mu, gw = gauss_legendre(q)
    phi = np.array([(k + 0.5) * math.pi / q for k in range(2 * q)])
    x = np.sqrt(1.0 - mu**2)[:, None] * np.cos(phi)[None, :]
    y = np.sqrt(1.0 - mu**2)[:, None] * np.sin(phi)[None, :]
    z = mu[:, None] * np.ones(phi.size)[None, :]
    w = 2.0 * math.pi / q * np.repeat(gw[:, None], 2 * q, axis=1)
    pts = np.stack([x.ravel(order="F"), y.ravel(order="F"), z.ravel(order="F")], axis=1)
    return pts, w.ravel(order="F") * 0.5


def plm_unnormalized(x: float, lmax: int) -> np.ndarray:
    """SphericalHarmonics.jl ``computePlmx(x, lmax, norm=Unnormalized())``.

    Associated Legendre functions P_l^m(x), 0 <= m <= l <= lmax, WITHOUT the
    Condon-Shortley phase, stored at 0-based index l(l+1)/2 + m. Computed by the
    standard three-term recurrence in l (published algorithm):
    P_m^m = (2m-1)!! (1-x^2)^{m/2}, P_{m+1}^m = x (2m+1) P_m^m,
    (l-m) P_l^m = x (2l-1) P_{l-1}^m - (l+m-1) P_{l-2}^m.
    """
    out = np.zeros((lmax + 1) * (lmax + 2) // 2)
    s = math.sqrt(max(0.0, 1.0 - x * x))
    pmm = 1.0
    for m in range(0, lmax + 1):
        if m > 0:
            pmm = pmm * (2 * m - 1) * s
        out[m * (m + 1) // 2 + m] = pmm
        if m + 1 <= lmax:
            p1 = x * (2 * m + 1) * pmm
            out[(m + 1) * (m + 2) // 2 + m] = p1
            p0 = pmm
            for l in range(m + 2, lmax + 1):
                p2 = (x * (2 * l - 1) * p1 - (l + m - 1) * p0) / (l - m)
                out[l * (l + 1) // 2 + m] = p2
                p0, p1 = p1, p2
    return out


def _norm_lm(l: int, m: int) -> float:
    # sqrt((2l+1)/(4pi) (l-|m|)!/(l+|m|)!) evaluated in exact integer arithmetic,
    # as utils.jl:18 does with factorial(big(...)).
    ma = abs(m)
    num = math.factorial(l - ma)
    den = math.factorial(l + ma)
    return math.sqrt((2 * l + 1) / (4 * math.pi) * (num / den))


def real_sph(phi: float, l: int, k: int, z: np.ndarray) -> float:
    """Real spherical harmonic ``real_sph(mu, phi, l, k, z)`` (``utils.jl:32-41``).

    Expanding ``sph_cc`` (``utils.jl:14-20``) gives
    k > 0: sqrt2 N P_l^k cos(k phi); k < 0: sqrt2 N P_l^|k| sin(|k| phi); k = 0: N P_l^0.
    """
    ma = abs(k)
    p = z[l * (l + 1) // 2 + ma]
    nrm = _norm_lm(l, k)
    if k > 0:
        return math.sqrt(2.0) * nrm * p * math.cos(k * phi)
    if k < 0:
        return math.sqrt(2.0) * nrm * p * math.sin(ma * phi)
    return nrm * p


def compute_trafo_matrices(q: int, npn: int):
    """``ComputeTrafoMatrices(Q, Norder, nPN)`` (``Quadrature.jl:173-208``).

    O (nq x N): real SH at the quadrature points; M = O^T diag(w) (N x nq).
    """
    nt = n_moments(npn)
    mu, gw = gauss_legendre(q)
    phi = np.array([(k + 0.5) * math.pi / q for k in range(2 * q)])
    w = (2.0 * math.pi / q * np.repeat(gw[:, None], 2 * q, axis=1)).ravel(order="F") * 0.5
    nq = 2 * q * q
    O = np.zeros((nq, nt))
    for k in range(q):
        z = plm_unnormalized(mu[k], npn)
        for j in range(2 * q):
            row = j * q + k
            c = 0
            for l in range(npn + 1):
                for m in range(-l, l + 1):
                    O[row, c] = real_sph(phi[j], l, m, z)
                    c += 1
    M = (O * w[:, None]).T.copy()
    return O, M
