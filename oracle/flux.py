"""FP64 restatement of ``solveFlux!`` (``code/SolverCSD.jl:295-386``), the
second-order limited upwind flux of the uncollided ordinates, with its
limiter helpers ``minmod`` (:288) and ``slopefit`` (:290-293).

TEST INFRASTRUCTURE ONLY (see the package docstring): the checker for the CUDA
operator ``titus_limited_flux``.

Arrays are (nx, ny, q) with i along x (the reference's first index), j along y
and the ordinate last. Every arithmetic step is a single IEEE double operation
in the reference's evaluation order, so a GPU kernel that uses the same order
without FMA contraction matches bit for bit.
"""
from __future__ import annotations

import numpy as np


def _clamp(v, lo, hi):
    """Julia ``Base.clamp``: ``v > hi ? hi : (v < lo ? lo : v)``."""
    return np.where(v > hi, hi, np.where(v < lo, lo, v))


def minmod(x, y):
    """``minmod(x, y) = ifelse(x < 0, clamp(y, x, 0.0), clamp(y, 0.0, x))`` (:288)."""
    return np.where(x < 0, _clamp(y, x, 0.0), _clamp(y, 0.0, x))


def slopefit(left, center, right):
    """``slopefit`` (:290-293): minmod(2 (r - c), minmod((r - l)/2, 2 (c - l)))."""
    tmp = minmod(0.5 * (right - left), 2.0 * (center - left))
    return minmod(2.0 * (right - center), tmp)


def _axis_diff(m2, m1, c, p1, p2, positive):
    """(face after the centre) - (face before it) along one axis: the
    reference's ``eastflux - westflux`` / ``northflux - southflux``. Positive
    component: s1..s4 = offsets -2..+1 and ``s + slopefit/2``; negative:
    offsets -1..+2 and ``s - slopefit/2`` (:309-385)."""
    after_p = c + 0.5 * slopefit(m1, c, p1)
    before_p = m1 + 0.5 * slopefit(m2, m1, c)
    after_n = p1 - 0.5 * slopefit(c, p1, p2)
    before_n = c - 0.5 * slopefit(m1, c, p1)
    return np.where(positive, after_p - before_p, after_n - before_n)


def limited_flux(phi, omega_x, omega_z, dx, dy, flux=None):
    """``solveFlux!(obj, phi, flux)`` with ``obj.qReduced[:,1] = omega_x``,
    ``obj.qReduced[:,3] = omega_z``. Returns a copy of ``flux`` (zeros if None)
    with the interior cells 2 <= i < nx-2, 2 <= j < ny-2 (1-based ``3:N-2``,
    :306-307) overwritten; the other cells keep their values. The four
    quadrant loops of the reference are the sign choices ``omega >= 0``."""
    phi = np.asarray(phi, dtype=np.float64)
    nx, ny, q = phi.shape
    out = np.zeros_like(phi) if flux is None else np.array(flux, dtype=np.float64, copy=True)
    if nx < 5 or ny < 5:
        return out
    ox = np.asarray(omega_x, dtype=np.float64)
    oz = np.asarray(omega_z, dtype=np.float64)
    I = slice(2, nx - 2)
    J = slice(2, ny - 2)

    def sx(d):
        return phi[2 + d:nx - 2 + d, J, :]

    def sy(d):
        return phi[I, 2 + d:ny - 2 + d, :]

    ew = _axis_diff(sx(-2), sx(-1), sx(0), sx(1), sx(2), ox >= 0.0)
    ns = _axis_diff(sy(-2), sy(-1), sy(0), sy(1), sy(2), oz >= 0.0)
    out[I, J, :] = (ox / dx) * ew + (oz / dy) * ns
    return out


def limited_flux_loops(phi, omega_x, omega_z, dx, dy, flux=None):
    """Literal transcription of the four quadrant loops (:309-385), one
    element at a time. Slow: for small cases that pin ``limited_flux``."""
    phi = np.asarray(phi, dtype=np.float64)
    nx, ny, q = phi.shape
    out = np.zeros_like(phi) if flux is None else np.array(flux, dtype=np.float64, copy=True)

    def mm(x, y):
        lo, hi = (x, 0.0) if x < 0 else (0.0, x)
        return hi if y > hi else (lo if y < lo else y)

    def sf(l, c, r):
        return mm(2.0 * (r - c), mm(0.5 * (r - l), 2.0 * (c - l)))

    for j in range(2, ny - 2):
        for i in range(2, nx - 2):
            for k in range(q):
                if omega_z[k] >= 0.0:
                    s1, s2, s3, s4 = phi[i, j - 2, k], phi[i, j - 1, k], phi[i, j, k], phi[i, j + 1, k]
                    north = s3 + 0.5 * sf(s2, s3, s4)
                    south = s2 + 0.5 * sf(s1, s2, s3)
                else:
                    s1, s2, s3, s4 = phi[i, j - 1, k], phi[i, j, k], phi[i, j + 1, k], phi[i, j + 2, k]
                    north = s3 - 0.5 * sf(s2, s3, s4)
                    south = s2 - 0.5 * sf(s1, s2, s3)
                if omega_x[k] >= 0.0:
                    s1, s2, s3, s4 = phi[i - 2, j, k], phi[i - 1, j, k], phi[i, j, k], phi[i + 1, j, k]
                    east = s3 + 0.5 * sf(s2, s3, s4)
                    west = s2 + 0.5 * sf(s1, s2, s3)
                else:
                    s1, s2, s3, s4 = phi[i - 1, j, k], phi[i, j, k], phi[i + 1, j, k], phi[i + 2, j, k]
                    east = s3 - 0.5 * sf(s2, s3, s4)
                    west = s2 - 0.5 * sf(s1, s2, s3)
                out[i, j, k] = omega_x[k] / dx * (east - west) + omega_z[k] / dy * (north - south)
    return out
