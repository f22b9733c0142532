"""P_N flux matrices and their Roe absolute values (oracle restatement).

Follows ``code/PNSystem.jl`` (recursion coefficients ``:58-132``, dense assembly
``SetupSystemMatrices`` ``:142-194``, sparse assembly ``:196-250``) and the Roe
matrix construction in ``code/SolverCSD.jl:83-97``.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp


def global_index(l: int, k: int) -> int:
    """0-based moment index of (l, k): ``PNSystem.jl:124-128``."""
    return l * l + k + l


def n_moments(npn: int) -> int:
    """``GlobalIndex(N, N) + 1`` (``PNSystem.jl:28``)."""
    return global_index(npn, npn) + 1


# Recursion coefficients, PNSystem.jl:58-80. Integer arithmetic inside the
# square root exactly as the Julia code (Int products, then float division).
def _A(l, k):
    return math.sqrt(((l - k + 1) * (l + k + 1)) / ((2 * l + 3) * (2 * l + 1)))


def _B(l, k):
    return math.sqrt(((l - k) * (l + k)) / ((2 * l + 1) * (2 * l - 1)))


def _C(l, k):
    return math.sqrt(((l + k + 1) * (l + k + 2)) / ((2 * l + 3) * (2 * l + 1)))


def _D(l, k):
    return math.sqrt(((l - k) * (l - k - 1)) / ((2 * l + 1) * (2 * l - 1)))


def _E(l, k):
    return math.sqrt(((l - k + 1) * (l - k + 2)) / ((2 * l + 3) * (2 * l + 1)))


def _F(l, k):
    return math.sqrt(((l + k) * (l + k - 1)) / ((2 * l + 1) * (2 * l - 1)))


def _Ct(l, k):  # PNSystem.jl:82-89
    if k < 0:
        return 0.0
    return math.sqrt(2) * _C(l, k) if k == 0 else _C(l, k)


def _Dt(l, k):  # PNSystem.jl:91-98
    if k < 0:
        return 0.0
    return math.sqrt(2) * _D(l, k) if k == 0 else _D(l, k)


def _Et(l, k):  # PNSystem.jl:100-106
    return math.sqrt(2) * _E(l, k) if k == 1 else _E(l, k)


def _Ft(l, k):  # PNSystem.jl:108-114
    return math.sqrt(2) * _F(l, k) if k == 1 else _F(l, k)


def _sgn(k):  # PNSystem.jl:116-122
    return 1 if k >= 0 else -1


def _kplus(k):
    return k + _sgn(k)


def _kminus(k):
    return k - _sgn(k)


def setup_system_matrices(npn: int):
    """Dense Ax, Ay, Az: ``PNSystem.jl:142-194``.

    Assignment order is kept (a later write to the same entry wins), which
    matters nowhere in practice but keeps the restatement literal.
    """
    nt = n_moments(npn)
    Ax = np.zeros((nt, nt))
    Ay = np.zeros((nt, nt))
    Az = np.zeros((nt, nt))

    def ok(j):
        return 0 <= j < nt

    for l in range(0, npn + 1):
        for k in range(-l, l + 1):
            i = global_index(l, k)
            if k != -1:
                j = global_index(l - 1, _kminus(k))
                if ok(j):
                    Ax[i, j] = 0.5 * _Ct(l - 1, abs(k) - 1)
                j = global_index(l + 1, _kminus(k))
                if ok(j):
                    Ax[i, j] = -0.5 * _Dt(l + 1, abs(k) - 1)
            j = global_index(l - 1, _kplus(k))
            if ok(j):
                Ax[i, j] = -0.5 * _Et(l - 1, abs(k) + 1)
            j = global_index(l + 1, _kplus(k))
            if ok(j):
                Ax[i, j] = 0.5 * _Ft(l + 1, abs(k) + 1)

            if k != 1:
                j = global_index(l - 1, -_kminus(k))
                if ok(j):
                    Ay[i, j] = -0.5 * _sgn(k) * _Ct(l - 1, abs(k) - 1)
                j = global_index(l + 1, -_kminus(k))
                if ok(j):
                    Ay[i, j] = 0.5 * _sgn(k) * _Dt(l + 1, abs(k) - 1)
            j = global_index(l - 1, -_kplus(k))
            if ok(j):
                Ay[i, j] = -0.5 * _sgn(k) * _Et(l - 1, abs(k) + 1)
            j = global_index(l + 1, -_kplus(k))
            if ok(j):
                Ay[i, j] = 0.5 * _sgn(k) * _Ft(l + 1, abs(k) + 1)

            j = global_index(l - 1, k)
            if ok(j):
                Az[i, j] = _A(l - 1, k)
            j = global_index(l + 1, k)
            if ok(j):
                Az[i, j] = _B(l + 1, k)
    return Ax, Ay, Az


def setup_system_matrices_sparse(npn: int):
    """Sparse CSC Ax, Ay, Az: ``PNSystem.jl:196-250``.

    The sparse assembly visits the same (i, j) pairs with the same values as the
    dense one. Julia's ``sparse(I, J, V)`` sums duplicates; no pair repeats within
    one matrix, so this equals the dense matrices (checked in the tests).
    """
    Ax, Ay, Az = setup_system_matrices(npn)
    return sp.csc_matrix(Ax), sp.csc_matrix(Ay), sp.csc_matrix(Az)


def roe_abs(A: np.ndarray, drop: float = 1e-10) -> sp.csc_matrix:
    """Roe matrix ``V |Lambda| V^-1`` with entries of abs value <= ``drop`` removed.

    ``SolverCSD.jl:83-97``. ``A`` is symmetric up to rounding, so the matrix
    function |A| is evaluated from a symmetric eigendecomposition of the
    symmetrised matrix; |A| does not depend on the eigenvector gauge.
    """
    As = 0.5 * (A + A.T)
    lam, V = np.linalg.eigh(As)
    absA = (V * np.abs(lam)) @ V.T
    absA[np.abs(absA) <= drop] = 0.0
    return sp.csc_matrix(absA)
