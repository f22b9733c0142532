"""Oracle pins: P_N matrices, Roe |A| and the quadrature / SH transforms.

Golden vectors: the reference's ``validationData/{AxPlus,AxMinus,AyPlus,AyMinus}.csv``
(nPN = 7) hold A+- = (A +- |A|)/2; identities M O = I and M diag(Omega) O = A pin
the spherical-harmonic convention (no Condon-Shortley phase).
"""
import os

import numpy as np
import pytest

from oracle import pn, quadrature as qd

GOLD = os.path.join(os.path.dirname(__file__), "golden", "pn_golden.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_golden_ax_splitting(gold):
    Ax, Ay, Az = pn.setup_system_matrices(7)
    absAx = pn.roe_abs(Ax).toarray()
    # CSV precision is 6 significant digits
    assert np.abs(gold["AxPlus"] + gold["AxMinus"] - Ax).max() < 2e-6
    assert np.abs(gold["AxPlus"] - gold["AxMinus"] - absAx).max() < 2e-6


def test_golden_ay_splitting(gold):
    Ax, Ay, Az = pn.setup_system_matrices(7)
    absAy = pn.roe_abs(Ay).toarray()
    assert np.abs(gold["AyPlus"] + gold["AyMinus"] - Ay).max() < 2e-6
    assert np.abs(gold["AyPlus"] - gold["AyMinus"] - absAy).max() < 2e-6


@pytest.mark.parametrize("npn", [3, 7, 13])
def test_sparse_equals_dense(npn):
    A = pn.setup_system_matrices(npn)
    B = pn.setup_system_matrices_sparse(npn)
    for a, b in zip(A, B):
        assert np.array_equal(a, b.toarray())


@pytest.mark.parametrize("npn", [5, 7, 13])
def test_quadrature_identities(npn):
    q = npn + 1
    O, M = qd.compute_trafo_matrices(q, npn)
    pts, w = qd.standard_points(q)
    Ax, Ay, Az = pn.setup_system_matrices(npn)
    N = pn.n_moments(npn)
    assert O.shape == (2 * q * q, N) and M.shape == (N, 2 * q * q)
    assert abs(w.sum() - 4 * np.pi) < 1e-12
    assert np.abs(M @ O - np.eye(N)).max() < 1e-13
    assert np.abs(M @ (pts[:, 0:1] * O) - Ax).max() < 1e-13
    assert np.abs(M @ (pts[:, 1:2] * O) - Ay).max() < 1e-13
    assert np.abs(M @ (pts[:, 2:3] * O) - Az).max() < 1e-13


def test_roe_is_matrix_abs():
    Ax, _, Az = pn.setup_system_matrices(7)
    for A in (Ax, Az):
        absA = pn.roe_abs(A).toarray()
        # |A|^2 = A^2 and |A| is positive semi-definite
        assert np.abs(absA @ absA - A @ A).max() < 1e-9
        assert np.linalg.eigvalsh(0.5 * (absA + absA.T)).min() > -1e-9


def test_eigenvalues_are_legendre_roots():
    # Az's k = 0 block is the Jacobi matrix of the normalised Legendre polynomials
    npn = 7
    _, _, Az = pn.setup_system_matrices(npn)
    lam = np.sort(np.linalg.eigvalsh(Az))
    mu, _ = np.polynomial.legendre.leggauss(npn + 1)
    for m in mu:
        assert np.min(np.abs(lam - m)) < 1e-12
