"""Oracle pieces of the rank-adaptive integrators (CPU): truncate!'s rank rule
(SolverCSD.jl:3369-3399), the deterministic SVD / basis completion, the
augmented bases of qr([X K]) (:149-153), and checkpoint/resume of the loops."""
import math

import numpy as np
import pytest

from oracle import linalg as la
from oracle.settings import Settings
from oracle.solver import SolverCSD, solve_dlr_bug, solve_dlr_parallel


def _truncate_rank(D, theta, r_cap):
    """truncate!'s rule restated directly: first j with |sum_{i>=j} D_i| < theta ||D||_2."""
    rmax = D.size // 2
    tol = theta * np.linalg.norm(D)
    k = rmax
    for j in range(1, 2 * rmax + 1):
        if abs(np.sum(D[j - 1:2 * rmax])) < tol:
            k = j
            break
    return max(min(k, r_cap), 2)


@pytest.mark.parametrize("D", [
    [10.0, 1.0, 0.5, 0.05, 0.01, 0.0],   # tail from j=4 is 0.06 < 0.1 ||D|| -> keeps 4 (the l1 tail keeps D_j itself)
    [1.0, 1e-3, 1e-9, 0.0],              # keeps 2 (lower clamp reached with a tiny second value)
    [3.0, 2.9, 2.8, 2.7, 2.6, 2.5],      # nothing below tol -> j = 2 rmax ... tail at the last index
])
def test_truncate_rule(D):
    s = Settings(23, 23, 8, "csdWaterBeam", nPN=3)
    sol = SolverCSD(s)
    D = np.array(D)
    m = D.size
    rng = np.random.default_rng(0)
    U, _ = np.linalg.qr(rng.standard_normal((m, m)))
    V, _ = np.linalg.qr(rng.standard_normal((m, m)))
    S = U @ np.diag(D) @ V.T
    X = np.linalg.qr(rng.standard_normal((50, m)))[0]
    W = np.linalg.qr(rng.standard_normal((30, m)))[0]
    Xk, Sk, Wk = sol.truncate(X, S, W)
    k = _truncate_rank(D, s.theta, s.r)
    assert Sk.shape == (k, k)
    np.testing.assert_allclose(np.diag(Sk), D[:k], rtol=1e-12, atol=1e-14)
    # the kept factors reproduce the best rank-k part of X S W^T
    assert np.allclose(Xk.T @ Xk, np.eye(k), atol=1e-12)
    P = X @ (U[:, :k] * D[:k]) @ V[:, :k].T @ W.T
    if k < m and D[k - 1] > D[k] * (1 + 1e-8):
        np.testing.assert_allclose(Xk @ Sk @ Wk.T, P, atol=1e-10 * D[0])


def test_svd_det_completion():
    A = np.zeros((5, 5))
    A[0, 0] = 2.0
    A[1, 2] = 1e-20          # numerically null (below 1e-12 sigma_1)
    U, s, V = la.svd_det(A)
    assert np.allclose(U.T @ U, np.eye(5), atol=1e-14) and np.allclose(V.T @ V, np.eye(5), atol=1e-14)
    assert s[0] == pytest.approx(2.0)
    # null directions: canonical vectors in index order, skipping the range
    np.testing.assert_allclose(np.abs(U[:, 1]), [0, 1, 0, 0, 0], atol=1e-14)
    np.testing.assert_allclose(np.abs(V[:, 1]), [0, 1, 0, 0, 0], atol=1e-14)
    U0, s0, V0 = la.svd_det(np.zeros((3, 3)))
    np.testing.assert_allclose(U0, np.eye(3))
    np.testing.assert_allclose(s0, 0.0)


def test_svd_det_row_completion_is_gauge_free():
    """truncate!'s null directions completed from the rows of X and W: rotating
    the bases (X -> X Q, S -> Q^T S R, W -> W R) leaves X U and W V unchanged."""
    rng = np.random.default_rng(3)
    n, N, m = 40, 12, 5
    X = np.linalg.qr(rng.standard_normal((n, m)))[0]
    W = np.linalg.qr(rng.standard_normal((N, m)))[0]
    S = np.zeros((m, m))
    S[:2, :2] = rng.standard_normal((2, 2))       # rank 2: three null directions
    U, s, V = la.svd_det(S, basis_u=X, basis_v=W)
    assert np.allclose(U.T @ U, np.eye(m), atol=1e-14) and np.allclose(V.T @ V, np.eye(m), atol=1e-14)
    Q = np.linalg.qr(rng.standard_normal((m, m)))[0]
    R = np.linalg.qr(rng.standard_normal((m, m)))[0]
    U2, s2, V2 = la.svd_det(Q.T @ S @ R, basis_u=X @ Q, basis_v=W @ R)
    np.testing.assert_allclose(s2, s, rtol=1e-13, atol=1e-15)
    # range directions up to sign, null directions exactly
    for j in range(m):
        a, b = X @ U[:, j], X @ Q @ U2[:, j]
        sg = 1.0 if j >= 2 else np.sign(a @ b)
        np.testing.assert_allclose(sg * b, a, atol=1e-12)
        a, b = W @ V[:, j], W @ R @ V2[:, j]
        sg = 1.0 if j >= 2 else np.sign(a @ b)
        np.testing.assert_allclose(sg * b, a, atol=1e-12)
    # rows that vanish in the basis are skipped: first accepted candidate is row 2
    Xz = X.copy()
    Xz[:2] = 0.0
    Xz = np.linalg.qr(Xz)[0]
    Uz, _, _ = la.svd_det(S, basis_u=Xz, basis_v=W)
    r2 = Xz[2] - Uz[:, :2] @ (Uz[:, :2].T @ Xz[2])
    np.testing.assert_allclose(Uz[:, 2], r2 / np.linalg.norm(r2), atol=1e-12)


def test_svd_jacobi_relative_accuracy():
    rng = np.random.default_rng(1)
    d = np.array([1.0, 1e-4, 1e-8, 1e-11])
    Q1, _ = np.linalg.qr(rng.standard_normal((4, 4)))
    Q2, _ = np.linalg.qr(rng.standard_normal((4, 4)))
    A = Q1 @ np.diag(d) @ Q2.T
    U, s, V = la.svd_jacobi(A)
    np.testing.assert_allclose(s, d, rtol=1e-5)
    np.testing.assert_allclose(U @ np.diag(s) @ V.T, A, atol=1e-15)


def test_orth_augment_properties():
    rng = np.random.default_rng(2)
    n, r = 60, 5
    X = np.linalg.qr(rng.standard_normal((n, r)))[0]
    X[:3] = 0.0                               # zeroed rows as after X[bnd,:] = 0
    K = X @ rng.standard_normal((r, r)) + 1e-3 * rng.standard_normal((n, r))
    K[:3] = 0.0
    Q = la.orth_augment(X, K, "det", order=np.arange(3))
    assert Q.shape == (n, 2 * r)
    assert np.allclose(Q.T @ Q, np.eye(2 * r), atol=1e-12)
    # span([X K]) is contained in span(Q)
    for A in (X, K):
        assert np.linalg.norm(A - Q @ (Q.T @ A)) <= 1e-10 * np.linalg.norm(A)


def test_orth_augment_rank_deficient_completes_with_candidates():
    n, r = 40, 3
    X = np.zeros((n, r))
    K = np.zeros((n, r))
    K[10:20, 0] = 1.0
    cand = np.array([0, 1, 2, 3, 4, 5, 6])
    Q = la.orth_augment(X, K, "det", order=cand)
    assert np.allclose(Q.T @ Q, np.eye(2 * r), atol=1e-13)
    # Q1 (X has no range) = first candidates; K's range next, then the following candidates
    np.testing.assert_allclose(np.abs(Q[:, 0]), np.eye(n)[0])
    np.testing.assert_allclose(np.abs(Q[:, 3]), K[:, 0] / math.sqrt(10))
    np.testing.assert_allclose(np.abs(Q[:, 4]), np.eye(n)[3])


@pytest.mark.parametrize("fn", [solve_dlr_parallel, solve_dlr_bug])
def test_resume_is_exact(fn):
    s = Settings(23, 23, 8, "csdWaterBeam", nPN=3)
    full = fn(SolverCSD(s), max_steps=12, return_state=True)
    st = fn(SolverCSD(s), max_steps=7, return_state=True)
    rest = fn(SolverCSD(s), max_steps=5, state=st, n_begin=st["n_next"], return_state=True)
    assert np.array_equal(full["dose"], rest["dose"])
    assert np.array_equal(full["X"] @ full["S"] @ full["W"].T, rest["X"] @ rest["S"] @ rest["W"].T)


def test_bug_rejections_repeat_energies():
    s = Settings(30, 30, 12, "csdWaterBeam", nPN=5)
    out = solve_dlr_bug(SolverCSD(s), max_steps=40)
    energies = out[5][0]
    # a rejected step repeats its energy (n = n-1): some energy appears twice in a row
    assert np.any(energies[1:] == energies[:-1])
    ranks = out[5][1]
    assert ranks.max() <= s.r and ranks.min() >= 2


def test_completion_second_scan_fills_a_nearly_full_space():
    """With a wide basis the canonical candidates' residuals average
    sqrt((n - r)/n): the first scan (keep half the norm) can run out, the second
    (keep 1e-3 of it) completes the space."""
    rng = np.random.default_rng(5)
    n, r = 30, 24
    B = np.linalg.qr(rng.standard_normal((n, r)))[0]
    C = la._complete(B, n - r, n)
    Q = np.column_stack([B, C])
    np.testing.assert_allclose(Q.T @ Q, np.eye(n), atol=1e-12)
    # the same basis through the row rule of truncate!'s completion
    m = 8
    W = np.linalg.qr(rng.standard_normal((m + 2, m)))[0]
    keep = np.linalg.qr(rng.standard_normal((m, 6)))[0]
    V = la._complete_rows(keep, m - 6, W)
    Qv = np.column_stack([keep, V])
    np.testing.assert_allclose(Qv.T @ Qv, np.eye(m), atol=1e-12)
