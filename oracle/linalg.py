"""Orthonormal bases for the DLR substeps (oracle).

The reference takes left singular vectors from ``svd!(K)`` (LAPACK gesdd) and
Householder Q factors from ``numpy.linalg.qr`` (``SolverCSD.jl:149-153``). Every
downstream use is covariant under a change of orthonormal basis of the same
column space, so only the SPAN of these factors is observable -- except where
the input is (numerically) rank deficient, where LAPACK completes the basis
with directions fixed by rounding noise. This module offers:

* ``mode="lapack"``: the reference's calls verbatim;
* ``mode="det"``: a deterministic, rank-revealing rule that the CUDA path
  implements too. The numerical range of A is the span of the left singular
  vectors with sigma_j > tol * ||A||_2; missing directions are completed by
  canonical vectors e_c taken in the caller's candidate order (index order by
  default, LAPACK's result for an exactly zero input), each accepted when its
  residual after two Gram-Schmidt passes against the basis so far exceeds 1/2.
"""
from __future__ import annotations

import numpy as np

RANK_TOL = 1e-12


def svd_full(A: np.ndarray):
    """Julia ``svd!(A)`` -> (U, S, V), thin, V not transposed."""
    U, s, Vt = np.linalg.svd(A, full_matrices=False)
    return U, s, Vt.T


def svd_jacobi(A: np.ndarray):
    """SVD of a square matrix by LAPACK's preconditioned one-sided Jacobi
    (dgejsv, JOBA='F': high relative accuracy). ``truncate!``'s l1 tail rule
    keeps directions with sigma / sigma_1 down to ~1e-10; a Householder SVD
    (gesdd) determines their vectors only to eps sigma_1 / sigma_j, a one-sided
    Jacobi SVD to a few eps. Returns (U, s, V), s descending."""
    import scipy.linalg.lapack as lapack

    m = A.shape[0]
    if m == 0 or not np.any(A):
        return np.eye(m), np.zeros(m), np.eye(m)
    sva, u, v, work, _, info = lapack.dgejsv(np.asarray(A, dtype=np.float64, order="F"), joba=2, jobu=0, jobv=0,
                                              jobr=1, jobt=0, jobp=0)
    if info != 0:
        raise RuntimeError(f"dgejsv failed (info {info})")
    scale = work[1] / work[0] if work[0] != 0 else 1.0
    return u[:, :m], sva[:m] * scale, v[:, :m]


def svd_det(A: np.ndarray, tol: float | None = None, basis_u: np.ndarray | None = None,
            basis_v: np.ndarray | None = None):
    """Thin SVD (U, s, V) with the deterministic null-space rule.

    Computed by the one-sided Jacobi SVD (``svd_jacobi``) for relative accuracy.
    Singular vectors of singular values ``s_j <= tol * s_1`` are not fixed by A
    (LAPACK returns rounding-noise directions there). ``truncate!`` keeps such
    directions whenever its l1 tail test or its lower clamp reaches them, so
    they are replaced by canonical vectors in index order, completed against the
    columns kept so far (same acceptance rule as ``orth``). Singular values are
    returned as computed.
    """
    tol = RANK_TOL if tol is None else tol
    U, s, V = svd_jacobi(A)
    m = s.size
    rho = int(np.sum(s > tol * s[0])) if m and s[0] > 0 else 0
    if rho < m:
        if basis_u is not None:
            U = np.column_stack([U[:, :rho], _complete_rows(U[:, :rho], m - rho, basis_u)])
            V = np.column_stack([V[:, :rho], _complete_rows(V[:, :rho], m - rho, basis_v)])
        else:
            U = np.column_stack([U[:, :rho], _complete(U[:, :rho], m - rho, U.shape[0])])
            V = np.column_stack([V[:, :rho], _complete(V[:, :rho], m - rho, V.shape[0])])
    return U, s, V


def _complete_rows(Keep: np.ndarray, need: int, basis: np.ndarray, min_norm: float = 1e-6) -> np.ndarray:
    """Gauge-free completion for the SVD of a small matrix S expressed in the
    columns of ``basis`` (n x m): candidate c is u_c = basis[c, :] (the cell
    indicator e_c projected into span(basis), in basis coordinates), c in index
    order, then the canonical vectors of R^m; rows with ||u_c|| <= min_norm are
    skipped. A candidate is Gram-Schmidt'ed twice against Keep and the vectors
    accepted so far and accepted when the residual keeps at least half of
    ||u_c||. If the candidates run out first (many null directions in a wide
    basis: the canonical vectors' residuals then average sqrt((m - r)/m)), a
    second scan from the first candidate accepts residuals above 1e-3 ||u_c||.
    Rotating the basis rotates the result with it, so basis @ result does not
    depend on the basis chosen for the span."""
    m = Keep.shape[0]
    cols = []
    nrows = basis.shape[0]
    for frac in (0.5, 1e-3):
        c = 0
        while len(cols) < need and c < nrows + m:
            if c < nrows:
                u = np.array(basis[c, :], dtype=np.float64)
                nu = np.linalg.norm(u)
                c += 1
                if not nu > min_norm:
                    continue
            else:
                u = np.zeros(m)
                u[c - nrows] = 1.0
                nu = 1.0
                c += 1
            Bc = np.column_stack([Keep] + cols) if (Keep.shape[1] + len(cols)) else np.zeros((m, 0))
            v = u.copy()
            for _ in range(2):
                if Bc.shape[1]:
                    v = v - Bc @ (Bc.T @ v)
            nv = np.linalg.norm(v)
            if nv > frac * nu:
                cols.append(v / nv)
        if len(cols) >= need:
            break
    if len(cols) < need:
        raise RuntimeError("basis completion ran out of candidates")
    return np.column_stack(cols) if cols else np.zeros((m, 0))


def _complete(B: np.ndarray, need: int, n: int, order=None) -> np.ndarray:
    """``need`` unit vectors completing the columns of B: canonical vectors
    e_c, c in ``order``, Gram-Schmidt'ed twice against B and the vectors taken
    so far, accepted when the residual keeps at least half the norm. If the
    candidates run out first (B nearly fills the space), a second scan from the
    first candidate accepts residuals above 1e-3 (the best canonical candidate
    keeps at least sqrt((n - rank B)/n), so the scan always succeeds)."""
    cols = []
    order = np.arange(n) if order is None else order
    for frac in (0.5, 1e-3):
        it = 0
        while len(cols) < need and it < len(order):
            c = order[it]
            Bc = np.column_stack([B] + cols) if (B.shape[1] + len(cols)) else np.zeros((n, 0))
            v = np.zeros(n)
            v[c] = 1.0
            for _ in range(2):
                if Bc.shape[1]:
                    v = v - Bc @ (Bc.T @ v)
            nv = np.linalg.norm(v)
            if nv > frac:
                cols.append(v / nv)
            it += 1
        if len(cols) >= need:
            break
    if len(cols) < need:
        raise RuntimeError("basis completion ran out of canonical vectors")
    return np.column_stack(cols) if cols else np.zeros((n, 0))


def _range_basis(A: np.ndarray, scale: float, tol: float) -> np.ndarray:
    if A.shape[1] == 0:
        return np.zeros((A.shape[0], 0))
    U, s, _ = np.linalg.svd(A, full_matrices=False)
    rho = int(np.sum(s > tol * scale)) if scale > 0 else 0
    return U[:, :rho]


def orth(A: np.ndarray, mode: str = "lapack", tol: float | None = None, order=None) -> np.ndarray:
    """Orthonormal n x k basis with the span of ``svd!(A).U``."""
    if mode == "lapack":
        U, _, _ = np.linalg.svd(A, full_matrices=False)
        return U
    tol = RANK_TOL if tol is None else tol
    n, k = A.shape
    scale = np.linalg.norm(A, 2) if A.size else 0.0
    B = _range_basis(A, scale, tol)
    if B.shape[1] < k:
        B = np.column_stack([B, _complete(B, k - B.shape[1], n, order)])
    return B


def orth_augment(X: np.ndarray, K: np.ndarray, mode: str = "lapack", tol: float | None = None, order=None) -> np.ndarray:
    """Q of ``py"qr"([X K])`` (``SolverCSD.jl:149-153``), n x (rX + rK).

    Columns ``[:rX]`` span span(X) (completed if X is rank deficient), columns
    ``[rX:]`` span span([X K]) minus span(X) (completed likewise).
    """
    if mode == "lapack":
        Q, _ = np.linalg.qr(np.column_stack([X, K]))
        return Q
    tol = RANK_TOL if tol is None else tol
    n = X.shape[0]
    # scale of the rank cut: the Frobenius norm of [X K] (within sqrt(rX + rK)
    # of the 2-norm, and exactly reproducible from the Gram of [X K])
    scale = np.linalg.norm(np.column_stack([X, K]))
    Q1 = _range_basis(X, scale, tol)
    if Q1.shape[1] < X.shape[1]:
        Q1 = np.column_stack([Q1, _complete(Q1, X.shape[1] - Q1.shape[1], n, order)])
    Kp = K - Q1 @ (Q1.T @ K)
    Kp = Kp - Q1 @ (Q1.T @ Kp)
    Q2 = _range_basis(Kp, scale, tol)
    base = np.column_stack([Q1, Q2])
    if Q2.shape[1] < K.shape[1]:
        base = np.column_stack([base, _complete(base, K.shape[1] - Q2.shape[1], n, order)])
    return base
