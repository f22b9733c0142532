"""``SolverCSD`` and the DLR energy loops (oracle restatement, FP64).

Follows ``code/SolverCSD.jl``: constructor ``:63-146``, ``PsiBeam`` ``:240-276``,
``solveFluxUpwind!`` ``:388-463``, fixed-rank ``SolveFirstCollisionSourceDLR``
``:891-1120``, ``SolveFirstCollisionSourceDLRParallel`` ``:1726-2008``,
``SolveFirstCollisionSourceDLRBUGRejection`` ``:2011-2374`` and ``truncate!``
``:3369-3399``. Julia's in-place mutations (``X[bnd,:] .= 0``, ``S .= ...``) are
kept as numpy in-place writes so that aliasing behaves the same.

Index conventions: cell (i, j) (1-based in the reference) has row
``(i-1)*ny + j``; here 0-based ``i*ny + j``. psi is stored as an (nx, ny, q)
array; ``Mat2Vec(psi)`` is ``psi.reshape(nx*ny, q)``.
"""
from __future__ import annotations

import math

import numpy as np

from . import linalg as la
from . import pn as pnmod
from . import quadrature as qd
from .csd import CSD
from .stencils import Stencils


class SolverCSD:
    """``mutable struct SolverCSD`` + constructor (``SolverCSD.jl:20-146``) at T = Float64."""

    def __init__(self, settings, basis_mode: str = "det"):
        s = settings
        self.settings = s
        self.basis_mode = basis_mode
        self.x = s.x
        self.y = s.y
        self.gamma = np.array([2.0 / (2 * n + 1) for n in range(s.nPN + 1)])
        self.csd = CSD(s)
        Ax, _, Az = pnmod.setup_system_matrices(s.nPN)
        self.Ax_dense, self.Az_dense = Ax, Az
        Axs, _, Azs = pnmod.setup_system_matrices_sparse(s.nPN)
        self.Ax, self.Az = Axs.tocsr(), Azs.tocsr()
        self.AbsAx = pnmod.roe_abs(Ax).tocsr()
        self.AbsAz = pnmod.roe_abs(Az).tocsr()
        self.N = pnmod.n_moments(s.nPN)
        self.density = s.density.astype(np.float64)
        nx, ny = s.NCellsX, s.NCellsY
        self.n_cells = nx * ny
        self.densityVec = self.density.reshape(nx * ny)
        self.dose = np.zeros(nx * ny)
        # boundary cells, SolverCSD.jl:108-131 (0-based rows, order kept)
        bidx = []
        for i in range(nx):
            bidx.append(i * ny + 0)
            bidx.append(i * ny + ny - 1)
        for j in range(ny):
            bidx.append(0 * ny + j)
            bidx.append((nx - 1) * ny + j)
        self.boundaryIdx = np.array(bidx, dtype=np.int64)
        q = s.nPN + 1
        self.Q_points, self.Q_weights = qd.standard_points(q)
        self.O, self.M = qd.compute_trafo_matrices(q, s.nPN)
        self.stencil = Stencils(s)
        # Benchmark problems peak-normalise the angular Gaussian over the
        # quadrature (no ordinate sits exactly on the beam direction).
        self.psi_scale = s.psi_scale
        if s.beam_peak_normalized:
            pts = self.Q_points
            ang = np.exp(-s.sigmaO1Inv * (s.Omega1 - pts[:, 0]) ** 2) * np.exp(-s.sigmaO3Inv * (s.Omega3 - pts[:, 2]) ** 2)
            self.psi_scale = s.psi_scale / ang.max()
        # Completion candidates for rank-deficient bases (see oracle.linalg): the
        # canonical vectors in index order, which is what LAPACK returns for an
        # exactly zero input (identity columns). Spatial candidates are the
        # boundary cells, whose rows are zero in every K the loop builds.
        self.x_completion = np.unique(self.boundaryIdx)
        self.w_completion = np.arange(self.N)
        self.qReduced = None
        self.MReduced = None
        self.OReduced = None
        self.idxBeam = None

    # -- boundary source --------------------------------------------------
    def psi_beam(self, Omega, E, x, y, n):
        """``PsiBeam(obj, Omega, E, x, y, n)`` generic branch (``SolverCSD.jl:275``).

        ``n`` is the reference's 1-based energy index into ``csd.S``. Vectorised
        over ``Omega`` rows and ``x``/``y`` arrays by broadcasting.
        """
        s = self.settings
        E0 = s.eMax
        Om = np.atleast_2d(Omega)
        ang = np.exp(-s.sigmaO1Inv * (s.Omega1 - Om[:, 0]) ** 2) * np.exp(-s.sigmaO3Inv * (s.Omega3 - Om[:, 2]) ** 2)
        return (self.psi_scale * ang * math.exp(-s.sigmaEInv * (E0 - E) ** 2)
                * np.exp(-s.sigmaXInv * (x - s.x0) ** 2) * np.exp(-s.sigmaYInv * (y - s.y0) ** 2)
                * self.csd.S[n - 1] * s.densityMin)

    def setup_directions(self):
        """Direction reduction and psi initial condition (``SolverCSD.jl:910-925``)."""
        s = self.settings
        pts = self.Q_points
        psiBeam = np.array([self.psi_beam(pts[k], s.eMax, s.x0, s.y0, 1)[0] for k in range(pts.shape[0])])
        idx = np.nonzero(psiBeam > 1e-17 * psiBeam.max())[0]
        self.idxBeam = idx
        self.qReduced = pts[idx, :]
        self.MReduced = self.M[:, idx]
        self.OReduced = self.O[idx, :]
        # SetupIC -> IC(...) is zero for the beam problems (settings.jl:341-347)
        return np.zeros((s.NCellsX, s.NCellsY, idx.size))

    def apply_bc(self, psi, E, n):
        """Boundary inflow on the 4 boundary rows/cols for all ordinates (``:977-988``)."""
        s = self.settings
        xm, ym = s.xMid, s.yMid
        Om = self.qReduced
        # psi[j,1,k], psi[j,end,k] over j = 1..nx, then psi[1,j,k], psi[end,j,k] over j = 1..ny
        psi[:, 0, :] = self.psi_beam(Om, E, xm[:, None], ym[0], n)
        psi[:, -1, :] = self.psi_beam(Om, E, xm[:, None], ym[-1], n)
        psi[0, :, :] = self.psi_beam(Om, E, xm[0], ym[:, None], n)
        psi[-1, :, :] = self.psi_beam(Om, E, xm[-1], ym[:, None], n)

    def flux_upwind(self, phi):
        """``solveFluxUpwind!`` (``SolverCSD.jl:388-463``), interior cells only.

        Returns flux with zeros on boundary cells (the reference's ``flux`` buffer
        is allocated zero and only interior entries are ever written).
        """
        s = self.settings
        flux = np.zeros_like(phi)
        ox = self.qReduced[:, 0]
        oz = self.qReduced[:, 2]
        c = phi[1:-1, 1:-1, :]
        xm = phi[:-2, 1:-1, :]
        xp = phi[2:, 1:-1, :]
        ym = phi[1:-1, :-2, :]
        yp = phi[1:-1, 2:, :]
        ew = np.where(ox >= 0.0, c - xm, xp - c)
        ns = np.where(oz >= 0.0, c - ym, yp - c)
        flux[1:-1, 1:-1, :] = (ox / s.dx) * ew + (oz / s.dy) * ns
        return flux

    def flux_limited(self, phi, flux=None):
        """``solveFlux!`` (``SolverCSD.jl:295-386``) with this solver's
        ``qReduced`` and spacing; see ``oracle.flux.limited_flux``."""
        from .flux import limited_flux

        return limited_flux(phi, self.qReduced[:, 0], self.qReduced[:, 2], self.settings.dx, self.settings.dy, flux)

    def sweep(self, psi, dE, sigma0):
        """Uncollided update ``:1000-1005`` incl. the boundary-slab quirk.

        ``psi[boundaryIdx]`` linear-indexes the column-major (nx, ny, q) array, so
        only q-slab 1 is restored, at (a, b) = ((L-1) % nx, (L-1) // nx).
        """
        s = self.settings
        nx = s.NCellsX
        flux = self.flux_upwind(psi / self.density[:, :, None])
        L0 = self.boundaryIdx
        a, b = L0 % nx, L0 // nx
        psiBC = psi[a, b, 0].copy()
        psi[...] = (psi - dE * flux) / (1 + dE * sigma0)
        psi[a, b, 0] = psiBC

    def apply_bc_two_layer(self, psi, E, n):
        """Boundary inflow of ``SolveFirstCollisionSourceDLRHighOrder``
        (``SolverCSD.jl:679-695``): the two outer layers on every side, the
        second layer taking the coordinates of the first. The x-sides (first
        index) are written last, so they win at the corners."""
        s = self.settings
        xm, ym = s.xMid, s.yMid
        Om = self.qReduced
        for jj, yy in ((0, ym[0]), (-1, ym[-1]), (1, ym[0]), (-2, ym[-1])):
            psi[:, jj, :] = self.psi_beam(Om, E, xm[:, None], yy, n)
        for ii, xx in ((0, xm[0]), (-1, xm[-1]), (1, xm[0]), (-2, xm[-1])):
            psi[ii, :, :] = self.psi_beam(Om, E, xx, ym[:, None], n)

    def sweep_limited(self, psi, dE, sigma0):
        """Uncollided update of the HighOrder loop (``SolverCSD.jl:707-713``):
        the second-order limited flux ``solveFlux!`` of psi/rho, which writes
        interior cells 3:N-2 only (the flux buffer keeps zeros on the two outer
        rings), then the same boundary-slab restore as ``sweep``."""
        nx = self.settings.NCellsX
        flux = self.flux_limited(psi / self.density[:, :, None])
        L0 = self.boundaryIdx
        a, b = L0 % nx, L0 // nx
        psiBC = psi[a, b, 0].copy()
        psi[...] = (psi - dE * flux) / (1 + dE * sigma0)
        psi[a, b, 0] = psiBC

    def dvec(self, sigma):
        s = self.settings
        Dv = np.zeros(self.N)
        for l in range(s.nPN + 1):
            for k in range(-l, l + 1):
                Dv[pnmod.global_index(l, k)] = sigma[l]
        return Dv

    def dose_half(self, X, S, W, psi, dE, Sn):
        """``dose += 0.5 dE (X S W[1,:] + uOUnc) S[n] ./ rho`` (``:990-997``)."""
        uOUnc = psi.reshape(self.n_cells, -1) @ self.MReduced[0, :]
        self.dose += 0.5 * dE * (X @ (S @ W[0, :]) + uOUnc) * Sn / self.densityVec

    # Grams used by the streaming substeps
    def _w_grams(self, Wa, Wb):
        return (Wa.T @ (self.Ax @ Wb), Wa.T @ (self.Az @ Wb), Wa.T @ (self.AbsAx @ Wb), Wa.T @ (self.AbsAz @ Wb))

    def _x_grams(self, Xa, Xb):
        st = self.stencil
        return (Xa.T @ (st.L2x @ Xb), Xa.T @ (st.L2y @ Xb), Xa.T @ (st.L1x @ Xb), Xa.T @ (st.L1y @ Xb))

    def _k_stream(self, K, WAxW, WAzW, WAbsAxW, WAbsAzW, dE):
        st = self.stencil
        return K - dE * ((st.L2x @ K) @ WAxW + (st.L2y @ K) @ WAzW + (st.L1x @ K) @ WAbsAxW + (st.L1y @ K) @ WAbsAzW)

    def _l_stream(self, L, XL2xX, XL2yX, XL1xX, XL1yX, dE):
        return L - dE * ((self.Ax @ L) @ XL2xX.T + (self.Az @ L) @ XL2yX.T
                         + (self.AbsAx @ L) @ XL1xX.T + (self.AbsAz @ L) @ XL1yX.T)

    def _s_stream(self, S, G, C, dE, sign=-1.0):
        return S + sign * dE * (G[0] @ S @ C[0] + G[1] @ S @ C[1] + G[2] @ S @ C[2] + G[3] @ S @ C[3])

    def _op_sum(self, G, S, C):
        """sum_d G_d S C_d over the streaming operators (the eta products, ``:2220``)."""
        return G[0] @ S @ C[0] + G[1] @ S @ C[1] + G[2] @ S @ C[2] + G[3] @ S @ C[3]

    def truncate(self, X, S, W):
        """``truncate!`` (``SolverCSD.jl:3369-3399``): l1 tail test, clamp [2, r]."""
        s = self.settings
        # det mode: null directions completed from the rows of X and W (cells,
        # moments in index order), which does not depend on the bases chosen
        U, D, V = la.svd_det(S, basis_u=X, basis_v=W) if self.basis_mode == "det" else la.svd_full(S)
        rMaxTotal = s.r
        rMinTotal = 2
        tol = s.theta * np.linalg.norm(D) ** s.thetaIndex
        rmax = int(math.floor(D.size / 2))
        for j in range(1, 2 * rmax + 1):
            tmp = math.sqrt(np.sum(D[j - 1:2 * rmax]) ** 2)
            if tmp < tol:
                rmax = j
                break
        rmax = min(rmax, rMaxTotal)
        rmax = max(rmax, rMinTotal)
        return X @ U[:, :rmax], np.diag(D[:rmax]), W @ V[:, :rmax]

    def outputs(self, X, S, W, psi):
        U, Sig, V = la.svd_full(S)
        return X @ U, 0.5 * math.sqrt(self.gamma[0]) * Sig, self.O @ (W @ V), W @ V, self.dose, psi


def out_scatter_factor(L, mode, order=None):
    """``W,S1,S2 = svd!(L); S = S2*Diagonal(S1)`` (``SolverCSD.jl:1071-1074``).

    ``mode="det"`` returns W = orth(L) and S = L^T W, the same product W S^T = L.
    """
    if mode == "lapack":
        W, S1, S2 = la.svd_full(L)
        return W, S2 @ np.diag(S1)
    W = la.orth(L, mode, order=order)
    return W, L.T @ W


def init_factors(solver, r):
    """``svd!(zeros)`` factors (``SolverCSD.jl:931-938``): first r identity columns;
    X's boundary rows are then zeroed (``:955``)."""
    s = solver.settings
    n = solver.n_cells
    X = np.eye(n, r)
    W = np.eye(solver.N, r)
    S = np.zeros((r, r))
    X[solver.boundaryIdx, :] = 0.0
    return X, S, W


def _fixed_scatter(solver, X, S, W, psi, Dvec, D, dE):
    """Out-scattering and the in-scattering K/L/S steps of the fixed-rank loops
    (``SolverCSD.jl:1066-1102``; the HighOrder loop repeats them at ``:768-808``).
    X's boundary rows are zeroed in place, as the reference does."""
    s = solver.settings
    mode = solver.basis_mode
    bnd = solver.boundaryIdx
    Mr = solver.MReduced
    # out scattering
    L = W @ S.T
    L = L / (1.0 + dE * D)[:, None]
    W, S = out_scatter_factor(L, mode, solver.w_completion)
    # in scattering, K-step
    X[bnd, :] = 0.0
    K = X @ S
    psiv = psi.reshape(solver.n_cells, -1)
    K = K + dE * psiv @ (Mr.T @ (Dvec[:, None] * W))
    K[bnd, :] = 0.0
    XNew = la.orth(K, mode, order=solver.x_completion)
    MUp = XNew.T @ X
    # L-step
    L = W @ S.T
    L = L + dE * Dvec[:, None] * (Mr @ (psiv.T @ X))
    WNew = la.orth(L, mode, order=solver.w_completion)
    NUp = WNew.T @ W
    W = WNew
    X = XNew
    # S-step
    S = MUp @ S @ NUp.T
    S = S + dE * (X.T @ psiv) @ Mr.T @ (Dvec[:, None] * W)
    return X, S, W


def solve_dlr_fixed(solver: SolverCSD, max_steps: int | None = None, state: dict | None = None,
                    n_begin: int = 2, return_state: bool = False):
    """``SolveFirstCollisionSourceDLR`` (``SolverCSD.jl:891-1120``).

    Returns (X U, 1/2 sqrt(gamma_0) Sigma, O W V, W V, dose, psi). ``max_steps``
    stops after that many energy steps (a bounded sample of the sweep).
    ``state`` (X, S, W, psi, dose after step ``n_begin - 1``) resumes the loop at
    ``n_begin``; ``return_state`` returns that dict for the end of the run.
    """
    s = solver.settings
    mode = solver.basis_mode
    r = s.r
    eTrafo = solver.csd.eTrafo
    energy = solver.csd.eGrid
    Scsd = solver.csd.S
    psi = solver.setup_directions()
    nx, ny = s.NCellsX, s.NCellsY
    X, S, W = init_factors(solver, r)
    if state is not None:
        X, S, W = state["X"].copy(), state["S"].copy(), state["W"].copy()
        psi = state["psi"].reshape(psi.shape).copy()
        solver.dose = state["dose"].copy()
    bnd = solver.boundaryIdx
    nE = eTrafo.size
    dE = eTrafo[1] - eTrafo[0]
    s.dE = dE
    Mr = solver.MReduced
    last = nE if max_steps is None else min(nE, n_begin - 1 + max_steps)
    for n in range(n_begin, last + 1):
        sigma = solver.csd.sigma_at_energy(energy[n - 1])
        solver.apply_bc(psi, energy[n - 2], n - 1)
        solver.dose_half(X, S, W, psi, dE, Scsd[n - 2])
        solver.sweep(psi, dE, sigma[0])
        Dvec = solver.dvec(sigma)
        D = sigma[0] - Dvec
        if n > 2:
            # K-step
            X[bnd, :] = 0.0
            K = X @ S
            C = solver._w_grams(W, W)
            K = solver._k_stream(K, *C, dE)
            XNew = la.orth(K, mode, order=solver.x_completion)
            MUp = XNew.T @ X
            # L-step
            L = W @ S.T
            G = solver._x_grams(X, X)
            L = solver._l_stream(L, *G, dE)
            WNew = la.orth(L, mode, order=solver.w_completion)
            NUp = WNew.T @ W
            W = WNew
            X = XNew
            # S-step
            S = MUp @ S @ NUp.T
            G = solver._x_grams(X, X)
            C = solver._w_grams(W, W)
            S = solver._s_stream(S, G, C, dE)
        X, S, W = _fixed_scatter(solver, X, S, W, psi, Dvec, D, dE)
        solver.dose_half(X, S, W, psi, dE, Scsd[n - 1])
    if return_state:
        return dict(X=X.copy(), S=S.copy(), W=W.copy(), psi=psi.copy(), dose=solver.dose.copy(), n_next=last + 1)
    return solver.outputs(X, S, W, psi)


def rk4_accumulated(Y, dE, f):
    """One classical RK4 step of Y' = f(Y) in the K-step's form
    (``SolverCSD.jl:731-739``): KUP grows stage by stage."""
    k1 = f(Y)
    up = Y + dE * k1 / 6
    k2 = f(Y + 0.5 * dE * k1)
    up = up + 2 * dE * k2 / 6
    k3 = f(Y + 0.5 * dE * k2)
    up = up + 2 * dE * k3 / 6
    k4 = f(Y + dE * k3)
    return up + dE * k4 / 6


def rk4_summed(Y, dE, f):
    """The same step in the L- and S-steps' form (``:751-756``, ``:783-788``)."""
    k1 = f(Y)
    k2 = f(Y + 0.5 * dE * k1)
    k3 = f(Y + 0.5 * dE * k2)
    k4 = f(Y + dE * k3)
    return Y + dE * (k1 + 2 * k2 + 2 * k3 + k4) / 6


def solve_dlr_high_order(solver: SolverCSD, max_steps: int | None = None, state: dict | None = None,
                         n_begin: int = 2, return_state: bool = False):
    """``SolveFirstCollisionSourceDLRHighOrder`` (``SolverCSD.jl:588-889``).

    The fixed-rank loop with a second-order uncollided part and RK4 streaming:
    - inflow on the two outer layers (``:679-695``, ``apply_bc_two_layer``);
    - the limited flux ``solveFlux!`` for the sweep (``:707``);
    - K, L and S streaming with the central operators only (L2x/L2y with
      Ax/Az; no Roe diffusion terms), each advanced by one classical RK4 step
      of size dE (``:724-791``).
    The reference assigns ``KUP .= ...`` without allocating it (an
    UndefVarError when the loop reaches ``n = 3``); here KUP is a fresh array
    of K's shape, the evident intent. The out- and in-scattering steps and the
    dose half-steps are those of the fixed-rank loop. Arguments and return
    value as ``solve_dlr_fixed``.
    """
    s = solver.settings
    mode = solver.basis_mode
    r = s.r
    eTrafo = solver.csd.eTrafo
    energy = solver.csd.eGrid
    Scsd = solver.csd.S
    psi = solver.setup_directions()
    X, S, W = init_factors(solver, r)
    if state is not None:
        X, S, W = state["X"].copy(), state["S"].copy(), state["W"].copy()
        psi = state["psi"].reshape(psi.shape).copy()
        solver.dose = state["dose"].copy()
    bnd = solver.boundaryIdx
    st = solver.stencil
    nE = eTrafo.size
    dE = eTrafo[1] - eTrafo[0]
    s.dE = dE
    last = nE if max_steps is None else min(nE, n_begin - 1 + max_steps)

    for n in range(n_begin, last + 1):
        sigma = solver.csd.sigma_at_energy(energy[n - 1])
        solver.apply_bc_two_layer(psi, energy[n - 2], n - 1)
        solver.dose_half(X, S, W, psi, dE, Scsd[n - 2])
        solver.sweep_limited(psi, dE, sigma[0])
        Dvec = solver.dvec(sigma)
        D = sigma[0] - Dvec
        if n > 2:
            # K-step
            X[bnd, :] = 0.0
            K = X @ S
            WAzW = W.T @ (solver.Az @ W)
            WAxW = W.T @ (solver.Ax @ W)
            K = rk4_accumulated(K, dE, lambda Y: -(st.L2x @ Y) @ WAxW - (st.L2y @ Y) @ WAzW)
            XNew = la.orth(K, mode, order=solver.x_completion)
            MUp = XNew.T @ X
            # L-step
            L = W @ S.T
            XL2xX = X.T @ (st.L2x @ X)
            XL2yX = X.T @ (st.L2y @ X)
            L = rk4_summed(L, dE, lambda Y: -(solver.Ax @ Y) @ XL2xX.T - (solver.Az @ Y) @ XL2yX.T)
            WNew = la.orth(L, mode, order=solver.w_completion)
            NUp = WNew.T @ W
            W = WNew
            X = XNew
            # S-step
            S = MUp @ S @ NUp.T
            XL2xX = X.T @ (st.L2x @ X)
            XL2yX = X.T @ (st.L2y @ X)
            WAzW = W.T @ (solver.Az @ W)
            WAxW = W.T @ (solver.Ax @ W)
            S = rk4_summed(S, dE, lambda Y: -XL2xX @ Y @ WAxW - XL2yX @ Y @ WAzW)
        X, S, W = _fixed_scatter(solver, X, S, W, psi, Dvec, D, dE)
        solver.dose_half(X, S, W, psi, dE, Scsd[n - 1])
    if return_state:
        return dict(X=X.copy(), S=S.copy(), W=W.copy(), psi=psi.copy(), dose=solver.dose.copy(), n_next=last + 1)
    return solver.outputs(X, S, W, psi)

def _augment_tilde(solver, A_old, A_new, side):
    """``Xtmp,_ = py"qr"([X K]); X1Tilde = Xtmp[:, (r+1):end]`` and the full Q.

    Returns (Q, tilde) with Q the n x (r + r') factor and tilde = Q[:, r:].
    """
    order = solver.x_completion if side == "x" else solver.w_completion
    Q = la.orth_augment(A_old, A_new, solver.basis_mode, order=order)
    return Q, Q[:, A_old.shape[1]:]


def _step_prologue(solver, psi, X, S, W, n, dE):
    """BC, first dose half-step, uncollided sweep; returns (sigma, Dvec, D)."""
    energy = solver.csd.eGrid
    sigma = solver.csd.sigma_at_energy(energy[n - 1])
    solver.apply_bc(psi, energy[n - 2], n - 1)
    solver.dose_half(X, S, W, psi, dE, solver.csd.S[n - 2])
    solver.sweep(psi, dE, sigma[0])
    Dvec = solver.dvec(sigma)
    return sigma, Dvec, sigma[0] - Dvec


def solve_dlr_parallel(solver: SolverCSD, max_steps: int | None = None, state: dict | None = None,
                       n_begin: int = 2, return_state: bool = False, on_iter=None):
    """``SolveFirstCollisionSourceDLRParallel`` (``SolverCSD.jl:1726-2008``).

    Returns (X U, 1/2 sqrt(gamma_0) Sigma, O W V, W V, dose, rVec, psi) with
    rVec (2 x nEnergies): row 0 the accumulated pseudo-time t, row 1 the rank.
    ``state`` (X, S, W, psi, dose, optionally t) resumes the loop at ``n_begin``;
    ``return_state`` returns that dict (with ``n_next``) for the end of the run.
    ``on_iter(rank)`` is called at the start of every step with the rank
    entering it and once with None after the last (timing hook).
    """
    s = solver.settings
    mode = solver.basis_mode
    r = int(math.floor(s.r / 2))
    eTrafo = solver.csd.eTrafo
    psi = solver.setup_directions()
    nx, ny = s.NCellsX, s.NCellsY
    X, S, W = init_factors(solver, r)
    bnd = solver.boundaryIdx
    nE = eTrafo.size
    dE = eTrafo[1] - eTrafo[0]
    s.dE = dE
    Mr = solver.MReduced
    rVec = r * np.ones((2, nE))
    t = 0.0
    if state is not None:
        X, S, W = state["X"].copy(), state["S"].copy(), state["W"].copy()
        psi = state["psi"].reshape(psi.shape).copy()
        solver.dose = state["dose"].copy()
        r = S.shape[0]
        t = state.get("t", (n_begin - 2) * dE)
    last = nE if max_steps is None else min(nE, n_begin - 1 + max_steps)
    for n in range(n_begin, last + 1):
        if on_iter is not None:
            on_iter(S.shape[0])
        sigma, Dvec, D = _step_prologue(solver, psi, X, S, W, n, dE)
        if n > 2:
            G = solver._x_grams(X, X)  # before X[bnd] = 0 (:1856-1859)
            C = solver._w_grams(W, W)
            X[bnd, :] = 0.0
            K = X @ S
            K = solver._k_stream(K, *C, dE)
            _, X1T = _augment_tilde(solver, X, K, "x")
            L = W @ S.T
            L = solver._l_stream(L, *G, dE)
            _, W1T = _augment_tilde(solver, W, L, "w")
            S[...] = solver._s_stream(S, G, C, dE)  # S .= S .- dE ...
            SNew = np.zeros((2 * r, 2 * r))
            SNew[:r, :r] = S
            SNew[r:, :r] = X1T.T @ K
            SNew[:r, r:] = L.T @ W1T
            X, S, W = solver.truncate(np.column_stack([X, X1T]), SNew, np.column_stack([W, W1T]))
            r = S.shape[0]
        # out scattering
        L = W @ S.T
        L = L / (1.0 + dE * D)[:, None]
        W, Snew = out_scatter_factor(L, mode, solver.w_completion)
        S[...] = Snew  # S .= S2 * Diagonal(S1)
        # in scattering
        MtDW = Mr.T @ (Dvec[:, None] * W)
        psiv = psi.reshape(solver.n_cells, -1)
        Xtpsi = X.T @ psiv  # before X[bnd] = 0 (:1904)
        X[bnd, :] = 0.0
        K = X @ S
        K = K + dE * psiv @ MtDW
        K[bnd, :] = 0.0
        _, X1T = _augment_tilde(solver, X, K, "x")
        L = W @ S.T
        L = L + dE * Dvec[:, None] * (Mr @ Xtpsi.T)
        _, W1T = _augment_tilde(solver, W, L, "w")
        S[...] = S + dE * Xtpsi @ MtDW
        SNew = np.zeros((2 * r, 2 * r))
        SNew[:r, :r] = S
        SNew[r:, :r] = X1T.T @ K
        SNew[:r, r:] = L.T @ W1T
        solver.dose_half(X, S, W, psi, dE, solver.csd.S[n - 1])
        X, S, W = solver.truncate(np.column_stack([X, X1T]), SNew, np.column_stack([W, W1T]))
        r = S.shape[0]
        rVec[0, n - 1] = t
        rVec[1, n - 1] = r
        t += dE
    if on_iter is not None:
        on_iter(None)
    if return_state:
        return dict(X=X.copy(), S=S.copy(), W=W.copy(), psi=psi.copy(), dose=solver.dose.copy(), t=t,
                    n_next=last + 1, rVec=rVec)
    U, Sig, V = la.svd_full(S)
    return X @ U, 0.5 * math.sqrt(solver.gamma[0]) * Sig, solver.O @ (W @ V), W @ V, solver.dose, rVec, psi


def solve_dlr_bug(solver: SolverCSD, max_steps: int | None = None, state: dict | None = None,
                  n_begin: int = 2, return_state: bool = False, on_iter=None):
    """``SolveFirstCollisionSourceDLRBUGRejection`` (``SolverCSD.jl:2011-2374``).

    The undefined name ``rmax`` (``:2205, :2295``) is read as ``settings.r``,
    the bound the neighbouring branches use (``:2227, :2283``). Rejected steps
    repeat with the doubled basis exactly as the reference does, including the
    psi sweep and first dose half-step already applied (``n = n-1; continue``).
    ``max_steps`` bounds the number of loop iterations. ``state`` (X, S, W, psi,
    dose, optionally t) resumes the loop at energy index ``n_begin``;
    ``return_state`` returns that dict (with ``n_next``) at the end.
    ``on_iter(rank)``, if given, is called at the start of every loop iteration
    with the rank entering it, and once more with None when the loop ends (the
    CPU baseline times iterations by rank with it).

    Returns (X U, 1/2 sqrt(gamma_0) Sigma, O W V, W V, dose, [E rank]^T,
    [E eta], [E bound], psi).
    """
    s = solver.settings
    mode = solver.basis_mode
    rmax = s.r
    r = int(math.floor(s.r / 2))
    eTrafo = solver.csd.eTrafo
    energy = solver.csd.eGrid
    psi = solver.setup_directions()
    nx, ny = s.NCellsX, s.NCellsY
    X, S, W = init_factors(solver, r)
    bnd = solver.boundaryIdx
    nE = eTrafo.size
    dE = eTrafo[1] - eTrafo[0]
    s.dE = dE
    Mr = solver.MReduced
    t = 0.0
    n = 1
    if state is not None:
        X, S, W = state["X"].copy(), state["S"].copy(), state["W"].copy()
        psi = state["psi"].reshape(psi.shape).copy()
        solver.dose = state["dose"].copy()
        r = S.shape[0]
        t = state.get("t", (n_begin - 2) * dE)
        n = n_begin - 1
    timeVec, rankInTime, etaVec, etaVecTime, etaBoundVec = [], [], [], [], []
    iters = 0
    n_next = None
    while t < nE * dE:
        n += 1
        if n == nE:
            n_next = n
            break
        if max_steps is not None and iters >= max_steps:
            n_next = n
            break
        iters += 1
        if on_iter is not None:
            on_iter(r)
        timeVec.append(energy[n - 1])
        rankInTime.append(r)
        sigma, Dvec, D = _step_prologue(solver, psi, X, S, W, n, dE)
        if n > 2:
            G = solver._x_grams(X, X)
            C = solver._w_grams(W, W)
            X[bnd, :] = 0.0
            K = X @ S
            K = solver._k_stream(K, *C, dE)
            X1, X1T = _augment_tilde(solver, X, K, "x")
            Mu = X1.T @ X
            L = W @ S.T
            L = solver._l_stream(L, *G, dE)
            W1, W1T = _augment_tilde(solver, W, L, "w")
            Nu = W1.T @ W
            W = W1
            X = X1
            S = Mu @ S @ Nu.T
            G = solver._x_grams(X, X)
            C = solver._w_grams(W, W)
            Sup = solver._s_stream(S, G, C, dE)
            XUP, SUP, WUP = solver.truncate(X, Sup, W)
            if SUP.shape[0] == 2 * r and 2 * r < rmax:
                r = 2 * r
                n = n - 1
            else:
                Gt = solver._x_grams(X1T, X)
                Ct = solver._w_grams(W, W1T)
                eta = np.linalg.norm(solver._op_sum(Gt, S, Ct))
                etaVec.append(eta)
                etaVecTime.append(energy[n - 1])
                bound = s.c_eta * s.theta * max(1e-7, np.linalg.norm(Sup) ** s.thetaIndex) / dE
                etaBoundVec.append(bound)
                if eta > bound and 2 * r < s.r:
                    r = 2 * r
                    n = n - 1
                    continue
            S = SUP
            X = XUP
            W = WUP
            r = S.shape[0]
        # out scattering
        L = W @ S.T
        L = L / (1.0 + dE * D)[:, None]
        W, Snew = out_scatter_factor(L, mode, solver.w_completion)
        S[...] = Snew
        # in scattering
        MtDW = Mr.T @ (Dvec[:, None] * W)
        psiv = psi.reshape(solver.n_cells, -1)
        Xtpsi = X.T @ psiv
        X[bnd, :] = 0.0
        K = X @ S
        K = K + dE * psiv @ MtDW
        K[bnd, :] = 0.0
        X1, X1T = _augment_tilde(solver, X, K, "x")
        Mu = X1.T @ X
        L = W @ S.T
        L = L + dE * Dvec[:, None] * (Mr @ Xtpsi.T)
        W1, W1T = _augment_tilde(solver, W, L, "w")
        Nu = W1.T @ W
        W = W1
        X = X1
        S = Mu @ S @ Nu.T
        MtDW = Mr.T @ (Dvec[:, None] * W)
        Xtpsi = X.T @ psiv
        Sup = S + dE * Xtpsi @ MtDW
        XUP, SUP, WUP = solver.truncate(X, Sup, W)
        if SUP.shape[0] == 2 * r and 2 * r < s.r:
            r = 2 * r
            n = n - 1
        else:
            MtDWt = Mr.T @ (Dvec[:, None] * W1T)
            Xtpsit = X1T.T @ psiv
            eta = np.linalg.norm(Xtpsit @ MtDWt)
            bound = s.c_eta * s.theta * max(1e-7, np.linalg.norm(SUP) ** s.thetaIndex) / dE
            if eta > bound and 2 * r < rmax:
                r = 2 * r
                n = n - 1
                continue
        S = SUP
        X = XUP
        W = WUP
        r = S.shape[0]
        solver.dose_half(X, S, W, psi, dE, solver.csd.S[n - 1])
        t += dE
    if on_iter is not None:
        on_iter(None)
    if return_state:
        return dict(X=X.copy(), S=S.copy(), W=W.copy(), psi=psi.copy(), dose=solver.dose.copy(), t=t,
                    n_next=n_next if n_next is not None else n + 1, rank=rankInTime, eta=etaVec,
                    bound=etaBoundVec, iters=iters)
    U, Sig, V = la.svd_full(S)
    rank_hist = np.array([timeVec, rankInTime], dtype=float)
    eta_hist = np.array([etaVecTime, etaVec], dtype=float).T
    bound_hist = np.array([etaVecTime, etaBoundVec], dtype=float).T
    return (X @ U, 0.5 * math.sqrt(solver.gamma[0]) * Sig, solver.O @ (W @ V), W @ V, solver.dose,
            rank_hist, eta_hist, bound_hist, psi)


class ReferenceFailure(RuntimeError):
    """The reference loop raises an error at this point of the sweep."""


def solve_dlr_parallel_rejection(solver: SolverCSD, max_steps: int | None = None, state: dict | None = None,
                                 n_begin: int = 2, return_state: bool = False, on_iter=None):
    """``SolveFirstCollisionSourceDLRParallelRejection`` (``SolverCSD.jl:2376-2742``).

    The parallel integrator's augmented step (``:2520-2558`` streaming,
    ``:2600-2642`` scattering: ``S_new = [[Sbar, L^T W~], [X~^T K, 0]]``, then
    ``truncate!``) inside the BUG loop's rejection logic (``:2561-2594``,
    ``:2645-2668``). Readings of the reference, kept here:

    * ``rmax`` (undefined, ``:2561, :2586, :2645, :2660``) is ``settings.r``,
      as for the BUG loop;
    * ``Sup`` (undefined in this function) appears only in the printed message
      of the two rejections (``:2587, :2661``); the tests use ``norm(SUP)``,
      and the message is read as printing that same bound;
    * the loop runs ``while t < (nEnergies-1)*dE`` (``:2467``), not
      ``nEnergies*dE`` as the BUG loop does;
    * ``X0 = X; W0 = W; S0 = S`` (``:2518``) are aliases: the streaming K-step
      (``:2532``; at n = 2 the in-scattering K-step, ``:2618``) zeroes X0's
      boundary rows in place, and at n = 2 the out-scattering
      ``S .= S2*Diagonal(S1)`` (``:2611``) rewrites S0. numpy's in-place
      updates below keep the same aliasing;
    * the first-branch rejections (``size(SUP,1) == 2r``, ``:2561, :2645``) do
      not ``continue``: the truncated factors are kept and only ``n = n-1``
      survives (the dose then uses ``S[n]`` of the decremented n);
    * after a scattering rejection the basis is ``[X0 X~]`` with r0 + r'
      columns (r0 entering the energy, r' after the streaming step) and the
      reference sets ``r = 2r'`` (``:2662-2665``). When the streaming step
      changed the rank (r0 != r') the repeated step's
      ``SNew[1:r,1:r] .= SBar`` (``:2553``) raises a DimensionMismatch, so the
      reference solve fails there; this restatement raises
      :class:`ReferenceFailure` at the rejection instead.

    Same arguments and returns as :func:`solve_dlr_bug`.
    """
    s = solver.settings
    mode = solver.basis_mode
    rmax = s.r
    r = int(math.floor(s.r / 2))
    eTrafo = solver.csd.eTrafo
    energy = solver.csd.eGrid
    psi = solver.setup_directions()
    nx, ny = s.NCellsX, s.NCellsY
    X, S, W = init_factors(solver, r)
    bnd = solver.boundaryIdx
    nE = eTrafo.size
    dE = eTrafo[1] - eTrafo[0]
    s.dE = dE
    Mr = solver.MReduced
    t = 0.0
    n = 1
    if state is not None:
        X, S, W = state["X"].copy(), state["S"].copy(), state["W"].copy()
        psi = state["psi"].reshape(psi.shape).copy()
        solver.dose = state["dose"].copy()
        r = S.shape[0]
        t = state.get("t", (n_begin - 2) * dE)
        n = n_begin - 1
    timeVec, rankInTime, etaVec, etaVecTime, etaBoundVec = [], [], [], [], []
    iters = 0
    n_next = None
    while t < (nE - 1) * dE:
        n += 1
        if n == nE:
            n_next = n
            break
        if max_steps is not None and iters >= max_steps:
            n_next = n
            break
        iters += 1
        if on_iter is not None:
            on_iter(r)
        timeVec.append(energy[n - 1])
        rankInTime.append(r)
        sigma, Dvec, D = _step_prologue(solver, psi, X, S, W, n, dE)
        X0, W0, S0 = X, W, S
        if n > 2:
            G = solver._x_grams(X, X)
            C = solver._w_grams(W, W)
            X[bnd, :] = 0.0
            K = X @ S
            K = solver._k_stream(K, *C, dE)
            _, X1T = _augment_tilde(solver, X, K, "x")
            L = W @ S.T
            L = solver._l_stream(L, *G, dE)
            _, W1T = _augment_tilde(solver, W, L, "w")
            SBar = solver._s_stream(S, G, C, dE)
            SNew = np.zeros((2 * r, 2 * r))
            SNew[:r, :r] = SBar
            SNew[r:, :r] = X1T.T @ K
            SNew[:r, r:] = L.T @ W1T
            Xa, Wa = np.column_stack([X, X1T]), np.column_stack([W, W1T])
            XUP, SUP, WUP = solver.truncate(Xa, SNew, Wa)
            if SUP.shape[0] == 2 * r and 2 * r < rmax:
                r = 2 * r
                n = n - 1
            else:
                Gt = solver._x_grams(X1T, X)
                Ct = solver._w_grams(W, W1T)
                eta = np.linalg.norm(solver._op_sum(Gt, S, Ct))
                etaVec.append(eta)
                etaVecTime.append(energy[n - 1])
                bound = s.c_eta * s.theta * max(1e-7, np.linalg.norm(SUP) ** s.thetaIndex) / dE
                etaBoundVec.append(bound)
                if eta > bound and 2 * r < rmax:
                    S = (Xa.T @ X) @ S @ (W.T @ Wa)
                    X, W = Xa, Wa
                    r = 2 * r
                    n = n - 1
                    continue
            S = SUP
            X = XUP
            W = WUP
            r = S.shape[0]
        # out scattering (S .= S2*Diagonal(S1): in place, so S0 follows at n = 2)
        L = W @ S.T
        L = L / (1.0 + dE * D)[:, None]
        W, Snew = out_scatter_factor(L, mode, solver.w_completion)
        S[...] = Snew
        # in scattering
        MtDW = Mr.T @ (Dvec[:, None] * W)
        psiv = psi.reshape(solver.n_cells, -1)
        Xtpsi = X.T @ psiv
        X[bnd, :] = 0.0
        K = X @ S
        K = K + dE * psiv @ MtDW
        K[bnd, :] = 0.0
        _, X1T = _augment_tilde(solver, X, K, "x")
        L = W @ S.T
        L = L + dE * Dvec[:, None] * (Mr @ Xtpsi.T)
        _, W1T = _augment_tilde(solver, W, L, "w")
        SBar = S + dE * Xtpsi @ MtDW
        SNew = np.zeros((2 * r, 2 * r))
        SNew[:r, :r] = SBar
        SNew[r:, :r] = X1T.T @ K
        SNew[:r, r:] = L.T @ W1T
        XUP, SUP, WUP = solver.truncate(np.column_stack([X, X1T]), SNew, np.column_stack([W, W1T]))
        if SUP.shape[0] == 2 * r and 2 * r < rmax:
            r = 2 * r
            n = n - 1
        else:
            MtDWt = Mr.T @ (Dvec[:, None] * W1T)
            Xtpsit = X1T.T @ psiv
            eta = np.linalg.norm(Xtpsit @ MtDWt)
            bound = s.c_eta * s.theta * max(1e-7, np.linalg.norm(SUP) ** s.thetaIndex) / dE
            if eta > bound and 2 * r < rmax:
                if X0.shape[1] != r:
                    raise ReferenceFailure(f"scattering rejection at energy index {n} after the streaming step changed "
                                           f"the rank ({X0.shape[1]} -> {r}): the reference's next step raises "
                                           f"DimensionMismatch (SolverCSD.jl:2553)")
                Xa, Wa = np.column_stack([X0, X1T]), np.column_stack([W0, W1T])
                S = (Xa.T @ X0) @ S0 @ (W0.T @ Wa)
                X, W = Xa, Wa
                r = S.shape[0]
                n = n - 1
                continue
        S = SUP
        X = XUP
        W = WUP
        r = S.shape[0]
        solver.dose_half(X, S, W, psi, dE, solver.csd.S[n - 1])
        t += dE
    if on_iter is not None:
        on_iter(None)
    if return_state:
        return dict(X=X.copy(), S=S.copy(), W=W.copy(), psi=psi.copy(), dose=solver.dose.copy(), t=t,
                    n_next=n_next if n_next is not None else n + 1, rank=rankInTime, eta=etaVec,
                    bound=etaBoundVec, iters=iters)
    U, Sig, V = la.svd_full(S)
    rank_hist = np.array([timeVec, rankInTime], dtype=float)
    eta_hist = np.array([etaVecTime, etaVec], dtype=float).T
    bound_hist = np.array([etaVecTime, etaBoundVec], dtype=float).T
    return (X @ U, 0.5 * math.sqrt(solver.gamma[0]) * Sig, solver.O @ (W @ V), W @ V, solver.dose,
            rank_hist, eta_hist, bound_hist, psi)
