"""Full-rank P_N first-collision solver (oracle restatement of
``SolveFirstCollisionSource``, ``code/SolverCSD.jl:465-586``), FP64.

Test infrastructure only: the GPU path (``titus_pn_full_*``) is checked
against it. The collided flux is the full moment matrix u (n cells x N
moments, row i*ny + j); per energy step n = 2..nE:

* sigma = SigmaAtEnergy(energy[n]); Dvec[GlobalIndex(l,k)] = sigma_l;
  D = sigma_0 - Dvec (``:530-538``);
* boundary inflow at energy[n] with csd.S[n-1] (``PsiBeam(..., energy[n], ..., n-1)``,
  ``:517-527``), upwind sweep, psi <- (psi - dE flux) / (1 + dE sigma_0)
  (``:541-545``); the boundary cells' flux is zero, so they decay too;
* uTilde = u - dE (L2x u Ax + L2y u Az + L1x u |Ax| + L1y u |Az|), boundary
  rows zeroed (``:548-549``);
* interior cells: uNew = (uTilde + dE Dvec . (MReduced psiNew)) / (1 + dE D),
  uOUnc = psiNew . MReduced[0,:] (``:552-559``); boundary rows of uNew zero;
* dose += dE (uNew[:,0] + uOUnc) SMid[n-1] / rho / (1 + (n == 2 or n == nE))
  (``:575``).

Returns (1/2 sqrt(gamma_0) u, dose, psi) like the reference (``:585``).
"""
from __future__ import annotations

import math

import numpy as np

from .solver import SolverCSD


def sigma_vectors(solver: SolverCSD, n: int):
    """sigma_l at energy[n] (1-based n, ``:530``) and the per-moment Dvec, D (``:533-540``)."""
    sig = solver.csd.sigma_at_energy(solver.csd.eGrid[n - 1])
    Dvec = solver.dvec(sig)
    return sig, Dvec, sig[0] - Dvec


def solve_pn_full(solver: SolverCSD, max_steps: int | None = None, state: dict | None = None, n_begin: int = 2,
                  return_state: bool = False):
    s = solver.settings
    eTrafo = solver.csd.eTrafo
    energy = solver.csd.eGrid
    nx, ny = s.NCellsX, s.NCellsY
    n_cells = nx * ny
    N = solver.N
    psi = solver.setup_directions()
    Mr = solver.MReduced
    nE = eTrafo.size
    dE = eTrafo[1] - eTrafo[0]
    s.dE = dE
    u = np.zeros((n_cells, N))
    if state is not None:
        u = state["u"].copy()
        psi = state["psi"].reshape(psi.shape).copy()
        solver.dose = state["dose"].copy()
    st = solver.stencil
    bnd = solver.boundaryIdx
    inner = np.zeros((nx, ny), dtype=bool)
    inner[1:-1, 1:-1] = True
    inner = inner.ravel()
    last = nE if max_steps is None else min(nE, n_begin - 1 + max_steps)
    for n in range(n_begin, last + 1):
        sig, Dvec, D = sigma_vectors(solver, n)
        dE = eTrafo[n - 1] - eTrafo[n - 2]
        solver.apply_bc(psi, energy[n - 1], n - 1)
        flux = solver.flux_upwind(psi)
        psi = psi - dE * flux
        psi_new = psi / (1.0 + dE * sig[0])
        # u A_d as (A_d^T u^T)^T: sparse times dense, the reference's u*Ax order of factors
        uA = [np.asarray((A.T @ u.T).T) for A in (solver.Ax, solver.Az, solver.AbsAx, solver.AbsAz)]
        uT = (u - dE * (st.L2x @ uA[0]) - dE * (st.L2y @ uA[1]) - dE * (st.L1x @ uA[2]) - dE * (st.L1y @ uA[3]))
        uT[bnd, :] = 0.0
        pv = psi_new.reshape(n_cells, -1)
        u_new = np.zeros_like(u)
        src = pv[inner] @ Mr.T                       # (MReduced psiNew) per interior cell
        u_new[inner] = (uT[inner] + dE * Dvec[None, :] * src) / (1.0 + dE * D)[None, :]
        u_unc = np.zeros(n_cells)
        u_unc[inner] = pv[inner] @ Mr[0, :]
        u_new[bnd, :] = 0.0
        solver.dose += dE * (u_new[:, 0] + u_unc) * solver.csd.SMid[n - 2] / solver.densityVec / (
            1 + (n == 2 or n == nE))
        u = u_new
        psi = psi_new
    if return_state:
        return dict(u=u.copy(), psi=psi.copy(), dose=solver.dose.copy(), n_next=last + 1)
    return 0.5 * math.sqrt(solver.gamma[0]) * u, solver.dose, psi


def _pn_step_pieces(solver: SolverCSD, n: int):
    """Per-step constants of ``solve_pn_full``'s step n: (dE_n, D, Dvec, c_n)
    with c_n = dE SMid[n-1] / (1 + (n == 2 or n == nE)) the dose weight."""
    eTrafo = solver.csd.eTrafo
    nE = eTrafo.size
    _, Dvec, D = sigma_vectors(solver, n)
    dE = eTrafo[n - 1] - eTrafo[n - 2]
    c = dE * solver.csd.SMid[n - 2] / (1 + (n == 2 or n == nE))
    return dE, D, Dvec, c


def inflow_factor(solver: SolverCSD, E: float, n: int):
    """PsiBeam without its spatial factor: the inflow of every reduced ordinate
    at energy E with csd.S[n-1] (``SolverCSD.jl:275``), so that the boundary
    value of cell c is ``bc_profile[c] * inflow_factor``."""
    s = solver.settings
    Om = solver.qReduced
    ang = np.exp(-s.sigmaO1Inv * (s.Omega1 - Om[:, 0]) ** 2) * np.exp(-s.sigmaO3Inv * (s.Omega3 - Om[:, 2]) ** 2)
    return solver.psi_scale * ang * math.exp(-s.sigmaEInv * (s.eMax - E) ** 2) * solver.csd.S[n - 1] * s.densityMin


def beam_profile(settings, x0: float | None = None, y0: float | None = None):
    """Spatial factor of PsiBeam at every cell (row i*ny + j) for a beam centred at (x0, y0)."""
    s = settings
    x0 = s.x0 if x0 is None else x0
    y0 = s.y0 if y0 is None else y0
    xm = s.xMid[np.arange(s.NCellsX * s.NCellsY) // s.NCellsY]
    ym = s.yMid[np.arange(s.NCellsX * s.NCellsY) % s.NCellsY]
    return np.exp(-s.sigmaXInv * (xm - x0) ** 2) * np.exp(-s.sigmaYInv * (ym - y0) ** 2)


def flux_upwind_T(solver: SolverCSD, w):
    """Transpose of ``solver.flux_upwind`` (the interior-cell upwind differences
    of ``solveFluxUpwind!``, ``SolverCSD.jl:388-463``) applied to w (nx, ny, q)."""
    s = solver.settings
    ax = solver.qReduced[:, 0] / s.dx
    az = solver.qReduced[:, 2] / s.dy
    px = solver.qReduced[:, 0] >= 0.0
    pz = solver.qReduced[:, 2] >= 0.0
    W = w[1:-1, 1:-1, :]
    out = np.zeros_like(w)
    # ew = c - xm (Omega_x >= 0) or xp - c: coefficient +ax on c and -ax on xm, or +ax on xp and -ax on c
    out[1:-1, 1:-1, :] += np.where(px, ax * W, -ax * W)
    out[:-2, 1:-1, :] += np.where(px, -ax * W, 0.0)
    out[2:, 1:-1, :] += np.where(px, 0.0, ax * W)
    out[1:-1, 1:-1, :] += np.where(pz, az * W, -az * W)
    out[1:-1, :-2, :] += np.where(pz, -az * W, 0.0)
    out[1:-1, 2:, :] += np.where(pz, 0.0, az * W)
    return out


def pn_full_dose_adjoint(solver: SolverCSD, g, max_steps: int | None = None, bc_profile=None):
    """Discrete adjoint of ``solve_pn_full``'s dose: gradients of a dose
    objective J with respect to the cell densities and to the inflow profile.

    ``g`` is dJ/d(dose) (n cells), or a callable taking the dose and returning
    it. ``bc_profile`` (n) replaces PsiBeam's spatial factor on the boundary
    cells (a weighted sum of spot profiles for a treatment plan; None keeps the
    settings' beam). Returns (dose, dJ/drho, dJ/dprofile): the last is nonzero
    on boundary cells only, and for a plan with profile sum_s w_s p_s the
    spot-weight gradient is p_s . dJ/dprofile. The energy grid (the tau step
    follows min(rho) when Settings is built) and PsiBeam's rho_min stay fixed.

    It is the exact transpose of the forward recursion, run from the last
    energy step back to the first:

    * forward step n: psi_bc = inflow on boundary cells, psi' = (psi_bc - dE F
      psi_bc) / (1 + dE sigma_0); V_d = u A_d, uT = u - dE sum_d L_d V_d with
      the stencils L_d = Ltilde_d diag(1/rho) (stencils.jl: every entry carries
      1/rho of its column cell), boundary rows zero, u' = P_int (uT + dE Dvec .
      (MReduced psi')) / (1 + dE D), dose += c_n (u'[:,0] + uOUnc) / rho;
    * backward: lambda (adjoint of u') gets g c_n / rho in its moment 0;
      mu = P_int lambda / (1 + dE D); Y_d = L_d^T mu;
      dJ/drho += (dE / rho) sum_d rowsum(Y_d * V_d);
      lambda <- mu - dE sum_d Y_d A_d^T (the adjoint of the previous u);
      psibar' += P_int (dE (mu Dvec) MReduced + g c_n / rho MReduced[0, :]);
      psibar_bc = (psibar' - dE F^T psibar') / (1 + dE sigma_0); its boundary
      cells are the inflow's sensitivity (dJ/dprofile += psibar_bc . inflow
      factor), its interior cells carry to the previous step;
    * the explicit 1/rho of the dose adds -g dose / rho.

    The oracle keeps every step's u in memory, so it is for small cases (the
    GPU path checkpoints u and psi and recomputes). TEST INFRASTRUCTURE ONLY.
    """
    s = solver.settings
    eTrafo = solver.csd.eTrafo
    energy = solver.csd.eGrid
    nx, ny = s.NCellsX, s.NCellsY
    n_cells = nx * ny
    N = solver.N
    psi = solver.setup_directions()
    Mr = solver.MReduced
    nE = eTrafo.size
    u = np.zeros((n_cells, N))
    st = solver.stencil
    ops = (solver.Ax, solver.Az, solver.AbsAx, solver.AbsAz)
    Ls = (st.L2x, st.L2y, st.L1x, st.L1y)
    bnd = solver.boundaryIdx
    inner = np.zeros((nx, ny), dtype=bool)
    inner[1:-1, 1:-1] = True
    inner = inner.ravel()
    bmask = ~inner.reshape(nx, ny)
    rho = solver.densityVec
    dose = np.zeros(n_cells)
    last = nE if max_steps is None else min(nE, 1 + max_steps)
    prof = None if bc_profile is None else np.asarray(bc_profile, dtype=np.float64).reshape(nx, ny)
    u_hist = {}
    for n in range(2, last + 1):
        sig, Dvec, D = sigma_vectors(solver, n)
        dE = eTrafo[n - 1] - eTrafo[n - 2]
        if prof is None:
            solver.apply_bc(psi, energy[n - 1], n - 1)
        else:
            psi[bmask, :] = prof[bmask][:, None] * inflow_factor(solver, energy[n - 1], n - 1)[None, :]
        psi = psi - dE * solver.flux_upwind(psi)
        psi_new = psi / (1.0 + dE * sig[0])
        V = [np.asarray((A.T @ u.T).T) for A in ops]
        u_hist[n] = u
        uT = u - dE * sum(L @ Vd for L, Vd in zip(Ls, V))
        uT[bnd, :] = 0.0
        pv = psi_new.reshape(n_cells, -1)
        u_new = np.zeros_like(u)
        u_new[inner] = (uT[inner] + dE * Dvec[None, :] * (pv[inner] @ Mr.T)) / (1.0 + dE * D)[None, :]
        u_unc = np.zeros(n_cells)
        u_unc[inner] = pv[inner] @ Mr[0, :]
        _, _, _, c = _pn_step_pieces(solver, n)
        dose += c * (u_new[:, 0] + u_unc) / rho
        u = u_new
        psi = psi_new
    g = np.asarray(g(dose) if callable(g) else g, dtype=np.float64)
    lam = np.zeros((n_cells, N))
    psibar = np.zeros((nx, ny, Mr.shape[1]))
    grad = np.zeros(n_cells)
    gprof = np.zeros((nx, ny))
    for n in range(last, 1, -1):
        dE, D, Dvec, c = _pn_step_pieces(solver, n)
        sig, _, _ = sigma_vectors(solver, n)
        lam[:, 0] += g * c / rho
        mu = lam / (1.0 + dE * D)[None, :]
        mu[~inner, :] = 0.0
        Y = [np.asarray(L.T @ mu) for L in Ls]
        V = [np.asarray((A.T @ u_hist[n].T).T) for A in ops]
        grad += (dE / rho) * sum(np.sum(Yd * Vd, axis=1) for Yd, Vd in zip(Y, V))
        lam = mu - dE * sum(np.asarray((A @ Yd.T).T) for A, Yd in zip(ops, Y))
        # psi' feeds the in-scattering source and uOUnc of interior cells
        pb = psibar.reshape(n_cells, -1)
        pb[inner] += dE * (mu[inner] * Dvec[None, :]) @ Mr + np.outer(g[inner] * c / rho[inner], Mr[0, :])
        w = psibar / (1.0 + dE * sig[0])
        pbc = w - dE * flux_upwind_T(solver, w)
        gprof[bmask] += pbc[bmask] @ inflow_factor(solver, energy[n - 1], n - 1)
        pbc[bmask, :] = 0.0
        psibar = pbc
    grad += -g * dose / rho
    return dose, grad, gprof.ravel()
