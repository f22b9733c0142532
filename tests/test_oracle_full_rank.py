"""The full-rank P_N oracle (oracle/full_rank.py) against a literal
transcription of the reference's per-cell loops (SolverCSD.jl:517-586) on a
tiny grid: boundary inflow, solveFluxUpwind!, the four stencil products, the
collision solve of each interior cell, the dose with SMid and the halved first
and last steps. Pure-Python loops, so only a few steps on a 7 x 7 grid."""
import math

import numpy as np

from oracle.full_rank import solve_pn_full
from oracle.settings import Settings
from oracle.solver import SolverCSD


def literal(nx, npn, steps):
    o = SolverCSD(Settings(nx, nx, 4, "csdWaterBeam", nPN=npn))
    s = o.settings
    psi = o.setup_directions()
    NX, NY = s.NCellsX, s.NCellsY
    nq = psi.shape[2]
    N = o.N
    eTrafo, energy = o.csd.eTrafo, o.csd.eGrid
    nE = eTrafo.size
    u = np.zeros((NX * NY, N))
    dose = np.zeros(NX * NY)
    Ax, Az, AAx, AAz = (A.toarray() for A in (o.Ax, o.Az, o.AbsAx, o.AbsAz))
    L = {k: getattr(o.stencil, k).toarray() for k in ("L1x", "L1y", "L2x", "L2y")}
    flux = np.zeros_like(psi)
    for n in range(2, min(nE, steps + 1) + 1):                   # for n = 2:nEnergies
        sigma = o.csd.sigma_at_energy(energy[n - 1])
        dE = eTrafo[n - 1] - eTrafo[n - 2]
        for k in range(nq):                                     # PsiBeam at energy[n], index n-1
            for j in range(NX):
                psi[j, 0, k] = o.psi_beam(o.qReduced[k], energy[n - 1], s.xMid[j], s.yMid[0], n - 1)[0]
                psi[j, -1, k] = o.psi_beam(o.qReduced[k], energy[n - 1], s.xMid[j], s.yMid[-1], n - 1)[0]
            for j in range(NY):
                psi[0, j, k] = o.psi_beam(o.qReduced[k], energy[n - 1], s.xMid[0], s.yMid[j], n - 1)[0]
                psi[-1, j, k] = o.psi_beam(o.qReduced[k], energy[n - 1], s.xMid[-1], s.yMid[j], n - 1)[0]
        Dvec = np.zeros(N)
        for l in range(npn + 1):
            for kk in range(-l, l + 1):
                Dvec[l * l + kk + l] = sigma[l]
        D = sigma[0] - Dvec
        for i in range(1, NX - 1):                              # solveFluxUpwind!
            for j in range(1, NY - 1):
                for q in range(nq):
                    ox, oz = o.qReduced[q, 0], o.qReduced[q, 2]
                    ew = psi[i, j, q] - psi[i - 1, j, q] if ox >= 0 else psi[i + 1, j, q] - psi[i, j, q]
                    ns = psi[i, j, q] - psi[i, j - 1, q] if oz >= 0 else psi[i, j + 1, q] - psi[i, j, q]
                    flux[i, j, q] = ox / s.dx * ew + oz / s.dy * ns
        psi = psi - dE * flux
        psiNew = psi / (1 + dE * sigma[0])
        uT = u - dE * L["L2x"] @ u @ Ax - dE * L["L2y"] @ u @ Az - dE * L["L1x"] @ u @ AAx - dE * L["L1y"] @ u @ AAz
        uT[o.boundaryIdx, :] = 0.0
        uNew = np.zeros_like(u)
        uOUnc = np.zeros(NX * NY)
        for i in range(1, NX - 1):
            for j in range(1, NY - 1):
                idx = i * NY + j
                uNew[idx, :] = (uT[idx, :] + dE * Dvec * (o.MReduced @ psiNew[i, j, :])) / (1 + dE * D)
                uOUnc[idx] = psiNew[i, j, :] @ o.MReduced[0, :]
        uNew[o.boundaryIdx, :] = 0.0
        dose += dE * (uNew[:, 0] + uOUnc) * o.csd.SMid[n - 2] / o.densityVec / (1 + (n == 2 or n == nE))
        u = uNew
        psi = psiNew
    return 0.5 * math.sqrt(o.gamma[0]) * u, dose, psi


def test_full_rank_oracle_matches_literal_loops():
    nx, npn, steps = 8, 2, 12
    u_l, d_l, p_l = literal(nx, npn, steps)
    o = SolverCSD(Settings(nx, nx, 4, "csdWaterBeam", nPN=npn))
    u, d, p = solve_pn_full(o, max_steps=steps)
    assert np.abs(d).max() > 0 and np.abs(u).max() > 0
    np.testing.assert_allclose(d, d_l, rtol=1e-12, atol=1e-12 * np.abs(d_l).max())
    np.testing.assert_allclose(u, u_l, rtol=1e-12, atol=1e-12 * np.abs(u_l).max())
    np.testing.assert_allclose(p, p_l, rtol=1e-12, atol=1e-12 * np.abs(p_l).max())


def test_full_rank_dose_is_positive_and_matches_dlr_scale():
    """The DLR integrators approximate the same transport problem: at r = N the
    fixed-rank DLR dose stays within the discretisation difference of the two
    reference schemes (BC energy index, SMid against trapezoid halves)."""
    from oracle.solver import solve_dlr_fixed

    nx, npn = 21, 3
    N = (npn + 1) ** 2
    _, d_full, _ = solve_pn_full(SolverCSD(Settings(nx, nx, N, "csdWaterBeam", nPN=npn)))
    d_dlr = solve_dlr_fixed(SolverCSD(Settings(nx, nx, N, "csdWaterBeam", nPN=npn)))[4]
    assert d_full.min() >= -1e-12 * d_full.max()
    rel = np.linalg.norm(d_full - d_dlr) / np.linalg.norm(d_full)
    assert rel < 0.5
