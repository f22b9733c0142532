"""Three-dimensional extension of the CSD scheme (oracle, FP64).

TEST INFRASTRUCTURE ONLY: the GPU 3D paths are checked against it; the package
never imports it.

The reference solves 2D problems only: ``code/stencils.jl:7-130`` builds x and
y stencils, ``code/SolverCSD.jl:1017-1063`` streams with the pairs
(L2x, Ax), (L2y, Az), (L1x, |Ax|), (L1y, |Az|), and ``solveFluxUpwind!``
(``:388-463``) sweeps in x and y with the ordinate components Omega_x and
Omega_z. This module adds a z direction to the same scheme, with no other
change:

* cell (i, j, k) has row ``(k*nx + i)*ny + j`` (z slowest): every z layer is a
  2D grid in the reference's row order, the x / y neighbours keep their row
  offsets (ny, 1) and the z neighbours are nx*ny rows away. Boundary (ghost)
  cells are the cells on any of the six faces;
* z streams with the P_N matrix Ay (``PNSystem.jl:142-194``, built but unused in
  2D; it equals M diag(Omega_y) O like Ax and Az) and its Roe |Ay|
  (``SolverCSD.jl:83-97``). The density-weighted stencils L2z, L1z are the x / y
  rows of ``stencils.jl`` with dz. The operator list is
  (L2x Ax, L2y Az, L1x |Ax|, L1y |Az|, L2z Ay, L1z |Ay|): the 2D list with the
  z pair appended, summed in that order;
* the uncollided sweep adds (Omega_y / dz) times the upwind z difference;
* PsiBeam gains exp(-sigmaO2Inv (Omega2 - Omega_y)^2) and
  exp(-sigmaZInv (z - z0)^2) and is applied on every face cell;
* the sweep's boundary-slab quirk (``psi[boundaryIdx] .= psiBC`` restores the
  ordinate-0 value only at the column-major positions of the 2D boundary
  indices, ``:1000-1005``) is applied in every z layer.

Pinned by reduction (``tests/test_oracle_3d.py``): a three-layer extrusion of a
2D problem with dz = 1e30 (every z coupling is ~1e-30 of the in-plane ones) and
no z or Omega_y beam factors reproduces the 2D oracle on its middle layer, for
the full-rank P_N loop and the rank-adaptive BUG loop.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

from . import pn as pnmod
from . import quadrature as qd
from .csd import CSD
from .solver import SolverCSD


def seeded_spheres(ncx: int, ncy: int, ncz: int, L: float, seed: int, n_lung: int = 3, n_bone: int = 1,
                   rho_water: float = 1.0, rho_lung: float = 0.25, rho_bone: float = 1.85,
                   rmin: float = 0.5, rmax: float = 2.0) -> np.ndarray:
    """Water cube [0, L]^3 with random lung, then bone spheres from ``default_rng(seed)``.

    Centres are uniform in the inner 80 % of the cube, radii U(rmin, rmax) cm.
    Returns density indexed [k, i, j] = (z, x, y).
    """
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, L, ncx)
    ys = np.linspace(0.0, L, ncy)
    zs = np.linspace(0.0, L, ncz)
    Z, X, Y = np.meshgrid(zs, xs, ys, indexing="ij")
    rho = np.full((ncz, ncx, ncy), rho_water)
    for val in [rho_lung] * n_lung + [rho_bone] * n_bone:
        c = rng.uniform(0.1 * L, 0.9 * L, 3)
        rad = rng.uniform(rmin, rmax)
        rho[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= rad * rad] = val
    return rho


def _ghost_grid(a: float, b: float, ncells: int):
    """``settings.jl:315-325``: cell centres spanning [a, b] with the ghost shift."""
    x = np.linspace(a, b, ncells)
    dx = x[1] - x[0]
    x = np.concatenate([[x[0] - dx], x]) + dx / 2
    return x, x[:-1] + 0.5 * dx, dx


class Settings3D:
    """Settings of the 3D problems (fields named like ``Settings``).

    ``"csdProton3D"``: a 96^3 grid at 1 mm ([0, 9.5]^3 cm with the reference's
    ghost-cell grid), seeded water / lung / bone spheres, a proton pencil beam
    along +x entering at x = 0 centred at (y0, z0) = (4.75, 4.75) cm (spatial
    sigma 0.3 cm, angular sigma 0.01 rad about +x), 90 -> 1 MeV with
    S(E) = (250 / E) ln(1 + 0.07 E) MeV cm^2/g, Henyey-Greenstein
    sigma_l = 100 * 0.95^l cm^-1, P_13, rank cap 40, theta = 1e-2.
    The energy step follows the explicit scheme's stability bound in
    transformed energy, dtau = tau_cfl min(dx, dy, dz) min(rho) with
    tau_cfl = 1/3 (the 2D problems' 1/2 scaled by 2/3 for the third direction).
    """

    def __init__(self, Nx: int = 97, Ny: int = 97, Nz: int = 97, r: int = 40, problem: str = "csdProton3D",
                 nPN: int = 13, seed: int = 20240605, nEnergies: int = 0, tau_cfl: float = 1.0 / 3.0,
                 L: float = 9.5):
        if problem != "csdProton3D":
            raise ValueError(f"3D problem {problem!r} is not defined")
        self.problem, self.particle = problem, "Protons"
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.NCellsX, self.NCellsY, self.NCellsZ = Nx - 1, Ny - 1, Nz - 1
        self.a, self.b, self.c, self.d, self.e, self.f = 0.0, L, 0.0, L, 0.0, L
        self.x, self.xMid, self.dx = _ghost_grid(0.0, L, self.NCellsX)
        self.y, self.yMid, self.dy = _ghost_grid(0.0, L, self.NCellsY)
        self.z, self.zMid, self.dz = _ghost_grid(0.0, L, self.NCellsZ)
        self.eRest = 938.26
        self.eMax, self.eMin = 90.0, 1.0
        self.stopping = "proton_log1p"
        self.hg_g, self.sigmaT_hg = 0.95, 100.0
        self.x0, self.y0, self.z0 = 0.0, 0.5 * L, 0.5 * L
        self.Omega1, self.Omega2, self.Omega3 = 1.0, 0.0, 0.0
        self.densityMin = 1.0
        self.sigmaXInv = self.sigmaYInv = self.sigmaZInv = 1.0 / (2 * 0.3**2)
        self.sigmaO1Inv = self.sigmaO2Inv = self.sigmaO3Inv = 1.0 / (2 * 0.01**2)
        self.sigmaEInv = 1.0
        self.psi_scale = 1e5
        self.beam_peak_normalized = True
        self.seed = seed
        self.density = seeded_spheres(self.NCellsX, self.NCellsY, self.NCellsZ, L, seed)
        self.r = r
        self.theta, self.thetaIndex, self.c_eta = 1e-2, 1.0, 5.0
        self.nPN = nPN
        self.nEnergies = nEnergies
        self.tau_cfl = tau_cfl
        self.cfl = tau_cfl
        self.dE = tau_cfl * min(self.dx, self.dy, self.dz) * self.density.min()

    @classmethod
    def extrude(cls, s2, nz: int = 3, dz: float = 1e30):
        """A z extrusion of the 2D settings ``s2`` (``oracle.settings.Settings``):
        ``nz`` identical layers of its density, dz = ``dz``, no z or Omega_y beam
        factors. With dz = 1e30 the middle layers evolve as the 2D problem."""
        o = cls.__new__(cls)
        o.__dict__.update({k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in s2.__dict__.items()})
        o.Nz, o.NCellsZ = nz + 1, nz
        o.dz = float(dz)
        o.zMid = (np.arange(nz) - (nz - 1) / 2) * o.dz
        o.z0 = 0.0
        o.Omega2 = 0.0
        o.sigmaZInv = 0.0
        o.sigmaO2Inv = 0.0
        o.density = np.repeat(np.asarray(s2.density, dtype=np.float64)[None, :, :], nz, axis=0)
        return o


class Stencils3D:
    """``stencils.jl:12-130`` rows in x and y plus the same rows in z, for the
    cells interior in all three directions (row ``(k*nx + i)*ny + j``)."""

    def __init__(self, s):
        rho = s.density
        nz, nx, ny = s.NCellsZ, s.NCellsX, s.NCellsY
        n = nz * nx * ny
        kk, ii, jj = np.meshgrid(np.arange(1, nz - 1), np.arange(1, nx - 1), np.arange(1, ny - 1), indexing="ij")
        kk, ii, jj = kk.ravel(), ii.ravel(), jj.ravel()

        def row(k, i, j):
            return (k * nx + i) * ny + j

        idx = row(kk, ii, jj)
        nbr = {"x": ((kk, ii - 1, jj), (kk, ii + 1, jj), s.dx), "y": ((kk, ii, jj - 1), (kk, ii, jj + 1), s.dy),
               "z": ((kk - 1, ii, jj), (kk + 1, ii, jj), s.dz)}
        for ax, (m, p, h) in nbr.items():
            rows3 = np.concatenate([idx, idx, idx])
            cols = np.concatenate([row(*m), idx, row(*p)])
            vals = np.concatenate([-1 / 2 / h / rho[m], 2.0 / 2 / h / rho[kk, ii, jj], -1 / 2 / h / rho[p]])
            setattr(self, "L1" + ax, sp.csr_matrix((vals, (rows3, cols)), shape=(n, n)))
            rows2 = np.concatenate([idx, idx])
            cols = np.concatenate([row(*m), row(*p)])
            vals = np.concatenate([-1 / 2 / h / rho[m], 1 / 2 / h / rho[p]])
            setattr(self, "L2" + ax, sp.csr_matrix((vals, (rows2, cols)), shape=(n, n)))


class SolverCSD3D(SolverCSD):
    """The solver data of ``SolverCSD`` (``SolverCSD.jl:63-146``) for a 3D grid.
    psi is held as an (nz, nx, ny, q) array, so ``psi.reshape(n, q)`` has the
    cells' row order."""

    def __init__(self, settings, basis_mode: str = "det"):
        s = settings
        self.settings = s
        self.basis_mode = basis_mode
        self.x, self.y = s.x, s.y
        self.gamma = np.array([2.0 / (2 * n + 1) for n in range(s.nPN + 1)])
        self.csd = CSD(s)
        Ax, Ay, Az = pnmod.setup_system_matrices(s.nPN)
        self.Ax_dense, self.Ay_dense, self.Az_dense = Ax, Ay, Az
        Axs, Ays, Azs = pnmod.setup_system_matrices_sparse(s.nPN)
        self.Ax, self.Ay, self.Az = Axs.tocsr(), Ays.tocsr(), Azs.tocsr()
        self.AbsAx = pnmod.roe_abs(Ax).tocsr()
        self.AbsAy = pnmod.roe_abs(Ay).tocsr()
        self.AbsAz = pnmod.roe_abs(Az).tocsr()
        self.N = pnmod.n_moments(s.nPN)
        nz, nx, ny = s.NCellsZ, s.NCellsX, s.NCellsY
        self.n_cells = nz * nx * ny
        self.density = np.asarray(s.density, dtype=np.float64)
        self.densityVec = self.density.reshape(self.n_cells)
        self.dose = np.zeros(self.n_cells)
        face = np.zeros((nz, nx, ny), dtype=bool)
        face[0], face[-1], face[:, 0], face[:, -1], face[:, :, 0], face[:, :, -1] = (True,) * 6
        self.face = face
        self.boundaryIdx = np.nonzero(face.ravel())[0]
        q = s.nPN + 1
        self.Q_points, self.Q_weights = qd.standard_points(q)
        self.O, self.M = qd.compute_trafo_matrices(q, s.nPN)
        self.stencil = Stencils3D(s)
        self.psi_scale = s.psi_scale
        if s.beam_peak_normalized:
            self.psi_scale = s.psi_scale / self._angular(self.Q_points).max()
        self.x_completion = self.boundaryIdx.copy()
        self.w_completion = np.arange(self.N)
        # the 2D boundary-slab restore positions (a, b) = (L % nx, L // nx) of the
        # reference's boundary order, in every z layer
        bidx = []
        for i in range(nx):
            bidx += [i * ny, i * ny + ny - 1]
        for j in range(ny):
            bidx += [j, (nx - 1) * ny + j]
        L0 = np.array(bidx, dtype=np.int64)
        self.restore_ab = (L0 % nx, L0 // nx)
        st = self.stencil
        self.ops = (self.Ax, self.Az, self.AbsAx, self.AbsAz, self.Ay, self.AbsAy)
        self.Ls = (st.L2x, st.L2y, st.L1x, st.L1y, st.L2z, st.L1z)
        self.qReduced = None
        self.MReduced = None
        self.OReduced = None
        self.idxBeam = None

    # -- boundary source --------------------------------------------------
    def _angular(self, Om):
        s = self.settings
        Om = np.atleast_2d(Om)
        return (np.exp(-s.sigmaO1Inv * (s.Omega1 - Om[:, 0]) ** 2) * np.exp(-s.sigmaO2Inv * (s.Omega2 - Om[:, 1]) ** 2)
                * np.exp(-s.sigmaO3Inv * (s.Omega3 - Om[:, 2]) ** 2))

    def spatial_profile(self, x0=None, y0=None, z0=None):
        """PsiBeam's spatial factor at every cell (row order), beam centred at (x0, y0, z0)."""
        s = self.settings
        x0 = s.x0 if x0 is None else x0
        y0 = s.y0 if y0 is None else y0
        z0 = s.z0 if z0 is None else z0
        zm = s.zMid[:, None, None]
        xm = s.xMid[None, :, None]
        ym = s.yMid[None, None, :]
        prof = np.exp(-s.sigmaXInv * (xm - x0) ** 2) * np.exp(-s.sigmaYInv * (ym - y0) ** 2) * \
            np.exp(-s.sigmaZInv * (zm - z0) ** 2)
        return np.broadcast_to(prof, (s.NCellsZ, s.NCellsX, s.NCellsY)).reshape(self.n_cells)

    def inflow_factor(self, E, n):
        """PsiBeam without the spatial factor, per reduced ordinate (csd.S[n-1])."""
        s = self.settings
        return (self.psi_scale * self._angular(self.qReduced) * math.exp(-s.sigmaEInv * (s.eMax - E) ** 2)
                * self.csd.S[n - 1] * s.densityMin)

    def setup_directions(self):
        """Direction reduction (``SolverCSD.jl:910-925``): ordinates whose
        PsiBeam at (eMax, x0, y0, z0) exceeds 1e-17 of the largest."""
        s = self.settings
        pts = self.Q_points
        beam = self.psi_scale * self._angular(pts) * self.csd.S[0] * s.densityMin
        idx = np.nonzero(beam > 1e-17 * beam.max())[0]
        self.idxBeam = idx
        self.qReduced = pts[idx, :]
        self.MReduced = self.M[:, idx]
        self.OReduced = self.O[idx, :]
        return np.zeros((s.NCellsZ, s.NCellsX, s.NCellsY, idx.size))

    def apply_bc(self, psi, E, n):
        """Inflow on every face cell for all reduced ordinates (``:977-988`` in 3D)."""
        prof = self.spatial_profile().reshape(self.face.shape)
        psi[self.face, :] = prof[self.face][:, None] * self.inflow_factor(E, n)[None, :]

    def flux_upwind(self, phi):
        """``solveFluxUpwind!`` with the z term, interior cells only."""
        s = self.settings
        flux = np.zeros_like(phi)
        ox, oy, oz = self.qReduced[:, 0], self.qReduced[:, 1], self.qReduced[:, 2]
        c = phi[1:-1, 1:-1, 1:-1, :]
        ew = np.where(ox >= 0.0, c - phi[1:-1, :-2, 1:-1, :], phi[1:-1, 2:, 1:-1, :] - c)
        ns = np.where(oz >= 0.0, c - phi[1:-1, 1:-1, :-2, :], phi[1:-1, 1:-1, 2:, :] - c)
        tb = np.where(oy >= 0.0, c - phi[:-2, 1:-1, 1:-1, :], phi[2:, 1:-1, 1:-1, :] - c)
        flux[1:-1, 1:-1, 1:-1, :] = (ox / s.dx) * ew + (oz / s.dy) * ns + (oy / s.dz) * tb
        return flux

    def sweep(self, psi, dE, sigma0):
        """Uncollided update with the boundary-slab quirk in every z layer."""
        flux = self.flux_upwind(psi / self.density[..., None])
        a, b = self.restore_ab
        psiBC = psi[:, a, b, 0].copy()
        psi[...] = (psi - dE * flux) / (1 + dE * sigma0)
        psi[:, a, b, 0] = psiBC

    # -- streaming products over the six (stencil, P_N) pairs -------------
    def _w_grams(self, Wa, Wb):
        return tuple(Wa.T @ (A @ Wb) for A in self.ops)

    def _x_grams(self, Xa, Xb):
        return tuple(Xa.T @ (Lm @ Xb) for Lm in self.Ls)

    def _k_stream(self, K, *C):
        dE = C[-1]
        acc = (self.Ls[0] @ K) @ C[0]
        for d in range(1, 6):
            acc = acc + (self.Ls[d] @ K) @ C[d]
        return K - dE * acc

    def _l_stream(self, L, *G):
        dE = G[-1]
        acc = (self.ops[0] @ L) @ G[0].T
        for d in range(1, 6):
            acc = acc + (self.ops[d] @ L) @ G[d].T
        return L - dE * acc

    def _op_sum(self, G, S, C):
        acc = G[0] @ S @ C[0]
        for d in range(1, 6):
            acc = acc + G[d] @ S @ C[d]
        return acc

    def _s_stream(self, S, G, C, dE, sign=-1.0):
        return S + sign * dE * self._op_sum(G, S, C)


def solve_pn_full_3d(solver: SolverCSD3D, max_steps: int | None = None):
    """``SolveFirstCollisionSource`` (``SolverCSD.jl:465-586``) on the 3D grid:
    the loop of ``oracle.full_rank.solve_pn_full`` with the six streaming pairs.
    Returns (1/2 sqrt(gamma_0) u, dose, psi)."""
    from .full_rank import sigma_vectors

    s = solver.settings
    eTrafo = solver.csd.eTrafo
    energy = solver.csd.eGrid
    n_cells = solver.n_cells
    psi = solver.setup_directions()
    Mr = solver.MReduced
    nE = eTrafo.size
    u = np.zeros((n_cells, solver.N))
    bnd = solver.boundaryIdx
    inner = ~solver.face.ravel()
    last = nE if max_steps is None else min(nE, 1 + max_steps)
    for n in range(2, last + 1):
        sig, Dvec, D = sigma_vectors(solver, n)
        dE = eTrafo[n - 1] - eTrafo[n - 2]
        solver.apply_bc(psi, energy[n - 1], n - 1)
        flux = solver.flux_upwind(psi)
        psi = psi - dE * flux
        psi_new = psi / (1.0 + dE * sig[0])
        uT = u.copy()
        for A, Lm in zip(solver.ops, solver.Ls):
            uT = uT - dE * (Lm @ np.asarray((A.T @ u.T).T))
        uT[bnd, :] = 0.0
        pv = psi_new.reshape(n_cells, -1)
        u_new = np.zeros_like(u)
        src = pv[inner] @ Mr.T
        u_new[inner] = (uT[inner] + dE * Dvec[None, :] * src) / (1.0 + dE * D)[None, :]
        u_unc = np.zeros(n_cells)
        u_unc[inner] = pv[inner] @ Mr[0, :]
        solver.dose += dE * (u_new[:, 0] + u_unc) * solver.csd.SMid[n - 2] / solver.densityVec / (
            1 + (n == 2 or n == nE))
        u = u_new
        psi = psi_new
    return 0.5 * math.sqrt(solver.gamma[0]) * u, solver.dose, psi
