"""``SolverCSD`` and the ``Solve*`` entry points, running on the B200 through libtitus.

Mirrors the reference API (``code/SolverCSD.jl``):

* ``SolverCSD(settings)`` -- builds the solver data (``:63-146``) on the host
  and uploads it to the device once (``titus_create``);
* ``SolveFirstCollisionSourceDLR(solver)`` -- fixed-rank integrator
  (``:891-1120``), returns ``(X U, 1/2 sqrt(gamma_0) Sigma, O W V, W V, dose, psi)``;
* ``SolveFirstCollisionSourceDLRParallel(solver)`` -- rank-adaptive parallel
  integrator (``:1726-2008``), the same tuple with ``rVec`` before ``psi``;
* ``SolveFirstCollisionSourceDLRBUGRejection(solver)`` -- rank-adaptive BUG
  integrator with step rejection (``:2011-2374``), returns ``(X U, Sigma, O W V,
  W V, dose, [E rank]^T, [E eta], [E bound], psi)``.

The energy loop itself always runs on the GPU; there is no CPU path.
"""
from __future__ import annotations

import copy
import ctypes as C
import math

import numpy as np

from . import _lib
from . import physics as ph


class SolverCSD:
    def __init__(self, settings, team_ctas: int = 0, precision: int = _lib.TITUS_PRECISION_FP64):
        s = settings
        self.settings = s
        self.team_ctas = team_ctas
        # TITUS_PRECISION_FP64 or TITUS_PRECISION_MIXED (tensor-core operator
        # Grams of the adaptive integrators; see include/titus.h)
        self.precision = precision
        nx, ny = s.NCellsX, s.NCellsY
        self.n = nx * ny
        npn = s.nPN
        self.N = (npn + 1) ** 2
        self.gamma = np.array([2.0 / (2 * l + 1) for l in range(npn + 1)])
        Ax, Az = ph.flux_matrices(npn)
        self.ops = [ph.to_csr(A) for A in (Ax, Az, ph.roe(Ax), ph.roe(Az))]
        q = npn + 1
        self.Q_points, self.Q_weights, self.O, self.M = ph.quadrature(q, npn)
        self.eGrid, self.eTrafo, self.S, self.SMid = ph.energy_grid(s, with_mid=True)
        self.nE = self.eTrafo.size
        # separable PsiBeam (SolverCSD.jl:275): angular x spatial x energy factors
        ang = np.exp(-s.sigmaO1Inv * (s.Omega1 - self.Q_points[:, 0]) ** 2) * \
            np.exp(-s.sigmaO3Inv * (s.Omega3 - self.Q_points[:, 2]) ** 2)
        scale = s.psi_scale / ang.max() if s.beam_peak_normalized else s.psi_scale
        # direction reduction, SolverCSD.jl:912-925 (PsiBeam at eMax, x0, y0, n=1)
        e0 = scale * math.exp(-s.sigmaEInv * (s.eMax - s.eMax) ** 2) * self.S[0] * s.densityMin
        beam = ang * e0 * math.exp(-s.sigmaXInv * (s.x0 - s.x0) ** 2) * math.exp(-s.sigmaYInv * (s.y0 - s.y0) ** 2)
        self.idxBeam = np.nonzero(beam > 1e-17 * beam.max())[0]
        self.qReduced = self.Q_points[self.idxBeam]
        self.MReduced = np.ascontiguousarray(self.M[:, self.idxBeam])
        self.OReduced = self.O[self.idxBeam]
        self.q = self.idxBeam.size
        self.bc_angle = np.ascontiguousarray(ang[self.idxBeam])
        self.bc_energy = scale * np.exp(-s.sigmaEInv * (s.eMax - self.eGrid) ** 2) * self.S * s.densityMin
        xm = s.xMid[np.arange(self.n) // ny]
        ym = s.yMid[np.arange(self.n) % ny]
        self.bc_space = np.exp(-s.sigmaXInv * (xm - s.x0) ** 2) * np.exp(-s.sigmaYInv * (ym - s.y0) ** 2)
        sig = np.array([s.sigmaT_hg * s.hg_g**l for l in range(npn + 1)])
        self.sigma = np.ascontiguousarray(np.tile(sig, (self.nE, 1)))
        self.density = np.ascontiguousarray(s.density.reshape(self.n), dtype=np.float64)
        # boundary cells in the reference's order (SolverCSD.jl:108-131)
        bidx = []
        for i in range(nx):
            bidx += [i * ny, i * ny + ny - 1]
        for j in range(ny):
            bidx += [j, (nx - 1) * ny + j]
        self.boundaryIdx = np.array(bidx, dtype=np.int64)
        # psi[boundaryIdx] linear-indexes the column-major (nx, ny, q) array:
        # ordinate-0 value of cell (L % nx, L // nx) survives the sweep
        Lb = self.boundaryIdx
        self.sweep_restore = np.unique((Lb % nx) * ny + Lb // nx).astype(np.int32)
        # completion candidates for rank-deficient bases: canonical vectors in
        # index order (LAPACK's identity columns for a zero input); spatial
        # candidates are boundary cells, whose rows are zero in every K
        self.x_completion = np.unique(self.boundaryIdx).astype(np.int32)
        self.w_completion = np.arange(self.N, dtype=np.int32)
        self.dose = np.zeros(self.n)
        self._handle = None
        self._keep = None

    @property
    def psi_shape(self):
        s = self.settings
        return (s.NCellsX, s.NCellsY, self.q)

    def beam_tables(self, energy: float, y0: float):
        """Energy grid and PsiBeam tables of a pencil beam entering at (x0, y0)
        with energy ``energy`` on this solver's phantom (``CSD.jl:47-89``,
        ``SolverCSD.jl:240-276``): (nE, dE, stopping, bc_energy, sigma, bc_space)."""
        s2 = copy.copy(self.settings)
        s2.eMax = float(energy)
        s2.y0 = float(y0)
        eGrid, eTrafo, S = ph.energy_grid(s2)
        ang = np.exp(-s2.sigmaO1Inv * (s2.Omega1 - self.Q_points[:, 0]) ** 2) * \
            np.exp(-s2.sigmaO3Inv * (s2.Omega3 - self.Q_points[:, 2]) ** 2)
        scale = s2.psi_scale / ang.max() if s2.beam_peak_normalized else s2.psi_scale
        bc_energy = scale * np.exp(-s2.sigmaEInv * (s2.eMax - eGrid) ** 2) * S * s2.densityMin
        ny = s2.NCellsY
        xm = s2.xMid[np.arange(self.n) // ny]
        ym = s2.yMid[np.arange(self.n) % ny]
        bc_space = np.exp(-s2.sigmaXInv * (xm - s2.x0) ** 2) * np.exp(-s2.sigmaYInv * (ym - s2.y0) ** 2)
        sig = np.array([s2.sigmaT_hg * s2.hg_g**l for l in range(s2.nPN + 1)])
        sigma = np.ascontiguousarray(np.tile(sig, (eTrafo.size, 1)))
        return (eTrafo.size, float(eTrafo[1] - eTrafo[0]), np.ascontiguousarray(S), np.ascontiguousarray(bc_energy),
                sigma, np.ascontiguousarray(bc_space))

    def spot_array(self, spots):
        """titus_spot_t array (and the host tables it points to) for [(energy, y0), ...]."""
        ns = len(spots)
        arr = (_lib.Spot * ns)()
        keep = []
        for i, (e, y) in enumerate(spots):
            nE, dE, S, bce, sig, bcs = self.beam_tables(e, y)
            keep += [S, bce, sig, bcs]
            arr[i].n_energies = nE
            arr[i].d_e = dE
            arr[i].stopping = _lib.as_dp(S)
            arr[i].bc_energy = _lib.as_dp(bce)
            arr[i].sigma = _lib.as_dp(sig)
            arr[i].bc_space = _lib.as_dp(bcs)
        return arr, keep

    def batch(self, spots):
        """Upload pencil beams once for repeated batched solves (PencilBeamBatch)."""
        return PencilBeamBatch(self, spots)

    def solve_batched(self, spots, method: int = _lib.TITUS_BUG_ADAPTIVE, team_ctas: int = 1, max_steps: int = 0):
        """All pencil beams ``spots`` = [(energy, y0), ...] in one persistent
        launch (titus_solve_batched). Returns (dose (nspots x n), rank, iterations)."""
        lib = _lib.load()
        h = self.handle()
        ns = len(spots)
        arr, keep = self.spot_array(spots)
        dose = np.zeros((ns, self.n))
        rank = np.zeros(ns, dtype=np.int32)
        iters = np.zeros(ns, dtype=np.int32)
        opt = self.options(max_steps)
        opt.team_ctas = team_ctas
        _lib.check(lib.titus_solve_batched(h, method, C.byref(opt), ns, arr, _lib.as_dp(dose), _lib.as_ip(rank),
                                           _lib.as_ip(iters)), "titus_solve_batched")
        return dose, rank, iters

    # -------------------------------------------------------------- device
    def problem_struct(self):
        s = self.settings
        p = _lib.Problem()
        keep = []

        def dp(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return _lib.as_dp(a)

        def ip(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            keep.append(a)
            return _lib.as_ip(a)

        p.nx, p.ny, p.npn, p.n_moments = s.NCellsX, s.NCellsY, s.nPN, self.N
        p.n_ordinates, p.n_energies, p.r = self.q, self.nE, s.r
        p.dx, p.dy = s.dx, s.dy
        p.theta, p.theta_index, p.c_eta = s.theta, s.thetaIndex, s.c_eta
        p.density = dp(self.density)
        p.e_trafo = dp(self.eTrafo)
        p.stopping = dp(self.S)
        p.bc_energy = dp(self.bc_energy)
        p.sigma = dp(self.sigma)
        p.bc_space = dp(self.bc_space)
        p.bc_angle = dp(self.bc_angle)
        p.omega = dp(self.qReduced)
        p.m_reduced = dp(self.MReduced)
        for d, (rp, ci, v) in enumerate(self.ops):
            p.op_rowptr[d] = ip(rp)
            p.op_col[d] = ip(ci)
            p.op_val[d] = dp(v)
        p.x_completion = ip(self.x_completion)
        p.n_x_completion = self.x_completion.size
        p.w_completion = ip(self.w_completion)
        p.n_w_completion = self.w_completion.size
        p.sweep_restore = ip(self.sweep_restore)
        p.n_sweep_restore = self.sweep_restore.size
        p.stopping_mid = dp(self.SMid)
        return p, keep

    def handle(self):
        if self._handle is None:
            lib = _lib.load()
            p, keep = self.problem_struct()
            h = C.c_void_p()
            _lib.check(lib.titus_create(C.byref(p), C.byref(h)), "titus_create")
            self._handle = h
        return self._handle

    def close(self):
        if self._handle is not None:
            _lib.load().titus_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_beam_profile(self, profile):
        """Replace PsiBeam's spatial factor (read on the boundary cells) by
        ``profile`` (n cells, row i*ny + j), e.g. a weighted sum of spot
        profiles; the device handle is rebuilt on next use."""
        profile = np.ascontiguousarray(profile, dtype=np.float64).reshape(self.n)
        if not np.all(np.isfinite(profile)):
            raise ValueError("beam profile must be finite")
        self.bc_space = profile
        self.close()

    def beam_profile(self, x0=None, y0=None):
        """PsiBeam's spatial factor at every cell for a beam centred at (x0, y0)
        (defaults: the settings' beam)."""
        s = self.settings
        x0 = s.x0 if x0 is None else x0
        y0 = s.y0 if y0 is None else y0
        xm = s.xMid[np.arange(self.n) // s.NCellsY]
        ym = s.yMid[np.arange(self.n) % s.NCellsY]
        return np.exp(-s.sigmaXInv * (xm - x0) ** 2) * np.exp(-s.sigmaYInv * (ym - y0) ** 2)

    def options(self, max_steps=0, rank_tol=0.0, profile=False):
        o = _lib.Options()
        o.team_ctas = self.team_ctas
        o.max_steps = max_steps
        o.rank_tol = rank_tol
        o.profile = 1 if profile else 0
        o.precision = self.precision
        return o

    def profile(self):
        """Per-phase device timers (ns) of the last solve run with profile=True."""
        lib = _lib.load()
        out = np.zeros(32)
        m = lib.titus_profile(self.handle(), _lib.as_dp(out), 32)
        nt = len(_lib.PROFILE_NAMES)
        d = {name: out[i] for i, name in enumerate(_lib.PROFILE_NAMES[:min(m, nt)])}
        d["total"] = float(sum(d.values()))
        for i, name in enumerate(_lib.PROFILE_COUNTERS):
            if m > nt + i:
                d[name] = out[nt + i]
        return d

    def _result(self, r_cap):
        res = _lib.Result()
        bufs = dict(
            dose=np.zeros(self.n), X=np.zeros((self.n, r_cap)), S=np.zeros((r_cap, r_cap)),
            W=np.zeros((self.N, r_cap)), psi=np.zeros((self.n, self.q)),
            rank_history=np.zeros(self.nE, dtype=np.int32), time_history=np.zeros(self.nE),
            eta_history=np.zeros(self.nE), bound_history=np.zeros(self.nE),
        )
        res.dose = _lib.as_dp(bufs["dose"])
        res.X = _lib.as_dp(bufs["X"])
        res.S = _lib.as_dp(bufs["S"])
        res.W = _lib.as_dp(bufs["W"])
        res.psi = _lib.as_dp(bufs["psi"])
        res.rank_history = _lib.as_ip(bufs["rank_history"])
        res.time_history = _lib.as_dp(bufs["time_history"])
        res.eta_history = _lib.as_dp(bufs["eta_history"])
        res.bound_history = _lib.as_dp(bufs["bound_history"])
        res.r_cap = r_cap
        return res, bufs

    def run(self, method: int, max_steps: int = 0, rank_tol: float = 0.0, profile: bool = False):
        """Run one integrator on the device; returns raw factors and histories."""
        lib = _lib.load()
        h = self.handle()
        r_cap = max(self.settings.r, 1)
        res, bufs = self._result(r_cap)
        opt = self.options(max_steps, rank_tol, profile)
        _lib.check(lib.titus_solve(h, method, C.byref(opt), C.byref(res)), "titus_solve")
        k = res.rank
        n_next, t = self.resume_point()
        return dict(X=bufs["X"][:, :k], S=bufs["S"][:k, :k], W=bufs["W"][:, :k], dose=bufs["dose"],
                    psi=bufs["psi"], rank=k, steps=res.steps_done, rank_history=bufs["rank_history"],
                    time_history=bufs["time_history"], eta_history=bufs["eta_history"],
                    bound_history=bufs["bound_history"], n_next=n_next, t=t)

    def resume_point(self):
        """(n_next, t): the energy index the loop would process next and the
        pseudo-time after the last solve (titus_resume_point)."""
        nn = np.zeros(1, dtype=np.int32)
        t = np.zeros(1)
        _lib.check(_lib.load().titus_resume_point(self.handle(), _lib.as_ip(nn), _lib.as_dp(t)),
                   "titus_resume_point")
        return int(nn[0]), float(t[0])

    def run_from(self, method: int, state: dict, n_next: int, n_stop: int, rank_tol: float = 0.0, max_steps: int = 0):
        """Resume the loop from a given state (checkpoint restart)."""
        lib = _lib.load()
        h = self.handle()
        X = np.ascontiguousarray(state["X"], dtype=np.float64)
        S = np.ascontiguousarray(state["S"], dtype=np.float64)
        W = np.ascontiguousarray(state["W"], dtype=np.float64)
        psi = np.ascontiguousarray(state["psi"], dtype=np.float64).reshape(self.n, self.q)
        dose = np.ascontiguousarray(state["dose"], dtype=np.float64)
        k = S.shape[0]
        _lib.check(lib.titus_set_state(h, k, _lib.as_dp(X), _lib.as_dp(S), _lib.as_dp(W), _lib.as_dp(psi),
                                       _lib.as_dp(dose), n_next), "titus_set_state")
        r_cap = max(self.settings.r, k)
        res, bufs = self._result(r_cap)
        opt = self.options(max_steps, rank_tol)
        _lib.check(lib.titus_solve_from(h, method, C.byref(opt), n_stop, C.byref(res)), "titus_solve_from")
        kk = res.rank
        n_next, t = self.resume_point()
        return dict(X=bufs["X"][:, :kk], S=bufs["S"][:kk, :kk], W=bufs["W"][:, :kk], dose=bufs["dose"],
                    psi=bufs["psi"], rank=kk, steps=res.steps_done, rank_history=bufs["rank_history"],
                    time_history=bufs["time_history"], eta_history=bufs["eta_history"],
                    bound_history=bufs["bound_history"], n_next=n_next, t=t)

    def outputs(self, out):
        """The reference's return tuple from raw factors (``SolverCSD.jl:1116-1118``)."""
        U, sig, Vt = np.linalg.svd(out["S"])
        V = Vt.T
        X, W = out["X"], out["W"]
        psi = out["psi"].reshape(self.psi_shape)
        return X @ U, 0.5 * math.sqrt(self.gamma[0]) * sig, self.O @ (W @ V), W @ V, out["dose"], psi


class PencilBeamBatch:
    """Pencil beams whose tables live on the device (titus_batch_upload), so
    repeated batched solves move no host data: ``solve_device(stream)``
    launches, ``fetch()`` waits and returns (dose (nspots x n), final rank,
    iterations); ``rank_sums()`` gives the per-spot sum of the ranks entering
    the iterations of the last fetched solve."""

    def __init__(self, solver: SolverCSD, spots):
        self.solver = solver
        self.nspots = len(spots)
        arr, keep = solver.spot_array(spots)
        self.n_energies = np.array([arr[i].n_energies for i in range(self.nspots)], dtype=np.int64)
        h = C.c_void_p()
        _lib.check(_lib.load().titus_batch_upload(solver.handle(), self.nspots, arr, C.byref(h)), "titus_batch_upload")
        self._h = h

    def solve_device(self, method: int = _lib.TITUS_BUG_ADAPTIVE, team_ctas: int = 1, max_steps: int = 0,
                     stream: int = 0):
        opt = self.solver.options(max_steps)
        opt.team_ctas = team_ctas
        _lib.check(_lib.load().titus_batch_solve_device(self._h, method, C.byref(opt), C.c_void_p(stream)),
                   "titus_batch_solve_device")

    def fetch(self, want_dose: bool = True):
        n = self.solver.n
        dose = np.zeros((self.nspots, n)) if want_dose else None
        rank = np.zeros(self.nspots, dtype=np.int32)
        iters = np.zeros(self.nspots, dtype=np.int32)
        _lib.check(_lib.load().titus_batch_fetch(self._h, _lib.as_dp(dose) if want_dose else None, _lib.as_ip(rank),
                                                  _lib.as_ip(iters)), "titus_batch_fetch")
        return dose, rank, iters

    def rank_sums(self):
        out = np.zeros(self.nspots, dtype=np.int32)
        _lib.check(_lib.load().titus_batch_rank_sums(self._h, _lib.as_ip(out)), "titus_batch_rank_sums")
        return out

    def close(self):
        if self._h is not None:
            _lib.load().titus_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolverCSD3D(SolverCSD):
    """Solver data of a 3D problem (``Settings3D``; no counterpart in the
    reference, which is 2D), uploaded with ``titus_create_3d``.

    Cell (i, j, k) has row ``(k*nx + i)*ny + j``; the boundary cells are those
    on any face. The z direction streams with the P_N matrix Ay and |Ay| (the
    x / y pairs are the reference's), the sweep's z term uses Omega_y, and
    PsiBeam gains the factors exp(-sigmaO2Inv (Omega2 - Omega_y)^2) and
    exp(-sigmaZInv (z - z0)^2), applied on every face cell. The sweep's
    boundary-slab quirk (``SolverCSD.jl:1002,1005``) is applied in every z
    layer. A 3D handle runs the full-rank P_N solver
    (``SolveFirstCollisionSource``) and the rank-adaptive BUG integrator
    (``SolveFirstCollisionSourceDLRBUGRejection``, plain and resumed with
    ``run_from``); the other DLR integrators raise.
    """

    def __init__(self, settings, team_ctas: int = 0, precision: int = _lib.TITUS_PRECISION_FP64):
        s = settings
        self.settings = s
        self.team_ctas = team_ctas
        self.precision = precision
        nz, nx, ny = s.NCellsZ, s.NCellsX, s.NCellsY
        self.n = nz * nx * ny
        npn = s.nPN
        self.N = (npn + 1) ** 2
        self.gamma = np.array([2.0 / (2 * l + 1) for l in range(npn + 1)])
        Ax, Az = ph.flux_matrices(npn)
        Ay = ph.flux_matrix_y(npn)
        self.ops = [ph.to_csr(A) for A in (Ax, Az, ph.roe(Ax), ph.roe(Az))]
        self.ops3 = [ph.to_csr(A) for A in (Ay, ph.roe(Ay))]
        q = npn + 1
        self.Q_points, self.Q_weights, self.O, self.M = ph.quadrature(q, npn)
        self.eGrid, self.eTrafo, self.S, self.SMid = ph.energy_grid(s, with_mid=True)
        self.nE = self.eTrafo.size
        P = self.Q_points
        ang = np.exp(-s.sigmaO1Inv * (s.Omega1 - P[:, 0]) ** 2) * np.exp(-s.sigmaO2Inv * (s.Omega2 - P[:, 1]) ** 2) * \
            np.exp(-s.sigmaO3Inv * (s.Omega3 - P[:, 2]) ** 2)
        scale = s.psi_scale / ang.max() if s.beam_peak_normalized else s.psi_scale
        # direction reduction (SolverCSD.jl:912-925): PsiBeam at eMax on the beam axis
        beam = scale * ang * self.S[0] * s.densityMin
        self.idxBeam = np.nonzero(beam > 1e-17 * beam.max())[0]
        self.qReduced = self.Q_points[self.idxBeam]
        self.MReduced = np.ascontiguousarray(self.M[:, self.idxBeam])
        self.OReduced = self.O[self.idxBeam]
        self.q = self.idxBeam.size
        self.bc_angle = np.ascontiguousarray(ang[self.idxBeam])
        self.bc_energy = scale * np.exp(-s.sigmaEInv * (s.eMax - self.eGrid) ** 2) * self.S * s.densityMin
        self.bc_space = self.beam_profile()
        sig = np.array([s.sigmaT_hg * s.hg_g**l for l in range(npn + 1)])
        self.sigma = np.ascontiguousarray(np.tile(sig, (self.nE, 1)))
        self.density = np.ascontiguousarray(np.asarray(s.density, dtype=np.float64).reshape(self.n))
        face = np.zeros((nz, nx, ny), dtype=bool)
        face[0], face[-1], face[:, 0], face[:, -1], face[:, :, 0], face[:, :, -1] = (True,) * 6
        self.boundaryIdx = np.nonzero(face.ravel())[0]
        # the 2D restore positions (L % nx, L // nx) of the reference's boundary order, per z layer
        bidx = []
        for i in range(nx):
            bidx += [i * ny, i * ny + ny - 1]
        for j in range(ny):
            bidx += [j, (nx - 1) * ny + j]
        Lb = np.array(bidx, dtype=np.int64)
        layer = np.unique((Lb % nx) * ny + Lb // nx)
        self.sweep_restore = (np.arange(nz)[:, None] * (nx * ny) + layer[None, :]).ravel().astype(np.int32)
        self.x_completion = self.boundaryIdx.astype(np.int32)
        self.w_completion = np.arange(self.N, dtype=np.int32)
        self.dose = np.zeros(self.n)
        self._handle = None
        self._keep = None

    @property
    def psi_shape(self):
        s = self.settings
        return (s.NCellsZ, s.NCellsX, s.NCellsY, self.q)

    def beam_profile(self, x0=None, y0=None, z0=None):
        """PsiBeam's spatial factor at every cell for a beam centred at (x0, y0, z0)."""
        s = self.settings
        x0 = s.x0 if x0 is None else x0
        y0 = s.y0 if y0 is None else y0
        z0 = s.z0 if z0 is None else z0
        prof = np.exp(-s.sigmaXInv * (s.xMid[None, :, None] - x0) ** 2) * \
            np.exp(-s.sigmaYInv * (s.yMid[None, None, :] - y0) ** 2) * \
            np.exp(-s.sigmaZInv * (s.zMid[:, None, None] - z0) ** 2)
        return np.ascontiguousarray(np.broadcast_to(prof, (s.NCellsZ, s.NCellsX, s.NCellsY)).reshape(self.n))

    def handle(self):
        if self._handle is None:
            lib = _lib.load()
            p, keep = self.problem_struct()
            e = _lib.Problem3D()
            e.nz, e.dz = self.settings.NCellsZ, self.settings.dz
            for d, (rp, ci, v) in enumerate(self.ops3):
                keep += [rp, ci, v]
                e.op_rowptr[d] = _lib.as_ip(rp)
                e.op_col[d] = _lib.as_ip(ci)
                e.op_val[d] = _lib.as_dp(v)
            h = C.c_void_p()
            _lib.check(lib.titus_create_3d(C.byref(p), C.byref(e), C.byref(h)), "titus_create_3d")
            self._handle = h
        return self._handle


def SolveFirstCollisionSource(solver: SolverCSD, max_steps: int = 0):
    """Full-rank P_N first-collision solver (``SolverCSD.jl:465-586``) on the GPU.

    Returns ``(1/2 sqrt(gamma_0) u, dose, psi)`` with u (n x N, row i*ny + j)
    and psi (nx, ny, q) like the reference.
    """
    lib = _lib.load()
    h = solver.handle()
    u = np.zeros((solver.n, solver.N))
    dose = np.zeros(solver.n)
    psi = np.zeros((solver.n, solver.q))
    opt = solver.options(max_steps)
    _lib.check(lib.titus_pn_full_solve(h, C.byref(opt), _lib.as_dp(u), _lib.as_dp(dose), _lib.as_dp(psi)),
               "titus_pn_full_solve")
    solver.dose = dose
    return 0.5 * math.sqrt(solver.gamma[0]) * u, dose, psi.reshape(solver.psi_shape)


def DoseAdjoint(solver: SolverCSD, weight=None, target=None, dj_ddose=None, checkpoint_every: int = 0,
                max_steps: int = 0):
    """Dose objective of the full-rank sweep and its gradients, by the
    discrete adjoint on the GPU (``titus_dose_adjoint``, method TITUS_PN_FULL).

    J = sum_c weight[c] (dose[c] - target[c])^2 (weight None = 1, target None =
    0), or any J given through ``dj_ddose``. Returns ``(J, dose, dJ/drho,
    dJ/dprofile)``; for a plan set with ``solver.set_beam_profile(sum_s w_s
    p_s)`` the spot-weight gradient is ``p_s @ dJ/dprofile``. The (u, psi)
    state is checkpointed every ``checkpoint_every`` energy steps (0 = about
    sqrt(steps)) and recomputed between checkpoints.
    """
    lib = _lib.load()
    h = solver.handle()
    n = solver.n

    def arr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(n)
        return a

    w, t, g = arr(weight), arr(target), arr(dj_ddose)
    dose = np.zeros(n)
    gr = np.zeros(n)
    gp = np.zeros(n)
    J = C.c_double(0.0)
    opt = solver.options(max_steps)
    nul = C.POINTER(C.c_double)()
    _lib.check(lib.titus_dose_adjoint(h, _lib.TITUS_PN_FULL, C.byref(opt), nul if w is None else _lib.as_dp(w),
                                      nul if t is None else _lib.as_dp(t), nul if g is None else _lib.as_dp(g),
                                      int(checkpoint_every), C.byref(J), _lib.as_dp(dose), _lib.as_dp(gr),
                                      _lib.as_dp(gp)), "titus_dose_adjoint")
    return J.value, dose, gr, gp


def SolveFirstCollisionSourceDLR(solver: SolverCSD, max_steps: int = 0):
    """Fixed-rank DLR (``SolverCSD.jl:891-1120``) on the GPU."""
    out = solver.run(_lib.TITUS_DLR_FIXED, max_steps=max_steps)
    res = solver.outputs(out)
    solver.dose = res[4]
    return res


def SolveFirstCollisionSourceDLRHighOrder(solver: SolverCSD, max_steps: int = 0):
    """Fixed-rank DLR with RK4 streaming (``SolverCSD.jl:588-889``) on the GPU:
    inflow on the two outer layers, the second-order limited sweep
    (``solveFlux!``) and RK4 K/L/S streaming with the central operators. Same
    return tuple as ``SolveFirstCollisionSourceDLR``."""
    out = solver.run(_lib.TITUS_DLR_HIGH_ORDER, max_steps=max_steps)
    res = solver.outputs(out)
    solver.dose = res[4]
    return res


def SolveFirstCollisionSourceDLRParallel(solver: SolverCSD, recordGif: bool = False, max_steps: int = 0):
    """Rank-adaptive parallel integrator (``SolverCSD.jl:1726-2008``) on the GPU.

    Returns ``(X U, 1/2 sqrt(gamma_0) Sigma, O W V, W V, dose, rVec, psi)`` with
    rVec (2 x nEnergies): row 0 the pseudo-time t at which each step started,
    row 1 the rank after the step (``:1947-1948``); entries of steps not run
    keep the initial rank as in the reference.
    """
    out = solver.run(_lib.TITUS_PARALLEL_ADAPTIVE, max_steps=max_steps)
    res = solver.outputs(out)
    solver.dose = res[4]
    r0 = solver.settings.r // 2
    rVec = float(r0) * np.ones((2, solver.nE))
    hist = out["rank_history"]
    done = hist >= 0
    rVec[1, done] = hist[done]
    rVec[0, 1:][done[1:]] = out["time_history"][1:][done[1:]]
    return res[0], res[1], res[2], res[3], res[4], rVec, res[5]


def SolveFirstCollisionSourceDLRBUGRejection(solver: SolverCSD, recordGif: bool = False, max_steps: int = 0):
    """Rank-adaptive BUG integrator with step rejection (``SolverCSD.jl:2011-2374``).

    Returns ``(X U, 1/2 sqrt(gamma_0) Sigma, O W V, W V, dose, [E rank]^T,
    [E eta], [E bound], psi)``: one (energy, rank) column per loop iteration
    (repeated energies included) and one (energy, eta) / (energy, bound) row per
    streaming rejection test. The device records at most nEnergies iterations.
    """
    return _rejection_outputs(solver, _lib.TITUS_BUG_ADAPTIVE, max_steps)


def SolveFirstCollisionSourceDLRParallelRejection(solver: SolverCSD, recordGif: bool = False, max_steps: int = 0):
    """Parallel integrator with step rejection (``SolverCSD.jl:2376-2742``).

    The parallel integrator's augmented step (``S_new = [[Sbar, L^T W~],
    [X~^T K, 0]]``, then ``truncate!``) inside the BUG loop's rejection tests.
    Same return tuple as :func:`SolveFirstCollisionSourceDLRBUGRejection`.
    Where the reference's next step raises a DimensionMismatch (a scattering
    rejection after a streaming step that changed the rank) the solve raises
    ``TitusError`` (``TITUS_ERR_DEVICE``).
    """
    return _rejection_outputs(solver, _lib.TITUS_PARALLEL_REJECTION, max_steps)


def _rejection_outputs(solver: SolverCSD, method: int, max_steps: int):
    out = solver.run(method, max_steps=max_steps)
    res = solver.outputs(out)
    solver.dose = res[4]
    it = min(out["steps"], solver.nE)
    nidx = out["time_history"][:it].astype(int)
    energies = solver.eGrid[nidx - 1]
    rank_hist = np.array([energies, out["rank_history"][:it].astype(float)])
    ne = int(np.count_nonzero(out["bound_history"]))
    eta = out["eta_history"][:ne]
    bound = out["bound_history"][:ne]
    # the reference pairs each eta with eGrid[n-1] of its iteration; the device
    # keeps the values only, so the energies are left as NaN here
    eta_hist = np.column_stack([np.full(ne, np.nan), eta])
    bound_hist = np.column_stack([np.full(ne, np.nan), bound])
    return res[0], res[1], res[2], res[3], res[4], rank_hist, eta_hist, bound_hist, res[5]


def SolveBatchedPencilBeams(solver: SolverCSD, spots, method: str = "bug", team_ctas: int = 1,
                            max_steps: int = 0):
    """Many pencil beams (energy, entry y0) on one phantom in one persistent
    launch; returns (dose per spot (nspots x n), final rank, loop iterations)."""
    mid = {"bug": _lib.TITUS_BUG_ADAPTIVE, "parallel": _lib.TITUS_PARALLEL_ADAPTIVE}[method]
    return solver.solve_batched(spots, mid, team_ctas, max_steps)


def scalar_flux(X, sigma, WV):
    """``u = X diag(Sigma) W_mod[1,:]`` (``main.jl:73``), cell order i*ny + j."""
    return X @ (sigma * WV[0, :])
