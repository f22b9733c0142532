"""GPU parity of the fixed-rank DLR energy loop (SolverCSD.jl:891-1120) against the FP64 oracle.

All cases call the CUDA path through the C ABI (libtitus.so via ctypes).
The fixed-rank integrator is well conditioned when r equals the number of
moments (exact-rank regime): there whole sweeps are compared. With r below
the solution's rank the integrator amplifies rounding in directions with tiny
singular values; there parity is checked per energy step from an identical
state (the same state is given to the oracle and to titus_set_state).
Tolerance: relative L2 <= 1e-10 on dose and scalar flux (plain FP64 mode).
"""
import numpy as np
import pytest

from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver
from oracle.solver import solve_dlr_fixed
from titus_b200 import Settings, SolverCSD, SolveFirstCollisionSourceDLR, scalar_flux
from titus_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def oracle_run(nx, ny, r, problem, npn, steps, **kw):
    s = OSettings(nx, ny, r, problem, nPN=npn)
    o = OSolver(s)
    X, sig, OWV, WV, dose, psi = solve_dlr_fixed(o, max_steps=steps, **kw)
    return dose.copy(), scalar_flux(X, sig, WV), sig, psi


def gpu_run(nx, ny, r, problem, npn, steps, team=0):
    s = Settings(nx, ny, r, problem, nPN=npn)
    g = SolverCSD(s, team_ctas=team)
    X, sig, OWV, WV, dose, psi = SolveFirstCollisionSourceDLR(g, max_steps=steps)
    return dose.copy(), scalar_flux(X, sig, WV), sig, psi


@pytest.mark.parametrize("nx,ny,npn,steps", [(22, 22, 3, 0), (17, 25, 2, 0), (33, 29, 3, 0)])
def test_exact_rank_sweep(nx, ny, npn, steps):
    r = (npn + 1) ** 2
    od, ou, osig, opsi = oracle_run(nx, ny, r, "csdWaterBeam", npn, steps or None)
    gd, gu, gsig, gpsi = gpu_run(nx, ny, r, "csdWaterBeam", npn, steps)
    assert rel(gd, od) <= TOL
    assert rel(gu, ou) <= TOL
    assert np.abs(gsig - osig).max() <= TOL * osig.max()
    assert rel(gpsi.ravel(), opsi.ravel()) <= TOL


def test_exact_rank_phantom():
    npn = 3
    r = 16
    od, ou, _, _ = oracle_run(26, 26, r, "csdPhantom", npn, 400)
    gd, gu, _, _ = gpu_run(26, 26, r, "csdPhantom", npn, 400)
    assert rel(gd, od) <= TOL and rel(gu, ou) <= TOL


@pytest.mark.parametrize("team", [1, 3, 16])
def test_team_sizes_agree(team):
    ref = gpu_run(22, 22, 16, "csdWaterBeam", 3, 200, team=16)
    got = gpu_run(22, 22, 16, "csdWaterBeam", 3, 200, team=team)
    assert rel(got[0], ref[0]) <= 1e-12 and rel(got[1], ref[1]) <= 1e-12


def test_deterministic_repeat():
    a = gpu_run(22, 22, 16, "csdWaterBeam", 3, 150, team=8)
    b = gpu_run(22, 22, 16, "csdWaterBeam", 3, 150, team=8)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[3], b[3])


@pytest.mark.parametrize("nx,r,npn,m", [(41, 12, 7, 40), (41, 8, 9, 25), (101, 20, 21, 12)])
def test_single_step_from_state(nx, r, npn, m):
    """Low-rank regime: one and three energy steps from the oracle's state after m steps."""
    s = OSettings(nx, nx, r, "csdWaterBeam", nPN=npn)
    o = OSolver(s)
    st = solve_dlr_fixed(o, max_steps=m, return_state=True)
    gs = Settings(nx, nx, r, "csdWaterBeam", nPN=npn)
    g = SolverCSD(gs)
    for nsteps in (1, 3):
        o2 = OSolver(OSettings(nx, nx, r, "csdWaterBeam", nPN=npn))
        ref = solve_dlr_fixed(o2, max_steps=nsteps, state=st, n_begin=st["n_next"], return_state=True)
        got = g.run_from(_lib.TITUS_DLR_FIXED, st, st["n_next"], st["n_next"] + nsteps - 1)
        U_ref = ref["X"] @ ref["S"] @ ref["W"].T
        U_got = got["X"] @ got["S"] @ got["W"].T
        assert rel(got["dose"], ref["dose"]) <= TOL
        assert rel(U_got, U_ref) <= TOL
        assert rel(got["psi"].ravel(), ref["psi"].ravel()) <= TOL


def test_benchmark_problem_first_steps():
    """Benchmark problem (100 x 100 cells, P_21, r = 20) for its first 10 energy steps."""
    od, ou, _, _ = oracle_run(101, 101, 20, "csdWaterBeam", 21, 10)
    gd, gu, _, _ = gpu_run(101, 101, 20, "csdWaterBeam", 21, 10)
    assert rel(gd, od) <= TOL and rel(gu, ou) <= TOL


def test_minimal_grid():
    # 3 x 3 cells: a single interior cell
    od, ou, _, _ = oracle_run(4, 4, 4, "csdWaterBeam", 3, 20)
    gd, gu, _, _ = gpu_run(4, 4, 4, "csdWaterBeam", 3, 20)
    assert rel(gd, od) <= TOL and rel(gu, ou) <= TOL


def test_rejects_rank_beyond_build():
    s = Settings(22, 22, _lib.load().titus_max_rank() + 1, "csdWaterBeam", nPN=7)
    g = SolverCSD(s)
    with pytest.raises(_lib.TitusError, match="rank"):
        g.handle()
