"""GPU parity of the RK4 ("HighOrder") DLR integrator
(SolveFirstCollisionSourceDLRHighOrder, code/SolverCSD.jl:588-889) against the
FP64 oracle, through the C ABI (method TITUS_DLR_HIGH_ORDER).

The integrator streams with the central operators only and takes its
uncollided part from the limited second-order flux. Measured on the oracle, it
is well conditioned on these cases (a 1e-14 relative density perturbation
moves the dose by <= 2e-14 over whole sweeps), so whole runs are compared.
Tolerance: relative L2 <= 1e-10 on dose, scalar flux, psi and X S W^T.
"""
import numpy as np
import pytest

from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver
from oracle.solver import solve_dlr_high_order
from titus_b200 import Settings, SolverCSD, SolveFirstCollisionSourceDLRHighOrder, scalar_flux
from titus_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def oracle_run(nx, r, problem, npn, steps):
    o = OSolver(OSettings(nx, nx, r, problem, nPN=npn))
    X, sig, _, WV, dose, psi = solve_dlr_high_order(o, max_steps=steps)
    return dose.copy(), scalar_flux(X, sig, WV), psi


def gpu_run(nx, r, problem, npn, steps, team=0):
    g = SolverCSD(Settings(nx, nx, r, problem, nPN=npn), team_ctas=team)
    X, sig, _, WV, dose, psi = SolveFirstCollisionSourceDLRHighOrder(g, max_steps=steps)
    return dose.copy(), scalar_flux(X, sig, WV), psi


@pytest.mark.parametrize("nx,r,npn,problem,steps", [
    (22, 16, 3, "csdWaterBeam", 0),      # exact rank, whole sweep
    (26, 16, 3, "csdPhantom", 400),
    (41, 12, 7, "csdWaterBeam", 40),     # below the solution's rank
    (31, 20, 5, "csdPhantom", 150),
])
def test_sweep_matches_oracle(nx, r, npn, problem, steps):
    od, ou, opsi = oracle_run(nx, r, problem, npn, steps or None)
    gd, gu, gpsi = gpu_run(nx, r, problem, npn, steps)
    assert rel(gd, od) <= TOL
    assert rel(gu, ou) <= TOL
    assert rel(gpsi.ravel(), opsi.ravel()) <= TOL


@pytest.mark.parametrize("team", [1, 5, 24])
def test_team_sizes_agree(team):
    ref = gpu_run(26, 16, "csdPhantom", 3, 120, team=16)
    got = gpu_run(26, 16, "csdPhantom", 3, 120, team=team)
    assert rel(got[0], ref[0]) <= 1e-12 and rel(got[1], ref[1]) <= 1e-12


def test_steps_from_state_at_benchmark_size():
    """100 x 100 water beam, P_21, r = 20: three steps from the oracle's state after 30."""
    nx, r, npn, m = 101, 20, 21, 30
    st = solve_dlr_high_order(OSolver(OSettings(nx, nx, r, "csdWaterBeam", nPN=npn)), max_steps=m,
                              return_state=True)
    g = SolverCSD(Settings(nx, nx, r, "csdWaterBeam", nPN=npn))
    ref = solve_dlr_high_order(OSolver(OSettings(nx, nx, r, "csdWaterBeam", nPN=npn)), max_steps=3, state=st,
                               n_begin=st["n_next"], return_state=True)
    got = g.run_from(_lib.TITUS_DLR_HIGH_ORDER, st, st["n_next"], st["n_next"] + 2)
    assert rel(got["dose"], ref["dose"]) <= TOL
    assert rel(got["X"] @ got["S"] @ got["W"].T, ref["X"] @ ref["S"] @ ref["W"].T) <= TOL
    assert rel(got["psi"].ravel(), ref["psi"].ravel()) <= TOL


def test_rejects_grid_too_small_for_the_limiter():
    g = SolverCSD(Settings(5, 5, 4, "csdWaterBeam", nPN=3))   # 4 x 4 cells
    with pytest.raises(_lib.TitusError, match="nx, ny >= 5"):
        SolveFirstCollisionSourceDLRHighOrder(g, max_steps=3)
