"""Pins of the oracle's RK4 ("HighOrder") integrator pieces against literal
transcriptions of the reference (SolveFirstCollisionSourceDLRHighOrder,
code/SolverCSD.jl:588-889), on the CPU.

- the two-layer inflow against the reference's element loops (:679-695);
- the limited sweep against the flux oracle (itself pinned to the quadrant
  loops in test_flux.py) and the boundary-slab restore of the upwind sweep;
- one RK4 step of a linear system against its exact fourth-order Taylor
  polynomial, in both of the reference's accumulation forms.
"""
import numpy as np

from oracle.settings import Settings
from oracle.solver import SolverCSD, rk4_accumulated, rk4_summed, solve_dlr_high_order


def _solver(nx=9, ny=11, npn=3):
    o = SolverCSD(Settings(nx, ny, 4, "csdWaterBeam", nPN=npn))
    o.setup_directions()
    return o


def test_two_layer_inflow_matches_element_loops():
    o = _solver()
    s = o.settings
    nx, ny, q = s.NCellsX, s.NCellsY, o.qReduced.shape[0]
    rng = np.random.default_rng(0)
    psi = rng.standard_normal((nx, ny, q))
    ref = psi.copy()
    E, n = o.csd.eGrid[3], 4
    xm, ym = s.xMid, s.yMid
    # literal transcription of :679-695 (1-based loops, 0-based storage)
    for k in range(q):
        Om = o.qReduced[k]
        for j in range(nx):
            ref[j, 0, k] = o.psi_beam(Om, E, xm[j], ym[0], n)[0]
            ref[j, ny - 1, k] = o.psi_beam(Om, E, xm[j], ym[ny - 1], n)[0]
            ref[j, 1, k] = o.psi_beam(Om, E, xm[j], ym[0], n)[0]
            ref[j, ny - 2, k] = o.psi_beam(Om, E, xm[j], ym[ny - 1], n)[0]
        for j in range(ny):
            ref[0, j, k] = o.psi_beam(Om, E, xm[0], ym[j], n)[0]
            ref[nx - 1, j, k] = o.psi_beam(Om, E, xm[nx - 1], ym[j], n)[0]
            ref[1, j, k] = o.psi_beam(Om, E, xm[0], ym[j], n)[0]
            ref[nx - 2, j, k] = o.psi_beam(Om, E, xm[nx - 1], ym[j], n)[0]
    got = psi.copy()
    o.apply_bc_two_layer(got, E, n)
    np.testing.assert_allclose(got, ref, rtol=1e-15, atol=0)
    # the interior (three and more cells in) is untouched
    assert np.array_equal(got[2:-2, 2:-2], psi[2:-2, 2:-2])


def test_limited_sweep_update():
    o = _solver()
    nx, ny = o.settings.NCellsX, o.settings.NCellsY
    rng = np.random.default_rng(1)
    psi = rng.uniform(0.0, 1.0, (nx, ny, o.qReduced.shape[0]))
    dE, s0 = 0.01, 3.0
    flux = o.flux_limited(psi / o.density[:, :, None])
    want = (psi - dE * flux) / (1 + dE * s0)
    L0 = o.boundaryIdx
    want[L0 % nx, L0 // nx, 0] = psi[L0 % nx, L0 // nx, 0]
    got = psi.copy()
    o.sweep_limited(got, dE, s0)
    assert np.array_equal(got, want)
    # the flux buffer is zero on the two outer rings: those cells only decay
    ring = np.ones((nx, ny), bool)
    ring[2:-2, 2:-2] = False
    ring_cells = got[ring][:, 1:]
    np.testing.assert_allclose(ring_cells, psi[ring][:, 1:] / (1 + dE * s0), rtol=1e-15)


def test_rk4_is_the_fourth_order_taylor_step():
    rng = np.random.default_rng(2)
    A = rng.standard_normal((6, 6))
    Y = rng.standard_normal((6, 3))
    dE = 0.07
    f = lambda Z: A @ Z
    taylor = Y.copy()
    term = Y.copy()
    for m in range(1, 5):
        term = dE * (A @ term) / m
        taylor = taylor + term
    for step in (rk4_accumulated, rk4_summed):
        np.testing.assert_allclose(step(Y, dE, f), taylor, rtol=1e-13, atol=1e-13)


def test_high_order_rank_and_shapes():
    """A short run keeps the fixed rank and returns the reference's tuple."""
    s = Settings(12, 12, 5, "csdWaterBeam", nPN=3)
    out = solve_dlr_high_order(SolverCSD(s), max_steps=6)
    X, sig, OWV, WV, dose, psi = out
    n = s.NCellsX * s.NCellsY
    assert X.shape == (n, 5) and sig.shape == (5,) and WV.shape == (16, 5)
    assert dose.shape == (n,) and np.all(np.isfinite(dose)) and dose.max() > 0
