"""Batched pencil beams (titus_solve_batched) against one oracle solve per spot.

Each spot is the base phantom with its own beam energy and entry point, so
the spots run different numbers of energy steps (8 to 58 here) and reach
different ranks; all advance in one persistent launch, teams of CTAs taking
spots in turn. BUG is well conditioned (whole solves compared, dose interior
<= 1e-10, ghost cells <= 1e-8 ||dose||, ranks and iteration counts exact); the
parallel integrator is compared over its first steps.
"""
import numpy as np
import pytest

from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver
from oracle.solver import solve_dlr_bug, solve_dlr_parallel
from titus_b200 import Settings, SolverCSD, SolveBatchedPencilBeams, _lib

pytestmark = pytest.mark.gpu
TOL = 1e-10
SPOTS = [(0.08, 0.42), (0.1, 0.5), (0.22, 0.4), (0.3, 0.45), (0.15, 0.55)]
NX, R, NPN = 31, 12, 5


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def dose_ok(gd, od):
    i, j = np.divmod(np.arange((NX - 1) ** 2), NX - 1)
    b = (i == 0) | (j == 0) | (i == NX - 2) | (j == NX - 2)
    return rel(gd[~b], od[~b]) <= TOL and np.abs(gd[b] - od[b]).max() <= 1e-8 * np.linalg.norm(od)


def oracle_spot(fn, energy, y0, max_steps=None):
    s = OSettings(NX, NX, R, "csdPhantom", nPN=NPN)
    s.eMax, s.y0 = energy, y0
    o = OSolver(s)
    st = fn(o, max_steps=max_steps, return_state=True)
    return st


@pytest.mark.parametrize("team", [2, 60])
def test_bug_batched_matches_per_spot_oracle(team):
    g = SolverCSD(Settings(NX, NX, R, "csdPhantom", nPN=NPN))
    dose, rank, iters = SolveBatchedPencilBeams(g, SPOTS, "bug", team_ctas=team)
    for i, (e, y) in enumerate(SPOTS):
        st = oracle_spot(solve_dlr_bug, e, y)
        assert rank[i] == st["S"].shape[0], (i, rank[i], st["S"].shape[0])
        assert iters[i] == st["iters"], (i, iters[i], st["iters"])
        assert dose_ok(dose[i], st["dose"]), (i, rel(dose[i], st["dose"]))


def test_parallel_batched_first_steps():
    g = SolverCSD(Settings(NX, NX, R, "csdPhantom", nPN=NPN))
    dose, rank, iters = SolveBatchedPencilBeams(g, SPOTS, "parallel", team_ctas=4, max_steps=4)
    for i, (e, y) in enumerate(SPOTS):
        st = oracle_spot(solve_dlr_parallel, e, y, max_steps=4)
        assert rank[i] == st["S"].shape[0]
        assert dose_ok(dose[i], st["dose"]), (i, rel(dose[i], st["dose"]))


def test_batched_equals_single_solves():
    """A spot solved in a batch equals the same spot solved alone (same team size)."""
    base = Settings(NX, NX, R, "csdPhantom", nPN=NPN)
    g = SolverCSD(base)
    dose, rank, iters = SolveBatchedPencilBeams(g, SPOTS[:2], "bug", team_ctas=3)
    for i, (e, y) in enumerate(SPOTS[:2]):
        s = Settings(NX, NX, R, "csdPhantom", nPN=NPN)
        s.eMax, s.y0 = e, y
        single = SolverCSD(s, team_ctas=3)
        out = single.run(_lib.TITUS_BUG_ADAPTIVE)
        assert np.array_equal(out["dose"], dose[i])
        assert out["rank"] == rank[i]
