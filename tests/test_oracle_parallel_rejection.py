"""The oracle's SolveFirstCollisionSourceDLRParallelRejection
(SolverCSD.jl:2376-2742) against its parts: without rejections its factors
follow the parallel integrator (SolverCSD.jl:1726-2008) bit for bit, only the
second dose half-step differs (taken after the truncation, :2683, instead of
before it, :1943); a scattering rejection after a streaming step that changed
the rank ends the solve where the reference raises DimensionMismatch (:2553)."""
import numpy as np
import pytest

from oracle.settings import Settings
from oracle.solver import (ReferenceFailure, SolverCSD, solve_dlr_parallel, solve_dlr_parallel_rejection)


def _solver(nx, r, npn, problem, theta=None, c_eta=None):
    s = Settings(nx, nx, r, problem, nPN=npn)
    if theta is not None:
        s.theta = theta
    if c_eta is not None:
        s.c_eta = c_eta
    return SolverCSD(s)


@pytest.mark.parametrize("steps", [1, 2, 12])
def test_factors_follow_parallel_integrator_without_rejections(steps):
    # 24x24 phantom, P7, cap 8 at the default tolerance: no rejection within 30 steps
    a = solve_dlr_parallel_rejection(_solver(24, 8, 7, "csdPhantom"), max_steps=steps, return_state=True)
    b = solve_dlr_parallel(_solver(24, 8, 7, "csdPhantom"), max_steps=steps, return_state=True)
    assert a["iters"] == steps and a["n_next"] == b["n_next"]
    for key in ("X", "S", "W", "psi"):
        assert np.array_equal(a[key], b[key]), key
    # the doses differ by the second half-steps' truncated parts only
    assert not np.array_equal(a["dose"], b["dose"])
    assert np.linalg.norm(a["dose"] - b["dose"]) < 0.05 * np.linalg.norm(b["dose"])


def test_rejections_repeat_energies():
    # 21x21 water beam, P7, cap 16, theta 1e-3: a first-branch rejection at n = 3
    # (rank 2 -> 4) and eta rejections at n = 3 (4 -> 8) and n = 4 (7 -> 14)
    o = solve_dlr_parallel_rejection(_solver(21, 16, 7, "csdWaterBeam", theta=1e-3), max_steps=10)
    ranks = o[5][1].astype(int).tolist()
    energies = o[5][0]
    assert ranks[:6] == [8, 2, 4, 8, 7, 14]
    assert energies[2] == energies[3] and energies[4] == energies[5]
    assert o[6].shape[0] == o[7].shape[0] >= 8


def test_scattering_rejection_after_rank_change_fails_like_the_reference():
    # 24x24 phantom, P5, cap 8, c_eta 0.1: at n = 3 a streaming rejection doubles
    # the rank to 4, the repeated step's truncation leaves rank 3, and then the
    # scattering test rejects
    with pytest.raises(ReferenceFailure, match="DimensionMismatch"):
        solve_dlr_parallel_rejection(_solver(24, 8, 5, "csdPhantom", theta=1e-2, c_eta=0.1), max_steps=10)
