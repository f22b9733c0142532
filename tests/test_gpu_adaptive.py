"""GPU parity of the rank-adaptive DLR loops against the FP64 oracle:
BUG with rejection (SolverCSD.jl:2011-2374) and the parallel integrator
(:1726-2008), both with truncate! (:3369-3399).

All cases call the CUDA path through the C ABI (libtitus.so via ctypes).
Conditioning measured on the oracle decides what is compared:
* BUG is well conditioned (a 1e-14 density perturbation moves the dose by at
  most 2e-11 over 60-80 steps), so whole runs are compared: dose, scalar flux
  and psi at relative L2 <= 1e-10, the rank of every iteration exactly, and the
  streaming eta values.
* The parallel integrator amplifies rounding by about 100x per step once the
  rank grows (1e-14 -> 3e-9 after 8 steps, then a rank decision flips), so it
  is compared over its first steps and per step from an identical state handed
  to titus_set_state, as the fixed-rank integrator is.
The dose is held to 1e-10 on interior cells. The boundary (ghost) cells hold
rounding noise whenever a completion vector (a canonical boundary-cell
direction with a numerically zero singular value) stays in the basis: X[c] S
W[0,:] there is ~1e-16 of the dose scale and depends on summation order (the
oracle's LAPACK SVD leaves 2e-16 where the GPU leaves 6e-20), so those cells are
bounded absolutely by 1e-8 ||dose||. The scalar flux and the factor product
X S W^T depend on singular directions that are less well determined (in the
(42, P7, 16) BUG run a 1e-14 density perturbation moves the oracle's own scalar
flux by 1e-9 while its dose moves by 2e-11), so their bound is
max(1e-10, 4 x the oracle's own change under 1e-14 input perturbations),
measured in the test.
"""
import numpy as np
import pytest

from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver
from oracle.solver import solve_dlr_bug, solve_dlr_parallel
from titus_b200 import (Settings, SolverCSD, SolveFirstCollisionSourceDLRBUGRejection,
                        SolveFirstCollisionSourceDLRParallel, scalar_flux)
from titus_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def bnd_mask(nx):
    i, j = np.divmod(np.arange((nx - 1) ** 2), nx - 1)
    return (i == 0) | (j == 0) | (i == nx - 2) | (j == nx - 2)


def dose_ok(gd, od, nx):
    """Interior relative L2 <= TOL; ghost cells absolutely <= 1e-8 ||dose||."""
    b = bnd_mask(nx)
    return rel(gd[~b], od[~b]) <= TOL and np.abs(gd[b] - od[b]).max() <= 1e-8 * np.linalg.norm(od)


def osolver(nx, r, npn, problem="csdWaterBeam", eps=0.0, seed=1):
    s = OSettings(nx, nx, r, problem, nPN=npn)
    if eps:
        rng = np.random.default_rng(seed)
        s.density = s.density * (1 + eps * rng.standard_normal(s.density.shape))
    return OSolver(s)


def oracle_sensitivity(fn, nx, r, npn, steps, problem="csdWaterBeam"):
    """The oracle's own relative change of the scalar flux and of the eta
    history (BUG) under 1e-14 density noise, max over two seeds."""
    base = fn(osolver(nx, r, npn, problem), max_steps=steps)
    u0 = scalar_flux(base[0], base[1], base[3])
    su = se = 0.0
    for seed in (1, 2):
        o = fn(osolver(nx, r, npn, problem, 1e-14, seed), max_steps=steps)
        su = max(su, rel(scalar_flux(o[0], o[1], o[3]), u0))
        if fn is solve_dlr_bug and o[6].shape == base[6].shape and base[6].size:
            se = max(se, np.max(np.abs(o[6][:, 1] - base[6][:, 1]) / np.abs(base[6][:, 1]).max()))
    return su, se


def gsolver(nx, r, npn, problem="csdWaterBeam", team=0):
    return SolverCSD(Settings(nx, nx, r, problem, nPN=npn), team_ctas=team)


@pytest.mark.parametrize("nx,npn,r,steps", [(23, 3, 8, 60), (30, 5, 12, 80), (42, 7, 16, 60), (23, 5, 16, 60)])
def test_bug_sweep(nx, npn, r, steps):
    o = solve_dlr_bug(osolver(nx, r, npn), max_steps=steps)
    g = SolveFirstCollisionSourceDLRBUGRejection(gsolver(nx, r, npn), max_steps=steps)
    np.testing.assert_array_equal(g[5][1], o[5][1])          # rank per iteration
    np.testing.assert_allclose(g[5][0], o[5][0], rtol=1e-12)  # energy per iteration
    assert dose_ok(g[4], o[4], nx)                           # dose
    assert rel(g[8].ravel(), o[8].ravel()) <= TOL            # psi
    assert g[6].shape[0] == o[6].shape[0]
    uerr = rel(scalar_flux(g[0], g[1], g[3]), scalar_flux(o[0], o[1], o[3]))
    eerr = np.max(np.abs(g[6][:, 1] - o[6][:, 1]) / np.abs(o[6][:, 1]).max()) if o[6].size else 0.0
    if uerr > TOL or eerr > 1e-8:
        su, se = oracle_sensitivity(solve_dlr_bug, nx, r, npn, steps)
        assert uerr <= max(TOL, 4 * su)
        assert eerr <= max(1e-8, 4 * se)
    np.testing.assert_allclose(g[7][:, 1], o[7][:, 1], rtol=1e-10)


def test_bug_phantom():
    o = solve_dlr_bug(osolver(26, 8, 3, "csdPhantom"), max_steps=100)
    g = SolveFirstCollisionSourceDLRBUGRejection(gsolver(26, 8, 3, "csdPhantom"), max_steps=100)
    np.testing.assert_array_equal(g[5][1], o[5][1])
    assert dose_ok(g[4], o[4], 26)
    assert rel(scalar_flux(g[0], g[1], g[3]), scalar_flux(o[0], o[1], o[3])) <= TOL


def test_bug_team_sizes_agree():
    ref = None
    for team in (1, 3, 16):
        g = SolveFirstCollisionSourceDLRBUGRejection(gsolver(30, 12, 5, team=team), max_steps=40)
        if ref is None:
            ref = g
            continue
        np.testing.assert_array_equal(g[5][1], ref[5][1])
        assert rel(g[4], ref[4]) <= 1e-12


@pytest.mark.parametrize("nx,npn,r,steps", [(23, 3, 8, 5), (30, 5, 12, 5), (42, 7, 16, 4)])
def test_parallel_first_steps(nx, npn, r, steps):
    o = solve_dlr_parallel(osolver(nx, r, npn), max_steps=steps)
    g = SolveFirstCollisionSourceDLRParallel(gsolver(nx, r, npn), max_steps=steps)
    np.testing.assert_array_equal(g[5][1], o[5][1])
    assert dose_ok(g[4], o[4], nx)
    assert rel(scalar_flux(g[0], g[1], g[3]), scalar_flux(o[0], o[1], o[3])) <= TOL
    assert rel(g[6].ravel(), o[6].ravel()) <= TOL


def _product(X, S, W):
    return X @ S @ W.T


@pytest.mark.parametrize("method", ["parallel", "bug"])
@pytest.mark.parametrize("nx,npn,r,warm,steps", [(23, 3, 8, 20, 1), (30, 5, 12, 40, 3), (42, 7, 16, 30, 1)])
def test_steps_from_state(method, nx, npn, r, warm, steps):
    fn = solve_dlr_parallel if method == "parallel" else solve_dlr_bug
    mid = _lib.TITUS_PARALLEL_ADAPTIVE if method == "parallel" else _lib.TITUS_BUG_ADAPTIVE
    st = fn(osolver(nx, r, npn), max_steps=warm, return_state=True)
    ref = fn(osolver(nx, r, npn), max_steps=steps, state=st, n_begin=st["n_next"], return_state=True)
    g = gsolver(nx, r, npn)
    n_stop = g.nE if method == "bug" else st["n_next"] + steps - 1
    if method == "bug":
        out = g.run_from(mid, st, st["n_next"], n_stop, max_steps=steps)
    else:
        out = g.run_from(mid, st, st["n_next"], n_stop)
    assert out["rank"] == ref["S"].shape[0]
    assert dose_ok(out["dose"], ref["dose"], nx)
    P_ref = _product(ref["X"], ref["S"], ref["W"])
    perr = rel(_product(out["X"], out["S"], out["W"]), P_ref)
    if perr > TOL:
        # the oracle's own change when the handed-over S carries 1e-14 noise
        sens = 0.0
        for seed in (1, 2):
            rng = np.random.default_rng(seed)
            st2 = dict(st)
            st2["S"] = st["S"] * (1 + 1e-14 * rng.standard_normal(st["S"].shape))
            o2 = fn(osolver(nx, r, npn), max_steps=steps, state=st2, n_begin=st["n_next"], return_state=True)
            sens = max(sens, rel(_product(o2["X"], o2["S"], o2["W"]), P_ref))
        assert perr <= max(TOL, 4 * sens)
    assert rel(out["psi"].ravel(), ref["psi"].ravel()) <= TOL


@pytest.mark.parametrize("method,steps", [(_lib.TITUS_PARALLEL_ADAPTIVE, 12), (_lib.TITUS_BUG_ADAPTIVE, 40)])
def test_deterministic_repeat(method, steps):
    g = gsolver(30, 12, 5, team=16)
    a = g.run(method, max_steps=steps)
    b = g.run(method, max_steps=steps)
    assert np.array_equal(a["dose"], b["dose"])
    assert np.array_equal(a["X"], b["X"]) and np.array_equal(a["S"], b["S"]) and np.array_equal(a["W"], b["W"])
    assert np.array_equal(a["rank_history"], b["rank_history"])


def test_fixed_rank_cap_rejected_at_solve():
    g = gsolver(22, 25, 7)
    with pytest.raises(_lib.TitusError, match="rank"):
        g.run(_lib.TITUS_DLR_FIXED, max_steps=2)


@pytest.mark.parametrize("method,theta,steps", [("bug", 1e-3, 30), ("parallel", 3e-5, 6)])
def test_rank_cap_80_with_growing_rank(method, theta, steps):
    """settings.r = 80 (the largest cap): rank 40 entering the first step
    (augmented width 80), then a tighter truncation tolerance lets the rank grow
    (BUG: to 26 through rejections within 30 steps)."""
    nx, npn, r = 26, 9, 80
    os_ = OSettings(nx, nx, r, "csdPhantom", nPN=npn)
    os_.theta = theta
    gs = Settings(nx, nx, r, "csdPhantom", nPN=npn)
    gs.theta = theta
    if method == "bug":
        o = solve_dlr_bug(OSolver(os_), max_steps=steps)
        g = SolveFirstCollisionSourceDLRBUGRejection(SolverCSD(gs), max_steps=steps)
        assert o[5][1].max() >= 20
    else:
        o = solve_dlr_parallel(OSolver(os_), max_steps=steps)
        g = SolveFirstCollisionSourceDLRParallel(SolverCSD(gs), max_steps=steps)
    np.testing.assert_array_equal(g[5][1], o[5][1])
    assert dose_ok(g[4], o[4], nx)


def test_rank_beyond_capacity_fails_cleanly():
    """A BUG rejection that doubles the rank past 40 (26 -> 52 here, with a
    tight tolerance on 100 moments) ends the solve with TITUS_ERR_LIMIT; the
    context stays usable for the next solve."""
    nx, npn, r = 26, 9, 80
    gs = Settings(nx, nx, r, "csdPhantom", nPN=npn)
    gs.theta = 1e-4
    g = SolverCSD(gs)
    with pytest.raises(_lib.TitusError, match="capacity"):
        g.run(_lib.TITUS_BUG_ADAPTIVE, max_steps=120)
    out = gsolver(23, 8, 3).run(_lib.TITUS_BUG_ADAPTIVE, max_steps=5)
    assert np.isfinite(out["dose"]).all()


def test_truncation_completes_with_canonical_vectors():
    """21x21 water beam, P7, cap 16, theta 1e-3: at n = 3 the augmented basis
    [X X~] has a zero column (X's second column was a boundary cell, zeroed by
    the K-step) and truncate! keeps all four directions of a rank-3 S_new. No
    row of the basis completes the fourth left direction, so the canonical
    vectors of R^4 must be tried, from the first one."""
    nx, npn, r, steps = 21, 7, 16, 3
    os_ = OSettings(nx, nx, r, "csdWaterBeam", nPN=npn)
    os_.theta = 1e-3
    gs = Settings(nx, nx, r, "csdWaterBeam", nPN=npn)
    gs.theta = 1e-3
    o = solve_dlr_parallel(OSolver(os_), max_steps=steps)
    g = SolveFirstCollisionSourceDLRParallel(SolverCSD(gs), max_steps=steps)
    np.testing.assert_array_equal(g[5][1], o[5][1])
    assert dose_ok(g[4], o[4], nx)
