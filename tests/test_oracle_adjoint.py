"""The oracle's discrete adjoint of the full-rank sweep
(oracle/full_rank.py:pn_full_dose_adjoint) against central finite
differences of the oracle's own forward sweep (h = 1e-4 relative).

Objective: J = sum_c mask_c (dose_c - P_c)^2 with a seeded mask and target.
Gradients: per-voxel density (with the energy grid held fixed, as the adjoint
defines it: Settings is built before the density is perturbed) and the
weights of a three-spot plan whose inflow profile is sum_s w_s p_s.
The forward with the settings' own beam reproduces solve_pn_full to rounding.
"""
import numpy as np
import pytest

from oracle.full_rank import beam_profile, pn_full_dose_adjoint, solve_pn_full
from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver

NX, NPN, STEPS = 14, 3, 40
H = 1e-4


def solver(scale=None):
    s = OSettings(NX, NX, 6, "csdPhantom", nPN=NPN)
    if scale is not None:
        s.density = s.density * scale.reshape(s.density.shape)
    return OSolver(s)


def forward(scale=None, profile=None):
    o = solver(scale)
    return pn_full_dose_adjoint(o, np.zeros(o.densityVec.size), max_steps=STEPS, bc_profile=profile)[0]


@pytest.fixture(scope="module")
def plan():
    o = solver()
    s = o.settings
    n = o.densityVec.size
    P = [beam_profile(s, y0=y) for y in (0.35, 0.5, 0.65)]
    w = np.array([0.7, 1.0, 1.3])
    prof = sum(wi * pi for wi, pi in zip(w, P))
    rng = np.random.default_rng(0)
    mask = (rng.random(n) < 0.5).astype(float)
    target = mask * forward(profile=prof).max() * 0.5
    dose, grho, gprof = pn_full_dose_adjoint(solver(), lambda d: 2 * mask * (d - target), max_steps=STEPS,
                                             bc_profile=prof)
    return dict(P=P, w=w, prof=prof, mask=mask, target=target, dose=dose, grho=grho, gprof=gprof, rho=o.densityVec)


def J(p, dose):
    return float(np.sum(p["mask"] * (dose - p["target"]) ** 2))


def test_forward_matches_solve_pn_full():
    d0 = solve_pn_full(solver(), max_steps=STEPS)[1]
    o = solver()
    d1 = pn_full_dose_adjoint(o, np.zeros(o.densityVec.size), max_steps=STEPS)[0]
    d2 = forward(profile=beam_profile(o.settings))
    assert np.linalg.norm(d1 - d0) <= 1e-14 * np.linalg.norm(d0)   # streaming terms summed in another order
    assert np.linalg.norm(d2 - d0) <= 1e-14 * np.linalg.norm(d0)


@pytest.mark.parametrize("spot", [0, 1, 2])
def test_spot_weight_gradient_vs_fd(plan, spot):
    wp, wm = plan["w"].copy(), plan["w"].copy()
    wp[spot] += H
    wm[spot] -= H
    prof = lambda w: sum(wi * pi for wi, pi in zip(w, plan["P"]))  # noqa: E731
    fd = (J(plan, forward(profile=prof(wp))) - J(plan, forward(profile=prof(wm)))) / (2 * H)
    ad = plan["P"][spot] @ plan["gprof"]
    assert abs(fd - ad) <= 1e-8 * abs(fd), (fd, ad)


@pytest.mark.parametrize("cell", [5 * NX + 6, 3 * NX + 3, 9 * NX + 10, 2 * NX + 7])
def test_density_gradient_vs_fd(plan, cell):
    n = plan["rho"].size
    e, em = np.ones(n), np.ones(n)
    e[cell] += H
    em[cell] -= H
    fd = (J(plan, forward(e, plan["prof"])) - J(plan, forward(em, plan["prof"]))) / (2 * H * plan["rho"][cell])
    # central differences carry O(h^2) truncation: 1e-6 relative covers it at h = 1e-4
    assert abs(fd - plan["grho"][cell]) <= 1e-6 * abs(fd), (fd, plan["grho"][cell])


def test_profile_gradient_lives_on_boundary_cells(plan):
    g = plan["gprof"].reshape(NX - 1, NX - 1)
    assert np.all(g[1:-1, 1:-1] == 0.0)
    assert np.abs(g[0, :]).max() > 0
