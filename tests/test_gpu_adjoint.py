"""GPU discrete adjoint of the full-rank sweep (titus_dose_adjoint,
TITUS_PN_FULL) through the C ABI.

* Against the oracle's adjoint (oracle/full_rank.py:pn_full_dose_adjoint,
  itself checked against central finite differences in
  tests/test_oracle_adjoint.py): dose, dJ/drho and dJ/dprofile at relative
  L2 <= 1e-10. The scheme is linear and explicit in the state, so rounding
  does not grow.
* Checkpoint interval k: every k gives bitwise the same result (the
  recomputed segments repeat the forward pass's arithmetic exactly).
* Central finite differences (h = 1e-4) through the GPU's own forward sweep
  on a 31 x 31, P5 phantom plan of 4 spots: 5 voxel densities and the 4 spot
  weights, relative error <= 1e-6 (the O(h^2) truncation of the difference).
* A 128 x 128 phantom at P21 with a 4-spot plan (the adjoint-optimisation
  grid), its first 20 energy steps, against the oracle.
"""
import numpy as np
import pytest

from oracle.full_rank import pn_full_dose_adjoint
from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver
from titus_b200 import DoseAdjoint, Settings, SolverCSD, SolveFirstCollisionSource, _lib

pytestmark = pytest.mark.gpu
TOL = 1e-10
H = 1e-4


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def plan_for(g, ys, w):
    P = [g.beam_profile(y0=y) for y in ys]
    return P, sum(wi * pi for wi, pi in zip(w, P))


def gsolver(nx, npn, problem, scale=None):
    st = Settings(nx, nx, 4, problem, nPN=npn)
    if scale is not None:
        st.density = st.density * scale.reshape(st.density.shape)   # energy grid stays as built
    return SolverCSD(st)


def osolver(nx, npn, problem):
    return OSolver(OSettings(nx, nx, 4, problem, nPN=npn))


def objective(nx, npn, problem, steps, ys, w, seed=0):
    g = gsolver(nx, npn, problem)
    P, prof = plan_for(g, ys, w)
    g.set_beam_profile(prof)
    d = SolveFirstCollisionSource(g, max_steps=steps)[1]
    rng = np.random.default_rng(seed)
    mask = (rng.random(g.n) < 0.5).astype(float)
    target = mask * 0.5 * d.max()
    return g, P, prof, mask, target


@pytest.mark.parametrize("nx,npn,problem,steps,every", [(23, 3, "csdWaterBeam", 0, 0), (26, 5, "csdPhantom", 200, 7),
                                                        (33, 7, "csdPhantom", 100, 1), (22, 3, "csdPhantom", 60, 60)])
def test_adjoint_matches_oracle(nx, npn, problem, steps, every):
    ys, w = (0.4, 0.5, 0.62), np.array([0.8, 1.0, 1.2])
    g, P, prof, mask, target = objective(nx, npn, problem, steps, ys, w)
    J, dose, grho, gprof = DoseAdjoint(g, weight=mask, target=target, checkpoint_every=every, max_steps=steps)
    o = osolver(nx, npn, problem)
    od, ogr, ogp = pn_full_dose_adjoint(o, lambda d: 2 * mask * (d - target), max_steps=steps or None,
                                        bc_profile=prof)
    assert rel(dose, od) <= TOL
    assert rel(grho, ogr) <= TOL, rel(grho, ogr)
    assert rel(gprof, ogp) <= TOL, rel(gprof, ogp)
    assert abs(J - np.sum(mask * (od - target) ** 2)) <= 1e-10 * abs(J)
    for s in range(len(ys)):
        assert abs(P[s] @ gprof - P[s] @ ogp) <= 1e-10 * abs(P[s] @ ogp)


def test_checkpoint_interval_is_bitwise_neutral():
    g, P, prof, mask, target = objective(26, 5, "csdPhantom", 90, (0.45, 0.55), np.array([1.0, 0.6]))
    ref = DoseAdjoint(g, weight=mask, target=target, checkpoint_every=1, max_steps=90)
    for k in (4, 13, 0, 90, 1000):
        got = DoseAdjoint(g, weight=mask, target=target, checkpoint_every=k, max_steps=90)
        assert got[0] == ref[0]
        for a, b in zip(got[1:], ref[1:]):
            assert np.array_equal(a, b), k


def test_given_dose_gradient_equals_least_squares():
    g, P, prof, mask, target = objective(22, 3, "csdPhantom", 80, (0.5,), np.array([1.0]))
    J, dose, grho, gprof = DoseAdjoint(g, weight=mask, target=target, max_steps=80)
    J2, dose2, grho2, gprof2 = DoseAdjoint(g, dj_ddose=2 * mask * (dose - target), max_steps=80)
    assert np.isnan(J2)
    assert np.array_equal(dose, dose2) and np.array_equal(grho, grho2) and np.array_equal(gprof, gprof2)


def test_fd_through_the_gpu_forward():
    nx, npn, steps = 31, 5, 300
    ys, w = (0.3, 0.45, 0.55, 0.7), np.array([0.9, 1.1, 1.0, 0.7])
    g, P, prof, mask, target = objective(nx, npn, "csdPhantom", steps, ys, w, seed=3)
    J, dose, grho, gprof = DoseAdjoint(g, weight=mask, target=target, checkpoint_every=16, max_steps=steps)

    def Jf(scale=None, weights=w):
        gg = gsolver(nx, npn, "csdPhantom", scale)
        gg.set_beam_profile(sum(wi * pi for wi, pi in zip(weights, P)))
        d = SolveFirstCollisionSource(gg, max_steps=steps)[1]
        gg.close()
        return float(np.sum(mask * (d - target) ** 2))

    assert abs(Jf() - J) <= 1e-12 * J
    for s in range(len(ys)):
        wp, wm = w.copy(), w.copy()
        wp[s] += H
        wm[s] -= H
        fd = (Jf(weights=wp) - Jf(weights=wm)) / (2 * H)
        assert abs(fd - P[s] @ gprof) <= 1e-6 * abs(fd), (s, fd, P[s] @ gprof)
    rho = g.density
    n1 = nx - 1
    for (i, j) in [(5, 15), (10, 12), (15, 18), (20, 10), (8, 22)]:
        c = i * n1 + j
        e, em = np.ones(g.n), np.ones(g.n)
        e[c] += H
        em[c] -= H
        fd = (Jf(e) - Jf(em)) / (2 * H * rho[c])
        assert abs(fd - grho[c]) <= 1e-6 * abs(fd), (c, fd, grho[c])


def test_phantom_128_P21_plan_first_steps():
    nx, npn, steps = 129, 21, 20
    ys, w = (0.35, 0.45, 0.55, 0.65), np.array([1.0, 0.8, 1.2, 0.9])
    g, P, prof, mask, target = objective(nx, npn, "csdPhantom", steps, ys, w, seed=5)
    J, dose, grho, gprof = DoseAdjoint(g, weight=mask, target=target, checkpoint_every=4, max_steps=steps)
    od, ogr, ogp = pn_full_dose_adjoint(osolver(nx, npn, "csdPhantom"), lambda d: 2 * mask * (d - target),
                                        max_steps=steps, bc_profile=prof)
    assert rel(dose, od) <= TOL
    assert rel(grho, ogr) <= TOL
    assert rel(gprof, ogp) <= TOL


def test_rejects_methods_without_an_adjoint():
    g = gsolver(22, 3, "csdWaterBeam")
    lib = _lib.load()
    nul = _lib.C.POINTER(_lib.C.c_double)()
    opt = g.options(5)
    rc = lib.titus_dose_adjoint(g.handle(), _lib.TITUS_BUG_ADAPTIVE, _lib.C.byref(opt), nul, nul, nul, 0, nul, nul,
                                nul, nul)
    assert rc == 1   # TITUS_ERR_ARG
    with pytest.raises(_lib.TitusError, match="no adjoint"):
        _lib.check(rc, "titus_dose_adjoint")
    g2 = SolverCSD(Settings(22, 22, 4, "csdWaterBeam", nPN=3), precision=_lib.TITUS_PRECISION_MIXED)
    with pytest.raises(_lib.TitusError, match="FP64 only"):
        DoseAdjoint(g2, max_steps=5)
