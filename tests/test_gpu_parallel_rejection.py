"""GPU parity of SolveFirstCollisionSourceDLRParallelRejection
(SolverCSD.jl:2376-2742, TITUS_PARALLEL_REJECTION) against the FP64 oracle.

The integrator is built on the parallel integrator's augmented step, which
amplifies rounding (the oracle's own dose moves by 1e-5 - 1e-2 after 40
iterations under 1e-14 density noise, with rank decisions flipping), so whole
runs are compared over their first iterations, where the rejections of both
kinds happen, and per iteration from an identical state handed to
titus_set_state. Ranks and energies per iteration must be equal; dose and
scalar flux within max(1e-10, 4 x the oracle's own change under 1e-14 density
noise), measured in the test; psi at 1e-10.
"""
import numpy as np
import pytest

from oracle.settings import Settings as OSettings
from oracle.solver import ReferenceFailure, SolverCSD as OSolver
from oracle.solver import solve_dlr_parallel_rejection
from titus_b200 import Settings, SolverCSD, SolveFirstCollisionSourceDLRParallelRejection, scalar_flux
from titus_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _settings(cls, nx, r, npn, problem, theta, c_eta):
    s = cls(nx, nx, r, problem, nPN=npn)
    s.theta = theta
    s.c_eta = c_eta
    return s


def osolver(nx, r, npn, problem, theta, c_eta, eps=0.0, seed=1):
    s = _settings(OSettings, nx, r, npn, problem, theta, c_eta)
    if eps:
        rng = np.random.default_rng(seed)
        s.density = s.density * (1 + eps * rng.standard_normal(s.density.shape))
    return OSolver(s)


def gsolver(nx, r, npn, problem, theta, c_eta):
    return SolverCSD(_settings(Settings, nx, r, npn, problem, theta, c_eta))


def inner(nx):
    i, j = np.divmod(np.arange((nx - 1) ** 2), nx - 1)
    return (i > 0) & (j > 0) & (i < nx - 2) & (j < nx - 2)


# (nx, r, nPN, problem, theta, c_eta, iterations): rejections covered
CASES = [
    (21, 16, 7, "csdWaterBeam", 1e-3, 5.0, 10),   # first-branch at n=3, eta rejections at n=3 and n=4
    (24, 12, 5, "csdPhantom", 3e-3, 1.0, 10),     # streaming eta rejection, scattering rejection at n=6
    (24, 16, 7, "csdWaterBeam", 3e-3, 5.0, 9),    # first-branch and eta rejections at n=3
]


@pytest.mark.parametrize("nx,r,npn,problem,theta,c_eta,steps", CASES)
def test_first_iterations(nx, r, npn, problem, theta, c_eta, steps):
    args = (nx, r, npn, problem, theta, c_eta)
    o = solve_dlr_parallel_rejection(osolver(*args), max_steps=steps)
    g = SolveFirstCollisionSourceDLRParallelRejection(gsolver(*args), max_steps=steps)
    assert len(set(o[5][0])) < steps                            # energies repeat: rejections happened
    np.testing.assert_array_equal(g[5][1], o[5][1])             # rank per iteration
    np.testing.assert_allclose(g[5][0], o[5][0], rtol=1e-12)    # energy per iteration
    assert rel(g[8].ravel(), o[8].ravel()) <= TOL               # psi
    assert g[6].shape[0] == o[6].shape[0]
    np.testing.assert_allclose(g[7][:, 1], o[7][:, 1], rtol=1e-8)
    m = inner(nx)
    derr = rel(g[4][m], o[4][m])
    uerr = rel(scalar_flux(g[0], g[1], g[3]), scalar_flux(o[0], o[1], o[3]))
    if derr > TOL or uerr > TOL:
        sd = su = 0.0
        u0 = scalar_flux(o[0], o[1], o[3])
        for seed in (1, 2):
            p = solve_dlr_parallel_rejection(osolver(*args, eps=1e-14, seed=seed), max_steps=steps)
            sd = max(sd, rel(p[4][m], o[4][m]))
            su = max(su, rel(scalar_flux(p[0], p[1], p[3]), u0))
        assert derr <= max(TOL, 4 * sd)
        assert uerr <= max(TOL, 4 * su)


def test_reference_failure_reported_and_handle_reusable():
    """A scattering rejection after a streaming step that changed the rank is
    where the reference's next step raises DimensionMismatch: the oracle
    raises, the GPU solve returns TITUS_ERR_DEVICE, and the handle still
    solves the next problem."""
    args = (24, 8, 5, "csdPhantom", 1e-2, 0.1)
    with pytest.raises(ReferenceFailure):
        solve_dlr_parallel_rejection(osolver(*args), max_steps=10)
    g = gsolver(*args)
    with pytest.raises(_lib.TitusError, match="DimensionMismatch"):
        g.run(_lib.TITUS_PARALLEL_REJECTION, max_steps=10)
    out = g.run(_lib.TITUS_BUG_ADAPTIVE, max_steps=5)
    assert np.isfinite(out["dose"]).all()


@pytest.mark.parametrize("warm,steps", [(30, 1), (45, 3)])
def test_steps_from_state(warm, steps):
    args = (24, 16, 7, "csdPhantom", 1e-3, 5.0)
    nx = args[0]
    st = solve_dlr_parallel_rejection(osolver(*args), max_steps=warm, return_state=True)
    ref = solve_dlr_parallel_rejection(osolver(*args), max_steps=steps, state=st, n_begin=st["n_next"],
                                       return_state=True)
    g = gsolver(*args)
    out = g.run_from(_lib.TITUS_PARALLEL_REJECTION, st, st["n_next"], g.nE, max_steps=steps)
    assert out["rank"] == ref["S"].shape[0]
    m = inner(nx)
    P_ref = ref["X"] @ ref["S"] @ ref["W"].T
    derr = rel(out["dose"][m], ref["dose"][m])
    perr = rel(out["X"] @ out["S"] @ out["W"].T, P_ref)
    if derr > TOL or perr > TOL:
        sd = sp = 0.0
        for seed in (1, 2):
            rng = np.random.default_rng(seed)
            st2 = dict(st)
            st2["S"] = st["S"] * (1 + 1e-14 * rng.standard_normal(st["S"].shape))
            o2 = solve_dlr_parallel_rejection(osolver(*args), max_steps=steps, state=st2, n_begin=st["n_next"],
                                              return_state=True)
            sd = max(sd, rel(o2["dose"][m], ref["dose"][m]))
            sp = max(sp, rel(o2["X"] @ o2["S"] @ o2["W"].T, P_ref))
        assert derr <= max(TOL, 4 * sd)
        assert perr <= max(TOL, 4 * sp)
    assert rel(out["psi"].ravel(), ref["psi"].ravel()) <= TOL


def test_deterministic_repeat():
    g = gsolver(24, 16, 7, "csdWaterBeam", 3e-3, 5.0)
    a = g.run(_lib.TITUS_PARALLEL_REJECTION, max_steps=20)
    b = g.run(_lib.TITUS_PARALLEL_REJECTION, max_steps=20)
    assert np.array_equal(a["dose"], b["dose"]) and np.array_equal(a["S"], b["S"])
    assert np.array_equal(a["rank_history"], b["rank_history"])


def test_mixed_precision_rejected():
    g = gsolver(21, 16, 7, "csdWaterBeam", 1e-3, 5.0)
    g.precision = _lib.TITUS_PRECISION_MIXED
    with pytest.raises(_lib.TitusError, match="MIXED"):
        g.run(_lib.TITUS_PARALLEL_REJECTION, max_steps=2)
