"""GPU parity of the full-rank P_N first-collision solver
(titus_pn_full_solve; SolverCSD.jl:465-586) against the FP64 oracle
(oracle/full_rank.py, itself checked against the reference's per-cell loops).

The scheme is linear and explicit, so rounding does not grow: whole sweeps are
compared at relative L2 <= 1e-10 on u, dose and psi (psi of the last step is
exactly zero once the beam energy factor has underflowed; it is then compared
absolutely)."""
import numpy as np
import pytest

from oracle.full_rank import solve_pn_full
from oracle.settings import Settings as OSettings
from oracle.solver import SolverCSD as OSolver
from titus_b200 import Settings, SolverCSD, SolveFirstCollisionSource

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("nx,npn,problem,steps", [(23, 3, "csdWaterBeam", 0), (33, 5, "csdPhantom", 0),
                                                  (16, 7, "csdWaterBeam", 0), (101, 21, "csdWaterBeam", 100)])
def test_full_rank_sweep(nx, npn, problem, steps):
    o = solve_pn_full(OSolver(OSettings(nx, nx, 4, problem, nPN=npn)), max_steps=steps or None)
    g = SolveFirstCollisionSource(SolverCSD(Settings(nx, nx, 4, problem, nPN=npn)), max_steps=steps)
    assert np.abs(o[1]).max() > 0
    assert rel(g[1], o[1]) <= TOL, rel(g[1], o[1])            # dose
    assert rel(g[0], o[0]) <= TOL, rel(g[0], o[0])            # 1/2 sqrt(gamma_0) u
    if np.linalg.norm(o[2]) > 0:
        assert rel(g[2].ravel(), o[2].ravel()) <= TOL
    else:
        assert np.abs(g[2]).max() <= 1e-300


def test_repeat_is_bitwise_identical():
    s = SolverCSD(Settings(23, 23, 4, "csdPhantom", nPN=3))
    a = SolveFirstCollisionSource(s, max_steps=200)
    b = SolveFirstCollisionSource(s, max_steps=200)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_needs_stopping_mid():
    from titus_b200 import _lib
    import ctypes as C

    s = SolverCSD(Settings(12, 12, 4, "csdWaterBeam", nPN=3))
    p, keep = s.problem_struct()
    p.stopping_mid = None
    h = C.c_void_p()
    lib = _lib.load()
    _lib.check(lib.titus_create(C.byref(p), C.byref(h)), "titus_create")
    opt = s.options()
    rc = lib.titus_pn_full_solve_device(h, C.byref(opt), None)
    lib.titus_destroy(h)
    assert rc == 1 and "stopping_mid" in _lib.last_error()
