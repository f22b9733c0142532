"""titus_solve_noalloc: the fixed-rank solve for callers that cannot allocate device memory.

Callers whose device memory is owned by a framework allocator or memory pool,
or who run under a policy against device allocation after start-up, hand the
library device pointers they already own; the library keeps its intermediates
in a static device array. Here torch plays that caller and owns the device
buffers. Two calls in a row must agree with the allocating entry point
(titus_solve) to the parity tolerance of the GPU tests. This file is named so
that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from titus_b200 import Settings, SolverCSD
from titus_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def device_problem(solver, torch):
    """A titus_problem_t whose arrays are device pointers to torch-owned copies."""
    p, keep = solver.problem_struct()
    hold = []

    def to_dev(ptr, count, ptype):
        host = np.ctypeslib.as_array(ptr, shape=(max(count, 1),)).copy()
        t = torch.from_numpy(host).cuda()
        hold.append(t)
        return C.cast(C.c_void_p(t.data_ptr()), ptype)

    n, N, q, nE = solver.n, solver.N, solver.q, solver.nE
    npn = solver.settings.nPN
    p.density = to_dev(p.density, n, _lib._dp)
    p.e_trafo = to_dev(p.e_trafo, nE, _lib._dp)
    p.stopping = to_dev(p.stopping, nE, _lib._dp)
    p.bc_energy = to_dev(p.bc_energy, nE, _lib._dp)
    p.sigma = to_dev(p.sigma, nE * (npn + 1), _lib._dp)
    p.bc_space = to_dev(p.bc_space, n, _lib._dp)
    p.bc_angle = to_dev(p.bc_angle, q, _lib._dp)
    p.omega = to_dev(p.omega, q * 3, _lib._dp)
    p.m_reduced = to_dev(p.m_reduced, N * q, _lib._dp)
    for d, (rp, ci, v) in enumerate(solver.ops):
        p.op_rowptr[d] = to_dev(p.op_rowptr[d], N + 1, _lib._ip)
        p.op_col[d] = to_dev(p.op_col[d], len(ci), _lib._ip)
        p.op_val[d] = to_dev(p.op_val[d], len(v), _lib._dp)
    p.x_completion = to_dev(p.x_completion, p.n_x_completion, _lib._ip)
    p.w_completion = to_dev(p.w_completion, p.n_w_completion, _lib._ip)
    p.sweep_restore = to_dev(p.sweep_restore, p.n_sweep_restore, _lib._ip)
    return p, (keep, hold)


def dptr(t):
    return C.cast(C.c_void_p(t.data_ptr()), _lib._dp)


@pytest.mark.parametrize("nx,npn,r,steps", [(22, 3, 16, 80), (41, 7, 12, 30)])
def test_noalloc_matches_allocating_entry_point(nx, npn, r, steps):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    lib = _lib.load()
    g = SolverCSD(Settings(nx, nx, r, "csdWaterBeam", nPN=npn), team_ctas=16)
    ref = g.run(_lib.TITUS_DLR_FIXED, max_steps=steps)
    p, hold = device_problem(g, torch)
    opt = g.options(max_steps=steps)
    n, N, q = g.n, g.N, g.q
    for call in range(2):
        # outputs start as NaN so that anything the call fails to write shows up
        out = [torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
               for shape in ((n,), (n, r), (r, r), (N, r), (n, q))]
        rank = C.c_int32(-1)
        err = C.create_string_buffer(512)
        rc = lib.titus_solve_noalloc(C.byref(p), C.byref(opt), *[dptr(t) for t in out], C.byref(rank),
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream), err, len(err))
        assert rc == 0, err.value.decode()
        assert rank.value == r
        d, Xh, Sh, Wh, ph = (t.cpu().numpy() for t in out)
        assert rel(d, ref["dose"]) <= TOL, call
        assert rel(Xh @ Sh @ Wh.T, ref["X"] @ ref["S"] @ ref["W"].T) <= TOL, call
        assert rel(ph, ref["psi"]) <= TOL, call


def test_noalloc_rejects_oversize_problem():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    lib = _lib.load()
    g = SolverCSD(Settings(801, 801, 8, "csdWaterBeam", nPN=3, nEnergies=3))
    p, hold = device_problem(g, torch)
    opt = g.options()
    n, N, q = g.n, g.N, g.q
    bufs = [torch.zeros(m, dtype=torch.float64, device="cuda") for m in (n, n * 8, 64, N * 8, n * q)]
    err = C.create_string_buffer(512)
    rc = lib.titus_solve_noalloc(C.byref(p), C.byref(opt), *[dptr(b) for b in bufs], None,
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream), err, len(err))
    assert rc == 4
    assert b"scratch" in err.value
