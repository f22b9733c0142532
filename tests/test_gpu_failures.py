"""Failure detection on the GPU without faulting it.

* A team barrier whose wait runs out: the test hook titus_debug_barrier_fault
  makes CTA 1 of the next launch skip its arrival at one barrier and bounds
  every wait by a few thousand polls. The other CTAs' waits run out, the kernel
  leaves, titus_solve returns TITUS_ERR_DEVICE naming that barrier, and the
  next solve on the same handle gives the same result as before the fault.
* A device allocation that fails inside titus_create (injected on the host,
  titus_debug_fail_alloc): TITUS_ERR_CUDA, and every allocation made before it
  is released (free device memory returns to where it was).
"""
import ctypes as C
import time

import numpy as np
import pytest

from titus_b200 import Settings, SolverCSD, _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,barrier", [(_lib.TITUS_DLR_FIXED, 7), (_lib.TITUS_BUG_ADAPTIVE, 9),
                                            (_lib.TITUS_PARALLEL_ADAPTIVE, 30)])
def test_barrier_wait_runs_out_and_handle_recovers(method, barrier):
    g = SolverCSD(Settings(23, 23, 8, "csdWaterBeam", nPN=3), team_ctas=4)
    ref = g.run(method, max_steps=10)
    lib = _lib.load()
    _lib.check(lib.titus_debug_barrier_fault(g.handle(), barrier, 1 << 14), "titus_debug_barrier_fault")
    t0 = time.perf_counter()
    with pytest.raises(_lib.TitusError) as ei:
        g.run(method, max_steps=10)
    assert time.perf_counter() - t0 < 20.0
    msg = str(ei.value)
    assert "status 3" in msg and "barrier timeout" in msg and f"at barrier {barrier} " in msg, msg
    again = g.run(method, max_steps=10)
    assert np.array_equal(again["dose"], ref["dose"])
    assert np.array_equal(again["X"], ref["X"]) and np.array_equal(again["S"], ref["S"])


def test_batched_barrier_wait_runs_out():
    g = SolverCSD(Settings(23, 23, 8, "csdPhantom", nPN=3))
    spots = [(0.1, 0.5), (0.2, 0.45)]
    from titus_b200 import SolveBatchedPencilBeams
    ref = SolveBatchedPencilBeams(g, spots, "bug", team_ctas=3, max_steps=8)
    _lib.check(_lib.load().titus_debug_barrier_fault(g.handle(), 5, 1 << 14), "titus_debug_barrier_fault")
    with pytest.raises(_lib.TitusError, match="status 3"):
        SolveBatchedPencilBeams(g, spots, "bug", team_ctas=3, max_steps=8)
    again = SolveBatchedPencilBeams(g, spots, "bug", team_ctas=3, max_steps=8)
    assert np.array_equal(again[0], ref[0])


def test_injected_allocation_failure_releases_everything():
    import torch

    s = SolverCSD(Settings(23, 23, 8, "csdWaterBeam", nPN=3))
    p, keep = s.problem_struct()
    lib = _lib.load()
    h = C.c_void_p()
    # one successful create/destroy first: module load and context set-up are not leaks
    _lib.check(lib.titus_create(C.byref(p), C.byref(h)), "titus_create")
    lib.titus_destroy(h)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for after in (1, 2, 7, 20, 33):
        _lib.check(lib.titus_debug_fail_alloc(after), "titus_debug_fail_alloc")
        h2 = C.c_void_p()
        rc = lib.titus_create(C.byref(p), C.byref(h2))
        _lib.check(lib.titus_debug_fail_alloc(0), "titus_debug_fail_alloc")
        if rc == 0:          # fewer allocations than `after`: nothing to inject
            lib.titus_destroy(h2)
            continue
        assert rc == 2 and "injected" in _lib.last_error(), (after, rc, _lib.last_error())
        assert not h2.value
        assert torch.cuda.mem_get_info()[0] == free0, after
    # the library still works afterwards
    out = s.run(_lib.TITUS_BUG_ADAPTIVE, max_steps=3)
    assert np.isfinite(out["dose"]).all()
