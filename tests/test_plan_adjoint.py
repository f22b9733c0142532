"""Plan objective with voxel-density gradients (titus_b200.spots.plan_adjoint):
energy groups solved with their weighted inflow profile, the total dose and
both gradients summed over ranks. A linear stand-in transport model (dose =
diag(1/rho) B_E profile, its exact adjoint) replaces the GPU calls, so the
host algebra is checked against central finite differences, and the gloo
world-2/3 runs against the single process. The GPU adjoint itself is checked
in tests/test_gpu_adjoint.py."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from titus_b200.spots import partition, plan_adjoint

N = 40
SPOTS = [(2.0, 0.2), (3.0, 0.5), (2.0, 0.7), (5.0, 0.4), (3.0, 0.9), (8.0, 0.3)]
WEIGHTS = np.array([1.0, 0.5, 2.0, 1.5, 0.8, 1.2])


class StandIn:
    """Dose = diag(1/rho) B_E profile for beams of energy E."""

    def __init__(self, energy, rho):
        rng = np.random.default_rng(int(energy * 10))
        self.B = rng.uniform(0.0, 1.0, (N, N))
        self.rho = rho
        self.energy = energy

    def beam_profile(self, y0=None):
        c = np.arange(N) / N
        return np.exp(-((c - y0) / 0.1) ** 2)


def forward(sv, profile):
    return (sv.B @ profile) / sv.rho


def adjoint(sv, profile, djdd, every):
    dose = forward(sv, profile)
    grho = -dose / sv.rho * djdd
    gprof = sv.B.T @ (djdd / sv.rho)
    return dose, grho, gprof


def _problem():
    rho = np.linspace(0.5, 1.5, N)
    P = np.full(N, 20.0)
    mask = (np.arange(N) % 4 != 0).astype(float)
    return rho, P, mask


def _run(rho, w):
    _, P, mask = _problem()
    return plan_adjoint(lambda e: StandIn(e, rho), SPOTS, w, P, mask, forward=forward, adjoint=adjoint)


def test_gradients_match_finite_differences():
    rho, _, _ = _problem()
    J, gw, grho, D = _run(rho, WEIGHTS)
    assert J > 0
    h = 1e-6
    for s in range(len(SPOTS)):
        e = np.zeros(len(SPOTS))
        e[s] = h
        fd = (_run(rho, WEIGHTS + e)[0] - _run(rho, WEIGHTS - e)[0]) / (2 * h)
        assert fd == pytest.approx(gw[s], rel=1e-6)
    for c in (0, 7, 19, 33):
        e = np.zeros(N)
        e[c] = h
        fd = (_run(rho + e, WEIGHTS)[0] - _run(rho - e, WEIGHTS)[0]) / (2 * h)
        assert fd == pytest.approx(grho[c], rel=1e-6, abs=1e-9)


def test_groups_share_one_solve_per_energy():
    rho, P, mask = _problem()
    calls = []

    def fwd(sv, profile):
        calls.append(sv.energy)
        return forward(sv, profile)

    plan_adjoint(lambda e: StandIn(e, rho), SPOTS, WEIGHTS, P, mask, forward=fwd, adjoint=adjoint)
    assert sorted(calls) == [2.0, 3.0, 5.0, 8.0]


def test_bad_weights():
    rho, P, mask = _problem()
    with pytest.raises(ValueError):
        plan_adjoint(lambda e: StandIn(e, rho), SPOTS, WEIGHTS[:3], P, mask, forward=forward, adjoint=adjoint)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rho, _, _ = _problem()
        out.put((rank, _run(rho, WEIGHTS)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_over_energy_groups_gloo(world):
    rho, _, _ = _problem()
    J, gw, grho, D = _run(rho, WEIGHTS)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(r for r, _ in res) == list(range(world))
    assert sum(partition(4, world, r).size for r in range(world)) == 4
    for _, (J2, gw2, grho2, D2) in res:
        assert J2 == pytest.approx(J, rel=1e-13)
        np.testing.assert_allclose(gw2, gw, rtol=1e-12)
        np.testing.assert_allclose(grho2, grho, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(D2, D, rtol=1e-13)
