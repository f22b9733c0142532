"""Spot-sharded pencil-beam plans (titus_b200.spots): round-robin partition,
weighted total dose by one SUM all-reduce, and the spot-weight gradient of the
plan objective. Multi-rank paths run as gloo ranks on CPU with a stand-in
per-spot dose; the CUDA path is checked on one GPU against the batched solver.
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from titus_b200.spots import partition, plan_dose, plan_objective

N_CELLS = 50
SPOTS = [(0.1 + 0.02 * i, 0.2 + 0.05 * i) for i in range(7)]
WEIGHTS = np.linspace(0.5, 2.0, len(SPOTS))


class FakeSolver:
    n = N_CELLS


def fake_solve(solver, spots, method, team_ctas, max_steps):
    """Stand-in per-spot dose: a Gaussian in the cell index set by (energy, y0)."""
    c = np.arange(solver.n)
    return np.array([e * 100 * np.exp(-((c - y * solver.n) / 6.0) ** 2) for e, y in spots])


def serial_reference():
    D_s = fake_solve(FakeSolver(), SPOTS, "bug", 1, 0)
    D = WEIGHTS @ D_s
    P = np.full(N_CELLS, 3.0)
    mask = (np.arange(N_CELLS) % 3 != 0).astype(float)
    res = mask * (D - P)
    return D_s, D, P, mask, float(res @ (D - P)), 2.0 * D_s @ res


def test_partition_covers_every_spot_once():
    for ns in (0, 1, 5, 16, 17):
        for world in (1, 2, 3, 8):
            parts = [partition(ns, world, r) for r in range(world)]
            allidx = np.sort(np.concatenate(parts))
            np.testing.assert_array_equal(allidx, np.arange(ns))
            sizes = [p.size for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        partition(4, 2, 2)
    with pytest.raises(ValueError):
        partition(4, 0, 0)


def test_single_process_matches_serial():
    D_s, D, P, mask, J, g = serial_reference()
    tot, idx, local = plan_dose(FakeSolver(), SPOTS, WEIGHTS, solve=fake_solve)
    np.testing.assert_array_equal(idx, np.arange(len(SPOTS)))
    np.testing.assert_allclose(tot, D, rtol=1e-14)
    J2, g2, D2 = plan_objective(FakeSolver(), SPOTS, WEIGHTS, P, mask, solve=fake_solve)
    assert J2 == pytest.approx(J, rel=1e-13)
    np.testing.assert_allclose(g2, g, rtol=1e-13)
    # the objective is quadratic in w: central differences are exact up to rounding
    h = 1e-3
    for s in range(len(SPOTS)):
        wp, wm = WEIGHTS.copy(), WEIGHTS.copy()
        wp[s] += h
        wm[s] -= h
        Jp = plan_objective(FakeSolver(), SPOTS, wp, P, mask, solve=fake_solve)[0]
        Jm = plan_objective(FakeSolver(), SPOTS, wm, P, mask, solve=fake_solve)[0]
        assert (Jp - Jm) / (2 * h) == pytest.approx(g[s], rel=1e-8)


def test_bad_arguments():
    with pytest.raises(ValueError, match="weights"):
        plan_dose(FakeSolver(), SPOTS, WEIGHTS[:3], solve=fake_solve)
    with pytest.raises(ValueError, match="prescription"):
        plan_objective(FakeSolver(), SPOTS, WEIGHTS, np.zeros(3), solve=fake_solve)

    def wrong_shape(solver, spots, m, t, k):
        return np.zeros((len(spots), solver.n + 1))

    with pytest.raises(ValueError, match="solve returned"):
        plan_dose(FakeSolver(), SPOTS, WEIGHTS, solve=wrong_shape)


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
        _, _, P, mask, _, _ = serial_reference()
        tot, idx, local = plan_dose(FakeSolver(), SPOTS, WEIGHTS, solve=fake_solve)
        J, g, D = plan_objective(FakeSolver(), SPOTS, WEIGHTS, P, mask, solve=fake_solve)
        out.put((rank, tot, idx, J, g))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_plan_gloo(world):
    D_s, D, P, mask, J, g = serial_reference()
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
    seen = []
    for rank, tot, idx, J2, g2 in res:
        np.testing.assert_array_equal(idx, partition(len(SPOTS), world, rank))
        seen += list(idx)
        np.testing.assert_allclose(tot, D, rtol=1e-13)      # every rank holds the total dose
        assert J2 == pytest.approx(J, rel=1e-13)
        np.testing.assert_allclose(g2, g, rtol=1e-13)      # and the whole gradient
    assert sorted(seen) == list(range(len(SPOTS)))


@pytest.mark.gpu
def test_plan_on_gpu_matches_batched_solve():
    from titus_b200 import Settings, SolverCSD, SolveBatchedPencilBeams

    spots = [(0.1, 0.5), (0.22, 0.4), (0.15, 0.55)]
    w = np.array([1.0, 0.5, 2.0])
    sv = SolverCSD(Settings(31, 31, 12, "csdPhantom", nPN=5))
    D_s = SolveBatchedPencilBeams(sv, spots, "bug", team_ctas=4)[0]
    tot, idx, local = plan_dose(sv, spots, w, team_ctas=4)
    np.testing.assert_array_equal(local, D_s)          # same launch, same spots: bitwise
    np.testing.assert_allclose(tot, w @ D_s, rtol=1e-14)
    P = np.full(sv.n, 0.5 * tot.max())
    J, g, D = plan_objective(sv, spots, w, P, team_ctas=4)
    res = D - P
    assert J == pytest.approx(float(res @ res), rel=1e-13)
    np.testing.assert_allclose(g, 2.0 * D_s @ res, rtol=1e-12)
