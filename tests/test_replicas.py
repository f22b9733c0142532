"""Multi-rank aggregation of replica runs (bench.py --gpus N), on CPU with gloo.

Each rank reports its own device time; the whole-job throughput uses the
slowest rank (max over ranks), identical on every rank.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from titus_b200.replicas import replica_throughput

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        value, t = replica_throughput(3, 1.0 + rank, world)   # rank r took 1 + r seconds for 3 solves
        out.put((rank, value, t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replica_throughput_gloo(world):
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
    t_max = 1.0 + (world - 1)
    for rank, value, t in res:
        assert t == pytest.approx(t_max)
        assert value == pytest.approx(world * 3 / t_max)


def test_single_process_identity():
    from titus_b200.replicas import replica_throughput

    value, t = replica_throughput(2, 4.0, 1)
    assert t == 4.0 and value == 0.5
