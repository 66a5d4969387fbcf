"""Multi-GPU mode of bench.py is replicas only: every rank times its own
independent system and the whole-job value is ranks x N^2 / (slowest rank's
step time).  The aggregation runs here on CPU ranks over gloo."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mx = bench.max_over_ranks_fn(world, dist, "cpu")
    ms = mx(times[rank])
    out[rank] = (ms, bench.replica_value(world, 65536.0 ** 2, ms))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_replica_aggregation_gloo(world):
    times = [4.5 + 0.25 * r for r in range(world)]
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), times, out), nprocs=world, join=True)
    slowest = max(times)
    expect = world * 65536.0 ** 2 / (slowest * 1e-3) / 1e9
    for r in range(world):
        ms, v = out[r]
        assert ms == slowest and abs(v - expect) < 1e-9 * expect


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks_fn(1, None, "cpu")(3.25) == 3.25
    assert bench.replica_value(1, 1e9, 1000.0) == 1.0
