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


def _rank_arms(rank, world, port, out):
    """The bench's post-measurement reductions with rank-dependent timings;
    rank 0 then leaves no collective pending (the others have returned)."""
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    mx = bench.max_over_ranks_fn(world, dist, "cpu")
    main_arm = {"ms_per_step": 4.0 + rank, "pair_ms": 3.9 + rank}
    other = {"ms_per_step": 8.0 + 2 * rank, "pair_ms": 7.9 + 2 * rank}
    bench.arms_over_ranks(mx, main_arm, other)
    dist.barrier()
    e2e = bench.e2e_over_ranks(mx, world, 1000, {"ms_per_call": 5.0 + 0.5 * rank, "value": 0.0})
    dist.barrier()
    if rank != 0:
        dist.destroy_process_group()
        return
    out[0] = (main_arm, other, e2e)
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_post_measurement_reductions_gloo(world):
    out = mp.Manager().dict()
    mp.spawn(_rank_arms, args=(world, _free_port(), out), nprocs=world, join=True)
    main_arm, other, e2e = out[0]
    w = world - 1
    assert main_arm == {"ms_per_step": 4.0 + w, "pair_ms": 3.9 + w}
    assert other == {"ms_per_step": 8.0 + 2 * w, "pair_ms": 7.9 + 2 * w}
    assert e2e["ms_per_call"] == 5.0 + 0.5 * w
    assert abs(e2e["value"] - world * 1e6 / ((5.0 + 0.5 * w) * 1e-3) / 1e9) < 1e-12


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


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_ensemble_cluster_shards(world):
    """bench.py --ensemble under torchrun shares the clusters out over the
    GPUs: every cluster on exactly one rank, the same assignment on every
    rank, per-rank work (sum of N^2) within one cluster's work of each other."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(3)
    sizes = np.exp(rng.uniform(np.log(256), np.log(8192), 512)).astype(np.int32)
    shards = [bench.shard_clusters(sizes, world, r) for r in range(world)]
    allc = np.sort(np.concatenate(shards))
    assert np.array_equal(allc, np.arange(sizes.size))
    assert all(np.array_equal(s, bench.shard_clusters(sizes, world, r)) for r, s in enumerate(shards))
    load = [float((sizes[s].astype(np.float64) ** 2).sum()) for s in shards]
    assert max(load) - min(load) <= float(sizes.max()) ** 2
