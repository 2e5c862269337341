"""Multi-process host logic on CPU (two gloo ranks): the whole-job step time
is the slowest rank's, and a ragged batch splits into balanced, disjoint,
complete instance ranges without any exchange."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import bench
    from socu_b200.problems import ragged_shapes
    from socu_b200.ragged import shard_instances
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.0 + rank, world, "cpu")
        N, n, _ = ragged_shapes(0, 4096)
        lo, hi = shard_instances(N, n, world, rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, (lo, hi))
        out[rank] = (t, gathered)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert [res[r][0] for r in range(world)] == [2.0, 2.0]   # the slowest rank's time everywhere
    ranges = res[0][1]
    assert ranges == res[1][1]
    assert ranges[0][0] == 0 and ranges[-1][1] == 4096
    assert all(ranges[r][1] == ranges[r + 1][0] for r in range(world - 1))


@pytest.mark.parametrize("world", [1, 3, 8])
def test_shards_balance_the_factor_work(world):
    from socu_b200.problems import ragged_shapes
    from socu_b200.ragged import shard_instances
    N, n, _ = ragged_shapes(0, 4096)
    work = N.astype(float) * n.astype(float) ** 3
    shards = [shard_instances(N, n, world, r) for r in range(world)]
    assert shards[0][0] == 0 and shards[-1][1] == 4096
    assert all(shards[r][1] == shards[r + 1][0] for r in range(world - 1))
    per = np.array([work[lo:hi].sum() for lo, hi in shards])
    assert per.max() <= work.sum() / world + work.max()
