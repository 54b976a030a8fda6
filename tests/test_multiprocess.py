"""The N > 1 host paths of bench.py on CPU: two gloo ranks on 127.0.0.1.

A plain fit does not shard (replicas only); a cross-validation grid shards by
instance with no data-path collective.  What the ranks do share is the timing
and the counts: the whole-job number is the units of all ranks over the
slowest rank's device time.  These tests run that host logic with the gloo
backend in place of NCCL."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # replicas: per-rank device seconds and coordinate updates
        secs = [1.5 + rank, 0.25 * (rank + 1)]
        mx = bench.allreduce(secs, dist.ReduceOp.MAX, world)
        sm = bench.allreduce([1000.0 * (rank + 1)], dist.ReduceOp.SUM, world)
        # the cross-validation grid's instance shards
        shard = bench.cv_shard(200, world, rank)
        shards = [None] * world
        dist.all_gather_object(shards, shard.tolist())
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.array([mx[0], mx[1], sm[0]], dtype=np.float64))
        if rank == 0:
            np.save(os.path.join(out_dir, "shards.npy"), np.array(sum(shards, []), dtype=np.int64))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_reduce_and_shard(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        mx0, mx1, tot = np.load(tmp_path / f"r{r}.npy")
        assert mx0 == 2.5 and mx1 == 0.5  # max over ranks
        assert tot == 3000.0              # sum over ranks
    shards = np.load(tmp_path / "shards.npy")
    assert sorted(shards.tolist()) == list(range(200))  # every instance exactly once


def test_cv_shard_round_robin():
    import bench
    parts = [bench.cv_shard(11, 3, r) for r in range(3)]
    assert [p.tolist() for p in parts] == [[0, 3, 6, 9], [1, 4, 7, 10], [2, 5, 8]]
