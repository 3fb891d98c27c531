"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks (world size 2).

A search does not shard (placement is sequential over the population), so
several GPUs run independent searches: batches are split round-robin over
the ranks and the whole-job figures are the max of the ranks' times and the
sum of their units.  These tests run that split and that exchange on two
processes over gloo, without a GPU."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, queue):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        items = list(range(13))
        mine = bench.shard(items, rank, world)
        seconds = 1.5 + rank  # rank 1 is the slower one
        secs, total = bench.combine_ranks(dist, seconds, len(mine), device="cpu")
        queue.put((rank, mine, secs, total))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_and_combine():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = [r[1] for r in results]
    assert sorted(shards[0] + shards[1]) == list(range(13))  # disjoint and complete
    assert not set(shards[0]) & set(shards[1])
    for _, _, secs, total in results:
        assert secs == pytest.approx(2.5)  # max over ranks
        assert total == 13                 # sum over ranks
