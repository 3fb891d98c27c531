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


def _search_rank(rank, world, port, queue):
    """One rank of a sharded batch: the oracle (the CPU restatement of the
    search) stands in for the device engine, so the test runs without a GPU;
    every rank runs only its round-robin share and rank 0 gathers the
    results, as `bench.py --workload batch` does on N GPUs."""
    sys.path.insert(0, ROOT)
    import bench
    from gagp_b200 import abi, task as T, workloads as W
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = [(64, 2, s) for s in range(5)]
        mine = bench.shard(list(range(len(specs))), rank, world)
        out = {}
        for i in mine:
            p, g, seed = specs[i]
            lt = T.from_files(W.polynomial(population=p, generations=g, seed=seed))
            r = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings)
            out[i] = {"history": r["history"], "best": r["final"][0]}
        gathered = [None] * world
        dist.all_gather_object(gathered, out)
        queue.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def test_two_ranks_run_their_share_of_searches():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = 31500 + os.getpid() % 2000
    procs = [ctx.Process(target=_search_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    merged = {}
    for part in results[0][1]:
        assert not set(part) & set(merged)  # every search ran on one rank only
        merged.update(part)
    assert sorted(merged) == list(range(5))
    assert results[0][1] == results[1][1]  # both ranks hold the same gathered view
    # a search's result does not depend on the rank that ran it
    sys.path.insert(0, ROOT)
    from gagp_b200 import abi, task as T, workloads as W
    from oracle import oracle
    lt = T.from_files(W.polynomial(population=64, generations=2, seed=3))
    alone = oracle.search(abi.GrammarBlob(lt.tables), lt.cases, lt.settings)
    assert merged[3] == {"history": alone["history"], "best": alone["final"][0]}
