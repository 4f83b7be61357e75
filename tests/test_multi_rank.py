"""Batch sharding across ranks (CPU, gloo, world size 2).

Every member of a batch is independent (reference src/batched_1d_plan.hpp:
85-128 splits the batch over OpenMP threads the same way), so a batch is
split into contiguous shards with no data-path collective.  Here two gloo
ranks each transform their shard with the CPU oracle standing in for the
device, and the gathered shards must equal the whole-batch result.
"""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

import plfft


@pytest.mark.parametrize("howmany,world", [(4096, 2), (7, 2), (1, 2), (5, 3), (0, 2)])
def test_shard_range_partitions_batch(howmany, world):
    spans = [plfft.shard_range(howmany, world, r) for r in range(world)]
    covered = []
    for first, cnt in spans:
        assert cnt >= 0
        covered.extend(range(first, first + cnt))
    assert covered == list(range(howmany))
    sizes = [c for _, c in spans]
    assert max(sizes) - min(sizes) <= 1


def test_shard_range_rejects_bad_rank():
    with pytest.raises(ValueError):
        plfft.shard_range(10, 2, 2)


def _worker(rank, world, port, n, howmany, q):
    import torch
    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(123)  # every rank sees the same global batch
    x = rng.uniform(-1, 1, (howmany, n)) + 1j * rng.uniform(-1, 1, (howmany, n))
    first, cnt = plfft.shard_range(howmany, world, rank)
    y = oracle.c2c(x[first:first + cnt], -1)
    mine = torch.from_numpy(np.ascontiguousarray(y.view(np.float64)))
    # gather variable-size shards: pad to the largest shard
    most = max(plfft.shard_range(howmany, world, r)[1] for r in range(world))
    pad = torch.zeros((most, 2 * n), dtype=torch.float64)
    pad[:cnt] = mine.reshape(cnt, 2 * n)
    out = [torch.zeros_like(pad) for _ in range(world)]
    dist.all_gather(out, pad)
    if rank == 0:
        parts = [out[r][: plfft.shard_range(howmany, world, r)[1]].numpy() for r in range(world)]
        full = np.concatenate(parts).view(np.complex128)
        q.put(float(np.abs(full - oracle.c2c(x, -1)).max()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_batch_shards_match_whole_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, 64, 37, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert q.get(timeout=5) == 0.0


def _bench_worker(rank, world, port, q):
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # each rank's own step count and timings; the bench line must use the maximum
    steps = bench.max_over_ranks(dist, [200 + 50 * rank], "cpu")
    ms = bench.max_over_ranks(dist, [1.5 - rank, 0.25 * (rank + 1), 0.0], "cpu")
    q.put((rank, steps, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_max_over_ranks_two_gloo_ranks():
    """bench.py's multi-rank reduction (one process per GPU under torchrun):
    every rank times the same step count and reports the slowest rank's time."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31500 + os.getpid() % 2000
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    for _, steps, ms in got:
        assert steps == [250.0]
        assert ms == [1.5, 0.5, 0.0]


def test_bench_max_over_ranks_single_process():
    import bench

    assert bench.max_over_ranks(None, [3, 1.5], "cpu") == [3.0, 1.5]
