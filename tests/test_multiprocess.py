"""Model sharding across ranks (gloo, world size 2, CPU).

The multi-GPU path shards models over one process per GPU and exchanges only
timing scalars and, when asked, the output blocks; these tests run that host
logic on two CPU ranks.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from modisp_b200 import sharding


def test_shard_rows_partition():
    for n in (0, 1, 7, 10_000, 10_001):
        for world in (1, 2, 3, 8):
            blocks = [sharding.shard_rows(n, r, world) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            for (s0, e0), (s1, e1) in zip(blocks, blocks[1:]):
                assert e0 == s1
            sizes = [e - s for s, e in blocks]
            assert max(sizes) - min(sizes) <= 1
            assert sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        sharding.shard_rows(10, 2, 2)
    with pytest.raises(ValueError):
        sharding.shard_rows(-1, 0, 1)


def test_shard_batch_rows():
    batch = {"thickness": np.arange(10.).reshape(5, 2), "vp": np.arange(5.)}
    a = sharding.shard_batch(batch, 0, 2)
    b = sharding.shard_batch(batch, 1, 2)
    assert a["vp"].tolist() == [0., 1., 2.] and b["vp"].tolist() == [3., 4.]
    assert np.array_equal(np.concatenate([a["thickness"], b["thickness"]]), batch["thickness"])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, queue):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        start, stop = sharding.shard_rows(n, rank, world)
        # each rank "solves" its own block: rows of a [n, 3, 4] result
        full = np.arange(n * 12, dtype=np.float64).reshape(n, 3, 4)
        block = full[start:stop].copy()
        gathered = sharding.gather_rows(block, n)
        ms = sharding.reduce_max(10.0 + rank)
        roots = sharding.reduce_sum(stop - start)
        queue.put((rank, bool(np.array_equal(gathered, full)), ms, roots))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [9, 10])
def test_two_rank_gather_and_timing_reduction(n):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, same, ms, roots in results:
        assert same, f"rank {rank} gathered a different batch"
        assert ms == 11.0          # max over ranks
        assert roots == n          # every model counted once
