"""Model sharding across GPUs: one process per GPU, no collective on the data path.

Every trace (model, period) is independent, so a batch is split by model rows:
each rank solves a contiguous block of models on its own engine, and results
meet only where the caller wants them in one place (a gather of the output
blocks).  The timing reduction of the benchmark (max of the ranks' device
times, sum of their roots) is the only other exchange.

The functions take an initialised ``torch.distributed`` process group (NCCL on
GPUs, gloo on CPU); with ``world == 1`` they are plain pass-throughs.
"""
from __future__ import annotations

import numpy as np


def shard_rows(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block [start, stop) of ``n`` models owned by ``rank``.

    Blocks differ in size by at most one model and the lower ranks take the
    larger ones, so every model is owned by exactly one rank.
    """
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n < 0:
        raise ValueError("n must be non-negative")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_batch(batch: dict, rank: int, world: int) -> dict:
    """The rows of every ``[B, ...]`` array of ``batch`` that ``rank`` owns."""
    n = len(next(iter(batch.values())))
    start, stop = shard_rows(n, rank, world)
    return {k: v[start:stop] for k, v in batch.items()}


def _dist():
    import torch.distributed as dist
    return dist


def reduce_max(x: float, device=None) -> float:
    """Largest ``x`` over the ranks (device times: the job ends with its slowest rank)."""
    import torch
    dist = _dist()
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float, device=None) -> float:
    """Sum of ``x`` over the ranks (roots solved by the whole job)."""
    import torch
    dist = _dist()
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t)
    return float(t.item())


def gather_rows(block: np.ndarray, n: int, device=None):
    """Reassemble the per-rank output blocks of an ``n``-model batch on every rank.

    ``block`` holds this rank's rows (``shard_rows`` order); the result is the
    full ``[n, ...]`` array.  Blocks are padded to the largest block for the
    all-gather and trimmed afterwards, so uneven shards need no second round.
    """
    import torch
    dist = _dist()
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return np.asarray(block)
    world, rank = dist.get_world_size(), dist.get_rank()
    start, stop = shard_rows(n, rank, world)
    if block.shape[0] != stop - start:
        raise ValueError(f"rank {rank} holds {block.shape[0]} rows, its shard has {stop - start}")
    width = shard_rows(n, 0, world)[1]
    pad = np.zeros((width,) + block.shape[1:], dtype=block.dtype)
    pad[: block.shape[0]] = block
    local = torch.from_numpy(pad).to(device) if device is not None else torch.from_numpy(pad)
    parts = [torch.empty_like(local) for _ in range(world)]
    dist.all_gather(parts, local)
    out = []
    for r, part in enumerate(parts):
        s, e = shard_rows(n, r, world)
        out.append(part.cpu().numpy()[: e - s])
    return np.concatenate(out, axis=0)
