"""Host logic of multi-GPU runs: one process per GPU, each holding a full
replica of the index and answering its own shard of the query batches.

Queries are independent, so the path shards with no data-path collective:
rank r of N takes the batches ``shard(total_batches, r, N)`` of a workload
whose batches are generated from (seed, batch index) alone, so every rank
derives its shard without communication and the union of the shards is the
whole workload.  The only collectives are the timing ones: a barrier around
the timed region and the max of the per-rank times (whole-job throughput is
the total work over the slowest rank's time).
"""
from __future__ import annotations

import numpy as np


def shard(total: int, rank: int, world: int) -> range:
    """Contiguous, balanced split of range(total) over `world` ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def batch_seed(seed: int, batch: int) -> int:
    """Seed of one batch's queries (independent of the rank that runs it)."""
    return (seed * 1_000_003 + batch * 7919) % (2 ** 63)


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """Max of a per-rank float over the process group (x itself when alone)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: int, dist=None, device=None) -> int:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return int(x)
    import torch
    t = torch.tensor([int(x)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def shard_queries(sizes: np.ndarray, rank: int, world: int):
    """(batch indices, query offset of each, sizes) of this rank's shard of a
    batch list."""
    idx = np.asarray(list(shard(len(sizes), rank, world)), dtype=np.int64)
    offs = np.concatenate([[0], np.cumsum(sizes)])[:-1]
    return idx, offs[idx], np.asarray(sizes)[idx]
