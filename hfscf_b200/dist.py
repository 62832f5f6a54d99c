"""Multi-process plumbing for the bench and the batched mode (one process per GPU).

The two-electron path shards without any data-path collective: independent
molecules of a batch are split across ranks (replicas), and every rank of a
single-molecule run does its own full build.  The only collective is the
max-over-ranks of the timed region.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a float over all ranks (identity without a process group)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(n_items: int, rank: int, world: int) -> list[int]:
    """Items of this rank when n_items independent objects are dealt round-robin."""
    return list(range(rank, n_items, world))
