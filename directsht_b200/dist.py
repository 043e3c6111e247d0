"""Multi-GPU helpers: one process per GPU, independent work per rank.

The transform has no exchange step: point sets, maps and requests are independent, so N
GPUs run N shards with no collective on the data path.  The only collectives are the
timing and counter reductions of a benchmark (max of the per-rank device times, sums of the
work done), on whatever process group the caller initialised (NCCL on GPUs, gloo on CPUs).
"""
from __future__ import annotations

import os


def rank_world():
    """(rank, world size, local rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items, rank: int, world: int):
    """Round-robin shard of a list of independent work items (requests, transforms)."""
    return list(items[rank::world])


def reduce_scalar(value: float, op: str = "max", device=None) -> float:
    """max or sum of one float over the ranks of the default process group (identity when
    no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())
