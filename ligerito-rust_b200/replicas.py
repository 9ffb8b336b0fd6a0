"""Replica scheduling across GPUs (one process per GPU).

A single Ligerito proof does not shard: its leaves are rows across all
columns, so splitting one proof needs an all-to-all transpose of the whole
encoded matrix.  Independent proofs do: each rank proves its own share with
no data-path collective, and only timings / counts are reduced.
"""
from __future__ import annotations

from typing import List, Sequence


def shard(items: Sequence, rank: int, world: int) -> List:
    """Round-robin share of `items` for `rank` (stable, covers every item once)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return [x for i, x in enumerate(items) if i % world == rank]


def reduce_max(value: float, group=None) -> float:
    """Max of a scalar over all ranks (torch.distributed; identity without it)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def reduce_sum(value: float, group=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
