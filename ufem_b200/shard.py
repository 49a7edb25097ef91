"""Sharding of Monte Carlo samples across ranks (one process per GPU).

Samples are independent, so every rank solves its own contiguous range of
sample ids (seeded per id, so the ranges never overlap) and nothing crosses
ranks on the data path; the only collective is the max over ranks of a step
time, taken on the process group the caller set up (NCCL on GPUs, gloo in
the CPU tests).
"""
from __future__ import annotations


def rank_samples(rank: int, per_rank: int, first: int = 0) -> tuple[int, int]:
    """(first sample id, count) of rank `rank` when each rank takes `per_rank`."""
    if rank < 0 or per_rank < 0:
        raise ValueError("rank and per_rank must be non-negative")
    return first + rank * per_rank, per_rank


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (the value itself without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
