"""Multi-GPU host logic: rays shard by view, one gradient all-reduce per step.

Rays are independent, so every rank holds the whole scene and traces its own share of
the views; the forward needs no communication. The per-ellipsoid gradients are then
summed across ranks with one all-reduce per tensor (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

from typing import Iterable, Sequence

import torch
import torch.distributed as dist


def view_shard(views: Sequence, rank: int, world: int) -> list:
    """The views rank `rank` traces: round robin, so uneven view sizes spread out."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} for world size {world}")
    return list(views[rank::world])


def allreduce_gradients(tensors: Iterable[torch.Tensor], group=None) -> None:
    """Sums each gradient tensor over all ranks, in place and in the same order on every rank."""
    for t in tensors:
        if t is not None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def max_over_ranks(value: float, device, group=None) -> float:
    """The slowest rank's time: what a multi-GPU step costs."""
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
