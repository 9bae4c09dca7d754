"""Multi-GPU host logic: rays shard by view, one gradient all-reduce per step.

Rays are independent, so every rank holds the whole scene and traces its own share of
the views; the forward needs no communication. The per-ellipsoid gradients are then
summed across ranks with ONE all-reduce over a flat bucket that holds all of them (NCCL on
GPUs, gloo on CPU).

Each rank's gradients are clipped by its own backward before the sum (as
fast_ellipsoid_splinetracer.py:204-219 clips per call), so the sum equals the sum of
per-view trace_rays calls, the reference's semantics for several views; it is not the
clip of the summed gradient.
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


def allreduce_gradients(tensors: Iterable[torch.Tensor], group=None, bucket: torch.Tensor | None = None) -> None:
    """Sums the gradient tensors over all ranks, in place, with one all-reduce.

    The tensors (same shapes, dtype and device on every rank, None entries skipped) are
    packed into one flat bucket, summed in a single collective and unpacked again.
    bucket: optional preallocated flat buffer of at least the total element count (kept
    across steps, e.g. for CUDA-graph capture).
    """
    ts = [t for t in tensors if t is not None]
    if not ts:
        return
    dtype, device = ts[0].dtype, ts[0].device
    for t in ts:
        if t.dtype != dtype or t.device != device:
            raise ValueError("allreduce_gradients: all tensors must share dtype and device")
    total = sum(t.numel() for t in ts)
    if bucket is None:
        bucket = torch.empty(total, dtype=dtype, device=device)
    elif bucket.numel() < total or bucket.dtype != dtype or bucket.device != device:
        raise ValueError("allreduce_gradients: bucket too small or of another dtype/device")
    flat = bucket[:total]
    off = 0
    for t in ts:
        n = t.numel()
        flat[off:off + n].copy_(t.reshape(-1))
        off += n
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for t in ts:
        n = t.numel()
        t.copy_(flat[off:off + n].view_as(t))
        off += n


def max_over_ranks(value: float, device, group=None) -> float:
    """The slowest rank's time: what a multi-GPU step costs."""
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
