"""Replica helpers for running the path on several GPUs of one node.

The dedispersion path shards without any data exchange (beams, chunks and
DM ranges are independent), so N GPUs run N independent replicas: each rank
takes a contiguous share of the units; timings are combined as the maximum
over ranks.  torch.distributed (NCCL on GPUs, gloo on CPU) carries only
these scalars.
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [lo, hi) share of n units for `rank` of `world`."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _reduce(value: float, op) -> float:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float) -> float:
    return _reduce(value, dist.ReduceOp.MAX)


def sum_over_ranks(value: float) -> float:
    return _reduce(value, dist.ReduceOp.SUM)


def barrier() -> None:
    """Barrier across ranks (no-op without an initialised process group)."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
