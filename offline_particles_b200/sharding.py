"""Particle sharding across GPUs: one process per GPU, no data-path collective.

Particles never interact, so a release splits into contiguous shards, one per
rank; each rank advances its shard on its own GPU with the fields replicated.
The only collectives are for bookkeeping: the maximum of per-rank timings and
gathering results on rank 0 (NCCL on GPUs, gloo on CPU).
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def shard_bounds(n_total: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's shard: sizes differ by at most one, lower ranks first."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    if n_total < 0:
        raise ValueError("negative particle count")
    base, extra = divmod(n_total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard(arrays, rank: int, world: int):
    """The rank's slice of each equal-length array."""
    arrays = list(arrays)
    n = len(arrays[0])
    if any(len(a) != n for a in arrays):
        raise ValueError("arrays differ in length")
    lo, hi = shard_bounds(n, rank, world)
    return [a[lo:hi] for a in arrays]


def _device_for_backend() -> torch.device:
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float) -> float:
    """The maximum of ``value`` over all ranks (``value`` itself without a process group)."""
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float) -> float:
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_shards(array: np.ndarray) -> np.ndarray | None:
    """Concatenate every rank's shard on rank 0 in rank order (None on the other ranks)."""
    if not dist.is_available() or not dist.is_initialized():
        return np.asarray(array)
    world = dist.get_world_size()
    parts = [None] * world if dist.get_rank() == 0 else None
    dist.gather_object(np.asarray(array), parts, dst=0)
    if dist.get_rank() != 0:
        return None
    return np.concatenate(parts)
