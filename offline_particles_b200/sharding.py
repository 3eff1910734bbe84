"""Particle sharding across GPUs: one process per GPU, no data-path collective.

Particles never interact, so a release splits into contiguous shards, one per
rank; each rank advances its shard on its own GPU with the fields replicated.
The only collectives are for bookkeeping: the maximum of per-rank timings and
gathering results on rank 0 (NCCL on GPUs, gloo on CPU).
"""

from __future__ import annotations

import datetime
import os
import time

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


class Ranks:
    """The ranks of a one-process-per-GPU job, as ``torch.distributed.run`` starts it.

    Reads ``RANK``, ``WORLD_SIZE`` and ``LOCAL_RANK`` from the environment
    (rendezvous through ``MASTER_ADDR`` / ``MASTER_PORT``) and, with more than
    one rank, joins the process group: NCCL when CUDA is there, else gloo.
    ``timeout_s`` bounds every collective, so a rank that dies or never
    arrives ends the others' next collective with an error instead of a hang.
    Every rank must call the same collectives in the same order.
    """

    def __init__(self, backend: str | None = None, timeout_s: float = 300.0) -> None:
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        if not 0 <= self.rank < self.world:
            raise ValueError(f"RANK {self.rank} out of range for WORLD_SIZE {self.world}")
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if self.backend == "nccl":
            torch.cuda.set_device(self.local)
        self.joined = False
        if self.world > 1 or backend is not None:
            dist.init_process_group(self.backend, rank=self.rank, world_size=self.world,
                                    timeout=datetime.timedelta(seconds=timeout_s))
            self.joined = True

    @property
    def device(self) -> torch.device:
        return torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")

    def barrier(self) -> None:
        if self.joined:
            if self.backend == "nccl":
                dist.barrier(device_ids=[self.local])
            else:
                dist.barrier()

    def max(self, value: float) -> float:
        return max_over_ranks(value)

    def sum(self, value: float) -> float:
        return sum_over_ranks(value)

    def gather(self, array) -> np.ndarray | None:
        """Every rank's array concatenated on rank 0 in rank order (None on the other ranks)."""
        if isinstance(array, torch.Tensor):
            array = array.detach().cpu().numpy()
        return gather_shards(np.asarray(array))

    def timed_ms(self, work) -> float:
        """Run ``work()`` on every rank between two barriers, with the device drained on both sides, and
        return the slowest rank's time in ms: CUDA events on the current stream on a GPU, the host clock
        otherwise."""
        cuda = self.device.type == "cuda"
        self.barrier()
        if cuda:
            torch.cuda.synchronize(self.device)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            work()
            e.record()
            torch.cuda.synchronize(self.device)
            ms = s.elapsed_time(e)
        else:
            t0 = time.perf_counter()
            work()
            ms = (time.perf_counter() - t0) * 1e3
        self.barrier()
        return self.max(ms)

    def close(self) -> None:
        if self.joined:
            dist.destroy_process_group()
            self.joined = False
