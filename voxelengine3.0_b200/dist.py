"""Multi-GPU plumbing for the replica mode: one process per GPU, no collective
on the data path.

Frames, views and requests are independent; every rank holds its own copy of
the octree and its own radiance cache and renders its share of the work.  The
only communication is for measurement: a barrier around the timed region and
the max (time) / sum (rays) over ranks.
"""
from __future__ import annotations

import datetime
import os
from typing import List, Optional, Sequence


def env_rank() -> tuple:
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0, device: Optional[int] = None):
    """Initialises torch.distributed when WORLD_SIZE > 1; returns the module or None."""
    rank, world, local = env_rank()
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist

    if backend == "nccl":
        torch.cuda.set_device(local if device is None else device)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def frame_assignment(n_steps: int, rank: int, world: int, period: int) -> List[int]:
    """Orbit frames of one rank: rank r renders frames r, r+world, r+2*world,
    ... (mod the orbit period) — equal work per rank (weak scaling)."""
    return [(rank + world * i) % period for i in range(n_steps)]


def split_evenly(items: Sequence, rank: int, world: int) -> list:
    """Contiguous near-equal shares of a work list (views or requests)."""
    n = len(items)
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return list(items[lo:hi])


def _reduce(value: float, dist, op, device=None) -> float:
    if dist is None:
        return float(value)
    import torch

    backend = dist.get_backend()
    dev = device if device is not None else ("cuda" if backend == "nccl" else "cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None:
        return float(value)
    return _reduce(value, dist, dist.ReduceOp.MAX, device)


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None:
        return float(value)
    return _reduce(value, dist, dist.ReduceOp.SUM, device)


def barrier(dist=None) -> None:
    if dist is not None:
        dist.barrier()


def shutdown(dist=None) -> None:
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
