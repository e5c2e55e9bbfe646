"""Multi-GPU plumbing for whole-image sharding (one process per GPU).

The decomposition is independent per image (and per pixel), so N GPUs run N
independent shares of the images with no collective on the data path; the
only collectives are the timing and count reductions below, which take the
maximum (time) or the sum (pixels) over ranks. Backend: NCCL on GPUs, gloo on
CPU (tests).
"""
from __future__ import annotations

import os


def env() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the launcher's environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def shard(items: list, rank: int, world: int) -> list:
    """Round-robin share of `items` for `rank` (every item on exactly one rank)."""
    return items[rank::world]


def reduce_max(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def throughput(pixels_per_rank: float, ms_per_rank: float, device=None) -> float:
    """Whole-job pixels/s: pixels of all ranks over the slowest rank's time."""
    return reduce_sum(pixels_per_rank, device) / (reduce_max(ms_per_rank, device) / 1e3)
