"""Independent frames across ranks (one process per GPU).

The reference reconstructs one frame per process, frame after frame
(src/QTGUI/rihvr.cpp:2414-2905 launches sparse-inverse-recon per hologram).
Frames of a time series are independent, so N GPUs take N disjoint sets of
frames with no data exchange; torch.distributed is used only to agree on
timing (barrier, max over ranks).
"""
from __future__ import annotations


def rank_frames(n_frames: int, world_size: int, rank: int) -> list:
    """Contiguous block of frame indices for `rank` (sizes differ by at most 1)."""
    if world_size < 1 or not (0 <= rank < world_size) or n_frames < 0:
        raise ValueError("bad frame partition arguments")
    base, extra = divmod(n_frames, world_size)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def frame_seed(base_seed: int, frame: int) -> int:
    """Seed of synthetic frame `frame` of a series."""
    return int(base_seed) + int(frame)


def reduce_max(value: float, device=None) -> float:
    """Maximum of `value` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def weak_throughput(total_voxel_iterations: float, max_ms: float) -> float:
    """Whole-job voxel iterations per second, timed by the slowest rank."""
    if not max_ms > 0:
        raise ValueError("elapsed time must be positive")
    return total_voxel_iterations / (max_ms / 1e3)
