"""Host-side helpers for rendering on several GPUs (one process per GPU).

The path shards with no exchange inside a frame: every rank renders whole
frames of the progressive sequence with disjoint Halton samples (rank r of N
renders frame step * N + r + 1 at each step, so the ranks together render
frames 1, 2, 3, ... once each), and one all-reduce per step combines them.
The combined image is the mean of the N frames, which is what accumulating
them one after another (ymrt_accumulate) gives. Times are reduced with the
maximum over ranks.
"""
from __future__ import annotations

import os
from datetime import timedelta


def env():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> None:
    """Joins the process group (rendezvous on 127.0.0.1 unless MASTER_ADDR is set)."""
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def frame_index(step: int, rank: int, world: int) -> int:
    """The progressive frame rank `rank` renders at `step` (1-based frames)."""
    return step * world + rank + 1


def combine_frames(image, world: int, mean: bool = True):
    """All-reduces one frame per rank in place: the sum, or (mean=True) the
    mean of the N frames."""
    import torch.distributed as dist
    if world > 1:
        dist.all_reduce(image)
    if mean and world > 1:
        image.div_(float(world))
    return image


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of a per-rank number (e.g. a timed region in ms)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
