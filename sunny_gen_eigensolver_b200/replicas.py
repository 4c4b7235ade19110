"""Multi-GPU execution of the batched solve: replicas, no collective.

Every matrix is independent, so N GPUs run N replicas of the solver over
their own slices of the work (one process per GPU, torch.distributed only
for the timing barrier and the max-over-ranks reduction of elapsed time).
There is no exchange step on the data path and therefore no NCCL traffic in
the timed region beyond two scalar reductions.
"""
from __future__ import annotations

from typing import Tuple


def partition(total: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous slice [start, stop) of `total` items for `rank` out of
    `world` (strong scaling); sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError("bad partition arguments")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed of rank `rank`'s inputs in weak scaling (each rank its own batch)."""
    return int(base_seed) + 1000003 * int(rank)


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks of the default process group (the
    value itself when torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None) -> None:
    """Barrier over all ranks through a tiny all-reduce (works for gloo and
    NCCL alike), then a device synchronise when `device` is a CUDA device."""
    import torch
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        t = torch.zeros(1, device=device)
        dist.all_reduce(t)
    if device is not None and torch.device(device).type == "cuda":
        torch.cuda.synchronize(device)
