"""Shot-parallel RTM across GPUs: host-side logic.

Shots are independent units of the RTM workload; their images add up (the
reference computes one shot per run and has no shot-level parallelism).
With one process per GPU, each rank takes every world_size-th shot of the
stream and the per-shot images are stacked with one all-reduce (NCCL on GPUs,
gloo on CPU).  Nothing here touches the kernels.
"""
from __future__ import annotations

from typing import Callable, Iterable, List, Optional


def shots_for_rank(n_shots: int, world_size: int, rank: int) -> List[int]:
    """Round-robin assignment: shot s goes to rank s % world_size."""
    if world_size < 1 or not (0 <= rank < world_size) or n_shots < 0:
        raise ValueError("bad shot partition")
    return list(range(rank, n_shots, world_size))


def stack(image, dist=None, group=None):
    """Sum a per-rank image tensor over all ranks in place (no-op when single)."""
    if dist is not None and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(image, op=dist.ReduceOp.SUM, group=group)
    return image


def run_shot_stream(n_shots: int, run_one: Callable[[int], "object"], zeros_like_image: Callable[[], "object"],
                    dist=None, group=None, steps: Optional[Iterable[int]] = None):
    """Run this rank's shots with ``run_one(shot) -> image`` and return the
    image stacked over every shot of every rank.  Every rank takes part in the
    single all-reduce even when it has no shot (equal collective sequence)."""
    ws = dist.get_world_size(group) if (dist is not None and dist.is_initialized()) else 1
    rank = dist.get_rank(group) if (dist is not None and dist.is_initialized()) else 0
    acc = zeros_like_image()
    for s in shots_for_rank(n_shots, ws, rank):
        acc += run_one(s)
    return stack(acc, dist, group)
