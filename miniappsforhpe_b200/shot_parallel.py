"""Shot-parallel RTM across GPUs: host-side logic.

Shots are independent units of the RTM workload; the images of the shots of
one survey (one earth model and grid) add up.  The reference computes one
shot per run and has no shot-level parallelism; its multi-GPU code is a
spatial domain decomposition with halo exchanges, which this build replaces
by whole shots per GPU (one process per GPU, NCCL between them).

Two drivers:

* ``run_shot_stream``: every rank runs its share of a list of shots of one
  survey one after another (``run_one(shot) -> image``) and the stack is
  summed over ranks with one all-reduce.
* ``serve_stream``: every rank feeds its share of a stream of shots (any
  grids, any surveys) to its own shot server (continuous batching on its
  GPU), collects the images of each survey into a stack, and at the end of
  the stream the stacks are summed over ranks with one all-reduce per survey,
  in the same order on every rank.

Nothing here touches the kernels; the collectives come from the caller's
``torch.distributed`` (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq
from typing import Callable, Dict, Hashable, Iterable, List, Optional, Sequence, Tuple


def shots_for_rank(n_shots: int, world_size: int, rank: int) -> List[int]:
    """Round-robin assignment: shot s goes to rank s % world_size."""
    if world_size < 1 or not (0 <= rank < world_size) or n_shots < 0:
        raise ValueError("bad shot partition")
    return list(range(rank, n_shots, world_size))


def assign_by_cost(costs: Sequence[float], world_size: int) -> List[List[int]]:
    """Longest-processing-time-first assignment of shots to ranks: shots in
    decreasing cost (ties: lower index first), each to the rank with the least
    total cost so far (ties: lower rank).  Deterministic, so every rank
    computes the same partition from the same list.  Each rank's shots are
    returned in stream order."""
    if world_size < 1 or any(c < 0 for c in costs):
        raise ValueError("bad shot partition")
    heap = [(0.0, r) for r in range(world_size)]
    out: List[List[int]] = [[] for _ in range(world_size)]
    for s in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(s)
        heapq.heappush(heap, (load + costs[s], r))
    return [sorted(o) for o in out]


def shot_cost(shot) -> float:
    """Work of one shot for balancing: grid points times time steps."""
    return float(shot.nx) * shot.ny * shot.nz * shot.nt


def stack(image, dist=None, group=None):
    """Sum a per-rank image tensor over all ranks in place (no-op when single)."""
    if dist is not None and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(image, op=dist.ReduceOp.SUM, group=group)
    return image


def _world(dist, group) -> Tuple[int, int]:
    if dist is not None and dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


def run_shot_stream(n_shots: int, run_one: Callable[[int], "object"], zeros_like_image: Callable[[], "object"],
                    dist=None, group=None, steps: Optional[Iterable[int]] = None):
    """Run this rank's shots with ``run_one(shot) -> image`` and return the
    image stacked over every shot of every rank.  Every rank takes part in the
    single all-reduce even when it has no shot (equal collective sequence)."""
    ws, rank = _world(dist, group)
    acc = zeros_like_image()
    for s in shots_for_rank(n_shots, ws, rank):
        acc += run_one(s)
    return stack(acc, dist, group)


def serve_stream(shots: Sequence, server, survey_of: Callable[[int], Hashable], dist=None, group=None,
                 device=None, timeout: float = -1.0, on_submit: Optional[Callable[[int], None]] = None):
    """Serve a stream of shots over all ranks, one server per rank.

    ``shots`` is the whole stream, identical on every rank (objects with the
    fields of ``serve.Shot``); ``server`` is this rank's server (``submit(shot)
    -> ticket``, ``wait(ticket, timeout) -> result``), ``survey_of(i)`` the
    survey key of shot i (shots of one survey share a grid).  Shots are
    assigned with ``assign_by_cost``; this rank submits its own in stream
    order (``on_submit(i)`` is called first, e.g. to wait for the shot's
    arrival time), then waits for them.  Each image pair is added into its
    survey's stack; at the end every rank all-reduces every survey's stack in
    sorted key order, creating zero stacks for surveys it had no shot of, so
    all ranks issue the same collectives.

    Returns ({survey: (vp_stack, rho_stack)} as torch tensors on ``device``,
    {shot index: result} of this rank's shots)."""
    import numpy as np
    import torch

    ws, rank = _world(dist, group)
    mine = assign_by_cost([shot_cost(s) for s in shots], ws)[rank]
    grids: Dict[Hashable, Tuple[int, int, int]] = {}
    for i, s in enumerate(shots):
        g = (s.nz, s.ny, s.nx)
        k = survey_of(i)
        if grids.setdefault(k, g) != g:
            raise ValueError(f"survey {k!r} has shots on different grids")
    dev = torch.device("cpu") if device is None else device
    stacks = {k: (torch.zeros(g, dtype=torch.float32, device=dev), torch.zeros(g, dtype=torch.float32, device=dev))
              for k, g in grids.items()}
    tickets = []
    for i in mine:
        if on_submit is not None:
            on_submit(i)
        tickets.append((i, server.submit(shots[i])))
    results = {}
    for i, t in tickets:
        results[i] = server.wait(t, timeout)
        vp, rho = stacks[survey_of(i)]
        vp += torch.from_numpy(np.ascontiguousarray(shots[i].image_vp)).to(dev)
        rho += torch.from_numpy(np.ascontiguousarray(shots[i].image_rho)).to(dev)
    for k in sorted(stacks, key=repr):
        for img in stacks[k]:
            stack(img, dist, group)
    return stacks, results
