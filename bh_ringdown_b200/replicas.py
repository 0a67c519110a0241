"""Several GPUs: independent replicas, one process (and one engine) per GPU.

Solves share nothing, so work is split at request granularity and no
collective touches the data path.  What the ranks do exchange is
bookkeeping: the max of their timed regions and, at the end, their
results' metadata.

* ``shard_requests`` assigns requests to ranks by estimated work (grid
  points times steps), longest first to the least loaded rank.  The rule
  is deterministic, so every rank computes the same assignment from the
  same request list without communicating.
* ``max_over_ranks`` and ``gather_objects`` wrap the two collectives (any
  ``torch.distributed`` backend; NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq
from typing import Callable, List, Sequence, TypeVar

T = TypeVar("T")


def request_work(params) -> float:
    """Estimated work of one solve: grid points x time steps (dt from the
    solver's Courant rule when params.dt <= 0, as the solver computes it)."""
    import numpy as np
    from . import grid
    if params.dt > 0:
        dt = params.dt
    else:
        _, r, _ = grid(params)
        dt = params.courant * min((params.Xmax - params.Xmin) / params.N, r[0] * np.pi / params.M)
        if params.out_every > 0:
            dt = params.out_every / np.ceil(params.out_every / dt)
    return float(params.N) * params.M * int(params.T / dt)


def shard_requests(work: Sequence[float], world: int) -> List[List[int]]:
    """Indices of the requests each rank runs: longest-processing-time
    first, each to the rank with the least work so far (ties to the lower
    rank); within a rank, indices stay in submission order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(work[i]), r))
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of ``value`` over all ranks (the value itself without a
    process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_objects(obj: T, dist=None) -> List[T]:
    """Every rank's ``obj``, in rank order, on every rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out: List[T] = [None] * dist.get_world_size()  # type: ignore[list-item]
    dist.all_gather_object(out, obj)
    return out


def run_shard(reqs: Sequence[T], rank: int, world: int, work_of: Callable[[T], float]) -> List[int]:
    """This rank's request indices."""
    return shard_requests([work_of(r) for r in reqs], world)[rank]
