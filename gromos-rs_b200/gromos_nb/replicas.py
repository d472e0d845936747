"""Multi-GPU host logic: independent systems spread over ranks (one process per GPU).

The nonbonded path has no exchange step, so several GPUs only ever run
independent systems -- replicas, lambda windows, serving jobs.  Ranks share
nothing on the force path; the only collectives are bookkeeping: the wall of
a timed region is the slowest rank's device time (max over ranks) and the
work done is the sum over ranks.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence, Tuple


def shard_by_work(work: Sequence[float], world: int) -> List[List[int]]:
    """Greedy longest-first bin packing of whole systems onto ``world`` ranks.

    ``work`` holds a cost per system (e.g. atom pairs per step).  Systems are
    taken in decreasing cost (ties by index) and each goes to the rank with
    the least work so far (ties by rank), so the result is deterministic and
    every rank can compute it without communication.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-float(work[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(work[i]), r))
    return [sorted(s) for s in shards]


def aggregate(local_ms: float, local_units: float, device=None) -> Tuple[float, float]:
    """(max over ranks of ``local_ms``, sum over ranks of ``local_units``).

    Uses the default process group (NCCL with CUDA tensors, gloo with CPU
    tensors; ``device`` picks the tensor device).  Without an initialised
    group it returns the local values.
    """
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(local_ms), float(local_units)
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(local_units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())
