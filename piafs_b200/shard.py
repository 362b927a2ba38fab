"""Work partition for runs over several GPUs, one process per GPU.

Ensemble members and serving requests are independent: a rank advances its
own share with no data exchanged during the run, and only per-rank results
(counts, timings, latencies) are gathered at the end.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def balance(work: Sequence[float], nranks: int) -> List[List[int]]:
    """Indices of the units per rank, balancing the summed work: units in
    decreasing work, each to the least-loaded rank (longest processing time
    first; makespan within 4/3 of the optimum, Graham 1969).  Ties go to the
    lower index and the lower rank, so every rank computes the same split."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    loads = [(0.0, r) for r in range(nranks)]
    heapq.heapify(loads)
    parts: List[List[int]] = [[] for _ in range(nranks)]
    for i in sorted(range(len(work)), key=lambda i: (-float(work[i]), i)):
        load, r = heapq.heappop(loads)
        parts[r].append(i)
        heapq.heappush(loads, (load + float(work[i]), r))
    return [sorted(p) for p in parts]


def round_robin(n: int, rank: int, nranks: int) -> List[int]:
    """Units rank, rank + nranks, ...: a rank's share of an arrival-ordered
    stream (a Poisson stream thinned this way stays Poisson at rate / nranks)."""
    return list(range(rank, n, nranks))


def gather(obj):
    """Every rank's obj, in rank order (the one collective of a sharded run:
    per-rank results after the work); [obj] without a process group."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
