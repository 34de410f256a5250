"""Request-level sharding over GPUs: one process per GPU (torch.distributed ranks), each solving
its own share of independent units — the scenarios of a batch, the requests of a serving stream.
There is no exchange on the data path: a unit is solved entirely on one GPU, and only the small
per-unit results travel (host bookkeeping, through the process group's object collectives).

* :func:`assign` splits units over ranks: round robin, or — given a cost per unit (e.g. its
  nonzeros) — longest-processing-time first, each unit to the least-loaded rank, which keeps the
  ranks' makespans balanced when the units' sizes differ by orders of magnitude (a serving
  stream's LPs span 1e3..2e5 rows). Deterministic: every rank computes the same assignment.
* :func:`gather` collects every rank's ``{unit index: result}`` on all ranks.
"""
from __future__ import annotations

import heapq


def assign(n: int, world: int, cost=None) -> list[list[int]]:
    """The unit indices [0, n) of every rank: ``out[r]`` in increasing order. With ``cost``
    (one non-negative number per unit), units are taken by decreasing cost (ties by index) and
    each goes to the rank with the smallest total so far (ties to the lowest rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    out = [[] for _ in range(world)]
    if cost is None:
        for k in range(n):
            out[k % world].append(k)
        return out
    if len(cost) != n:
        raise ValueError("one cost per unit")
    heap = [(0.0, r) for r in range(world)]
    for k in sorted(range(n), key=lambda k: (-float(cost[k]), k)):
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + float(cost[k]), r))
    return [sorted(v) for v in out]


def gather(local: dict, world: int) -> dict:
    """Every rank's ``{unit index: result}`` merged, on every rank (all_gather_object; the
    results must be picklable). world == 1 returns ``local``."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, local)
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"unit {k} solved on two ranks")
            merged[k] = v
    return merged
