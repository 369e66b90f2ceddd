"""Multi-process plumbing (one process per GPU, torch.distributed).

One patch splits into slabs of element layers with a p-layer exchange
(``jaxiga_b200.slab``). A batch of independent instances shards without
communication: ``partition_by_cost`` assigns instances to ranks so
that the per-rank work (elements, the apply's cost driver) is balanced --
largest first onto the least-loaded rank, ties to the lowest rank, so every
rank computes the same assignment without communication. Timings combine as
the maximum over ranks; results are gathered to every rank.
"""

from __future__ import annotations

import heapq


def partition_by_cost(costs, world):
    """Deterministic longest-processing-time assignment: list of index lists per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_by_index(local, parts, n):
    """Combine per-rank {instance index: result} dicts into a list ordered by instance."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        gathered = [None] * dist.get_world_size()
        dist.all_gather_object(gathered, local)
    else:
        gathered = [local]
    out = [None] * n
    for rank_result in gathered:
        for i, v in rank_result.items():
            out[i] = v
    missing = [i for i, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError(f"instances without a result: {missing[:10]}")
    return out
