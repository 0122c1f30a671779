"""Multi-GPU plumbing for batched analyses: one process per GPU, no collective on the data path.

Independent frame-and-record instances are partitioned across ranks balanced by fiber count
(greedy, largest first onto the least-loaded rank); each rank runs its share in its own handle.
The only exchanges are host-side: a max-reduction of the timed region and an optional gather
of per-instance statistics at the end.
"""
from __future__ import annotations

import heapq


def partition_by_weight(weights, world: int):
    """Assign item indices to ``world`` bins, largest weight first onto the lightest bin.
    Deterministic: ties break on the lower bin index.  Returns a list of index lists."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    bins = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        bins[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(b) for b in bins]


def rank_share(weights, world: int, rank: int):
    return partition_by_weight(weights, world)[rank]


def max_over_ranks(value: float, group=None) -> float:
    """Max of a host float over all ranks (gloo or nccl process group)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_stats(stats: dict, group=None):
    """All ranks' stats dicts (host objects) on every rank."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return [stats]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, stats, group=group)
    return out
