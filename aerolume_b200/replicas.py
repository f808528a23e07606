"""Host-side logic of multi-GPU runs: one process per GPU, no data-path collective.

A single instance of the solver does not shard (its spectral Poisson solve is global), so a
multi-GPU run is either replicas (every rank advances its own copy: weak scaling) or, for the
batched sweep, a partition of the independent instances over the ranks.  The only
communication is on the host side: the max of the ranks' device times, and the per-instance
results gathered to rank 0.  These helpers take a ``torch.distributed`` module (NCCL on the
GPUs, gloo in the CPU tests) or None for a single process.
"""
from __future__ import annotations

import heapq
from typing import Any, Sequence


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of ``value`` over all ranks (the value itself without a process group).
    ``device`` is where the reduction tensor lives (the rank's GPU for NCCL, CPU for gloo)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_instances(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Indices of the instances each of ``world`` ranks advances: largest first to the rank
    with the least work so far (ties to the lower rank), so the ranks' cell counts differ by
    at most the largest instance.  Every index appears exactly once; each rank's list is in
    increasing order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    heap = [(0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        shards[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return [sorted(s) for s in shards]


def gather_results(local: dict[int, Any], dist=None) -> dict[int, Any] | None:
    """Per-instance results (instance index -> picklable value) of every rank, merged on rank
    0; other ranks get None.  Without a process group the local dict is returned."""
    if dist is None:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(local))
    if dist.get_rank() != 0:
        return None
    out: dict[int, Any] = {}
    for p in parts:
        out.update(p)
    return out
