"""Multi-GPU plumbing for independent simulations: one process per GPU.

The batched sweep's instances are independent, so a sweep spread over GPUs
needs no data-path collective: each rank takes a cell-balanced share of the
instances and advances it on its own GPU.  The only collectives are the
host-side control ones below (timing max, result gather), which run on
whatever process group the caller initialised (NCCL on GPUs, gloo in tests).
"""

from __future__ import annotations

import heapq

import torch
import torch.distributed as dist


def shard_instances(cells, world):
    """Greedy longest-processing-time split of instances over ``world`` ranks.

    ``cells``: per-instance cell counts.  Returns ``world`` lists of instance
    indices whose cell totals differ by at most the largest instance."""
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for q in sorted(range(len(cells)), key=lambda q: -cells[q]):
        load, r = heapq.heappop(heap)
        out[r].append(q)
        heapq.heappush(heap, (load + int(cells[q]), r))
    return [sorted(s) for s in out]


def max_over_ranks(value: float, device=None) -> float:
    """The largest ``value`` over all ranks (e.g. a timed region)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_objects(obj):
    """All ranks' ``obj`` on every rank (results of a sharded sweep)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
