"""Sharding of independent pairs over ranks (one process per GPU).

The path has no exchange step: pairs are independent units, so multi-GPU is
data parallel over pairs with no collective on the data path.  What remains
is bookkeeping, which works with any torch.distributed backend (NCCL on the
GPUs, gloo in the CPU tests):

* ``shard``: size-balanced assignment (longest processing time first, by
  pixel count) of pair indices to ranks, identical on every rank;
* ``max_over_ranks``: the step time of a job is its slowest rank;
* ``gather_metrics``: per-rank result records to every rank.
"""

from __future__ import annotations

import heapq


def shard(sizes, rank: int, world: int) -> list:
    """Indices of the pairs ``rank`` processes.  ``sizes`` are the per-pair
    costs (e.g. W*H); every rank computes the same assignment."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside world of %d" % (rank, world))
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    heap = [(0, r) for r in range(world)]
    owner = [0] * len(sizes)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + sizes[i], r))
    return [i for i in range(len(sizes)) if owner[i] == rank]


def max_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_metrics(record: dict) -> list:
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [record]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, record)
    return out
