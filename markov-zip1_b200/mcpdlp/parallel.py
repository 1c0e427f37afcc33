"""Multi-GPU layout of batched solves: independent LPs sharded across ranks.

A single LP is not split (each iteration would need an all-gather of x-bar and
a reduction of A^T y, as much traffic as the iteration itself); N GPUs run N
replicas.  A batch of independent LPs shards naturally: ``shard_by_nnz``
assigns LPs to ranks greedily by nonzeros (largest first, to the least loaded
rank), every rank solves its shard with mc_pdlp_ctx_solve_batch, and the
results are gathered on the host.  No collective touches the data path; only
timing scalars and result summaries are reduced.
"""
from __future__ import annotations

import heapq


def shard_by_nnz(sizes: list, world: int) -> list:
    """Indices of the LPs each rank solves (deterministic; ties by index)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]) + 1, r))
    return [sorted(s) for s in shards]


def imbalance(sizes: list, shards: list) -> float:
    """max shard load / mean shard load (1.0 = perfect)."""
    loads = [sum(int(sizes[i]) + 1 for i in s) for s in shards]
    mean = sum(loads) / max(1, len(loads))
    return max(loads) / mean if mean > 0 else 1.0
