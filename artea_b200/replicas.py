"""Replicas across GPUs: every rank holds the whole index and answers a
contiguous shard of a batch; result rows are all-gathered.

Queries are independent (hierarchical_graph_router.hpp:336-346 runs them as a
parallel_for with no shared state), and the index fits one GPU, so there is no
exchange on the search path: the only collective gathers the finished rows.
"""

from __future__ import annotations

from typing import Callable

import numpy as np


def shard(nq: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of the queries rank answers: contiguous, sizes differ by at most one."""
    base, extra = divmod(nq, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class ReplicatedRouter:
    """Splits a batch across the ranks of a torch.distributed group.

    search(queries) -> (n, k_stride) uint64 result words runs on this rank's
    replica (the GPU router in production)."""

    def __init__(self, search: Callable[[np.ndarray], np.ndarray], k_stride: int, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.search = search
        self.k_stride = k_stride
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def batch_query(self, queries: np.ndarray) -> np.ndarray:
        import torch
        nq = queries.shape[0]
        lo, hi = shard(nq, self.rank, self.world)
        local = self.search(queries[lo:hi]) if hi > lo else np.empty((0, self.k_stride), np.uint64)
        # Pad every shard to the largest size so all_gather sees equal shapes.
        width = -(-nq // self.world)
        buf = np.zeros((width, self.k_stride), dtype=np.uint64)
        buf[: hi - lo] = local
        t = torch.from_numpy(buf.view(np.int64))
        parts = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(parts, t, group=self.group)
        rows = []
        for r in range(self.world):
            a, b = shard(nq, r, self.world)
            rows.append(parts[r].numpy().view(np.uint64)[: b - a])
        return np.concatenate(rows, axis=0)
