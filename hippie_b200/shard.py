"""Sharding of independent meshes across ranks (one process per GPU).

A batch of meshes partitions with no exchange on the data path: every rank
builds and traces its own meshes, and only per-rank statistics travel, on the
host. Meshes go to ranks by greedy longest-processing-time order (largest
work first, each to the currently least-loaded rank; ties to the lower rank),
with work = triangles + rays / 4, so every rank's build and trace load is
within one mesh of the mean.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_partition(work, world: int):
    """Assign item i (with cost work[i]) to a rank; returns a list of index arrays per rank
    (each sorted ascending, so a rank keeps the original mesh order)."""
    work = np.asarray(work, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(work[i]), r))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def mesh_work(triangles, rays):
    return np.asarray(triangles, np.float64) + np.asarray(rays, np.float64) / 4.0


def gather_rank_stats(stats: dict, group=None):
    """All ranks' host-side statistics (torch.distributed all_gather_object)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return [stats]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, stats, group=group)
    return out
