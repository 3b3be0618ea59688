"""Work across ranks (one process per GPU).

Many meshes: a batch partitions with no exchange on the data path. Every rank
builds and traces its own meshes, and only per-rank statistics travel, on the
host. Meshes go to ranks by greedy longest-processing-time order (largest
work first, each to the currently least-loaded rank; ties to the lower rank),
with work = triangles + rays / 4, so every rank's build and trace load is
within one mesh of the mean.

One mesh, many rays: every rank holds the whole BVH and traces a contiguous
slice of the rays. The BVH is replicated either by building it on every rank
from the same input (no collective on the data path) or by building it on one
rank and broadcasting its node, Woop and triangle-index arrays (with the node
counts, scene box and Morton scale) into the BVHs the other ranks reserved;
results go back by one all-gather or stay with the rank that traced them. The
functions below work on torch tensors of any device, so the same code runs
over NCCL on GPUs and over gloo on CPU tensors.
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


def ray_ranges(num_rays: int, world: int):
    """Contiguous ray slices [begin, end) per rank; sizes differ by at most one."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(int(num_rays), world)
    out, b = [], 0
    for r in range(world):
        e = b + base + (1 if r < extra else 0)
        out.append((b, e))
        b = e
    return out


def broadcast_bvh_arrays(arrays, info, src: int = 0, group=None):
    """Broadcast a BVH from rank `src` into the same-shaped tensors of every rank.

    arrays: the node, Woop and triangle-index tensors (the sender's hold the
    built BVH, the receivers' were reserved with the same capacity); only the
    first num_interior + num_leaf node rows are sent. info: on the sender a dict with
    num_interior, num_leaf, scene_box (6 floats), morton_scale (3 floats);
    receivers' values are replaced. Returns the info every rank now holds."""
    import torch
    import torch.distributed as dist
    dev = arrays[0].device
    meta = torch.zeros(11, dtype=torch.float64, device=dev)
    if dist.get_rank(group) == src:
        meta[0], meta[1] = float(info["num_interior"]), float(info["num_leaf"])
        meta[2:8] = torch.tensor(info["scene_box"], dtype=torch.float64)
        meta[8:11] = torch.tensor(info["morton_scale"], dtype=torch.float64)
    dist.broadcast(meta, src, group=group)
    m = meta.cpu().tolist()
    out = {"num_interior": int(m[0]), "num_leaf": int(m[1]), "scene_box": m[2:8], "morton_scale": m[8:11]}
    nodes, woop, tri = arrays
    count = out["num_interior"] + out["num_leaf"]
    dist.broadcast(nodes[:count], src, group=group)
    dist.broadcast(woop, src, group=group)
    dist.broadcast(tri, src, group=group)
    return out


def gather_ray_results(local, num_rays: int, group=None):
    """All-gather every rank's slice of per-ray results (rows) into the full
    array, in ray order, on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    ranges = ray_ranges(num_rays, world)
    width = max(e - b for b, e in ranges)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([parts[r][:e - b] for r, (b, e) in enumerate(ranges)])
