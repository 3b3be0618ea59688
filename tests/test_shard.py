"""Sharding of independent meshes across ranks: LPT balance, and a world-size-2
gloo run whose per-rank CPU builds, gathered on the host, equal one process
building every mesh."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from hippie_b200.shard import gather_rank_stats, lpt_partition, mesh_work


def test_lpt_balance():
    rng = np.random.default_rng(1)
    sizes = np.round(np.exp(rng.uniform(np.log(256), np.log(262144), 2048))).astype(np.int64)
    work = mesh_work(sizes, 4 * sizes)
    for world in (1, 2, 4, 8):
        parts = lpt_partition(work, world)
        assert sorted(np.concatenate(parts).tolist()) == list(range(len(sizes)))
        loads = [work[p].sum() for p in parts]
        assert max(loads) - min(loads) <= work.max()
        assert max(loads) <= work.sum() / world + work.max()


def test_lpt_edge_cases():
    assert [p.tolist() for p in lpt_partition([], 3)] == [[], [], []]
    assert [p.tolist() for p in lpt_partition([5, 5, 5], 3)] == [[0], [1], [2]]
    assert [p.tolist() for p in lpt_partition([1, 9, 1, 1], 2)] == [[1], [0, 2, 3]]
    with pytest.raises(ValueError):
        lpt_partition([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _mesh_stats(i):
    import hippie_b200 as hp
    import oracle
    n = 200 + 37 * i
    v, t = hp.gen.uniform_mesh(500 + i, n)
    r = oracle.build_lbvh(v, t, bits=30)
    return {"mesh": i, "interior": int(r["counts"][0]), "leaves": int(r["counts"][1]),
            "cost": float(oracle.cost(r["nodes"], r["box"])), "tri0": int(r["tri_idx"][0])}


def _worker(rank, world, port, sizes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = lpt_partition(mesh_work(sizes, 4 * np.asarray(sizes)), world)[rank]
        stats = {int(i): _mesh_stats(int(i)) for i in mine}
        allst = gather_rank_stats(stats)
        if rank == 0:
            merged = {}
            for d in allst:
                merged.update(d)
            q.put(merged)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo_equal_one_process():
    sizes = [200 + 37 * i for i in range(9)]
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(9))
    for i in range(9):
        assert merged[i] == _mesh_stats(i)


def test_ray_ranges_cover_every_ray_once():
    from hippie_b200.shard import ray_ranges
    for n in (0, 1, 7, 1000, 16777216):
        for world in (1, 2, 3, 8):
            rr = ray_ranges(n, world)
            assert rr[0][0] == 0 and rr[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rr, rr[1:]))
            sizes = [e - b for b, e in rr]
            assert max(sizes) - min(sizes) <= 1


def _scene_and_rays():
    import hippie_b200 as hp
    v, t = hp.gen.clustered_mesh(31, 6000, clusters=32)
    rays = hp.gen.rays_sphere(32, 10001, np.concatenate([v.min(0), v.max(0)]))
    return v, t, rays


def _ray_worker(rank, world, port, q):
    """One mesh, rays split across ranks: rank 0 builds (the oracle stands in
    for the device build here), the BVH arrays and their node counts, scene box
    and Morton scale are broadcast into same-shaped buffers on the other rank,
    every rank traces its contiguous slice and the slices are all-gathered."""
    import torch
    import torch.distributed as dist
    import oracle
    from hippie_b200.shard import broadcast_bvh_arrays, gather_ray_results, ray_ranges
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v, t, rays = _scene_and_rays()
        n = t.shape[0]
        cap = 2 * n - 1
        nodes = torch.zeros((cap, 16), dtype=torch.int32)
        woop = torch.zeros((n, 12), dtype=torch.float32)
        tri = torch.zeros(n, dtype=torch.int32)
        info = None
        if rank == 0:
            r = oracle.build_ploc(v, t, radius=4, max_radius=64)
            k = r["nodes"].shape[0]
            nodes[:k] = torch.from_numpy(r["nodes"])
            woop[:] = torch.from_numpy(r["woop"])
            tri[:] = torch.from_numpy(r["tri_idx"])
            info = {"num_interior": int(r["counts"][0]), "num_leaf": int(r["counts"][1]),
                    "scene_box": r["box"].tolist(), "morton_scale": r["scale"].tolist()}
        got = broadcast_bvh_arrays((nodes, woop, tri), info, src=0)
        k = got["num_interior"] + got["num_leaf"]
        b, e = ray_ranges(rays.shape[0], world)[rank]
        part = oracle.trace(nodes[:k].numpy(), woop.numpy(), tri.numpy(), rays[b:e])
        full = gather_ray_results(torch.from_numpy(part), rays.shape[0])
        if rank == 0:
            q.put((got, full.numpy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_ray_partition_two_ranks_gloo_equal_one_process():
    import oracle
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_ray_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, full = q.get(timeout=180)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    v, t, rays = _scene_and_rays()
    r = oracle.build_ploc(v, t, radius=4, max_radius=64)
    assert got["num_interior"] == int(r["counts"][0]) and got["num_leaf"] == int(r["counts"][1])
    np.testing.assert_array_equal(np.array(got["scene_box"], np.float32), r["box"])
    np.testing.assert_array_equal(full, oracle.trace(r["nodes"], r["woop"], r["tri_idx"], rays))
