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
