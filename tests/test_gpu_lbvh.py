"""GPU LBVH build against the CPU oracle: every stage bit-exact, the final 64-byte
nodes, Woop triangles and triangle indices byte-identical (sm_100a)."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def build_with_taps(ctx, v, t, params):
    n = t.shape[0]
    nn = max(2 * n - 1, 1)
    cuda = torch.device("cuda")
    taps = dict(
        morton_keys=torch.zeros(max(n, 1), dtype=torch.int64, device=cuda),
        sorted_keys=torch.zeros(max(n, 1), dtype=torch.int64, device=cuda),
        sorted_refs=torch.zeros(max(n, 1), dtype=torch.int32, device=cuda),
        node_parent=torch.zeros(nn, dtype=torch.int32, device=cuda),
        node_left=torch.zeros(nn, dtype=torch.int32, device=cuda),
        node_right=torch.zeros(nn, dtype=torch.int32, device=cuda),
        node_box_min=torch.zeros((nn, 4), dtype=torch.float32, device=cuda),
        node_box_max=torch.zeros((nn, 4), dtype=torch.float32, device=cuda),
        scene_box=torch.zeros(6, dtype=torch.float32, device=cuda),
    )
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, params, taps=taps)
    bvh.sync()
    ctx.check()
    return bvh, {k: x.cpu().numpy() for k, x in taps.items()}, V, T


CASES = [("uniform", 2, 30), ("uniform", 3, 60), ("uniform", 1000, 30), ("uniform", 65536, 30),
         ("uniform", 65536, 60), ("clustered", 100000, 60), ("clustered", 262144, 30),
         ("clustered", 1_200_000, 60)]  # over 2^20 keys of 60 bits: the wide-key sort


def mesh(kind, n, seed):
    if kind == "uniform":
        return hp.gen.uniform_mesh(seed, n)
    return hp.gen.clustered_mesh(seed, n, clusters=min(1024, max(1, n // 64)))


@pytest.mark.parametrize("kind,n,bits", CASES)
def test_lbvh_stages_bit_exact(ctx, kind, n, bits):
    v, t = mesh(kind, n, 1000 + n)
    bvh, taps, V, T = build_with_taps(ctx, v, t, hp.BuildParams(morton_bits=bits))
    bmin, bmax, box = oracle.tri_boxes(v, t)
    np.testing.assert_array_equal(taps["scene_box"], box)
    np.testing.assert_array_equal(np.array(bvh.c.scene_box, np.float32), box)
    gpu_scale = np.array(bvh.c.morton_scale, np.float32)
    # the GPU's approximate 1/diagonal is within one ulp of the IEEE quotient
    ieee = (np.float32(1) / (box[3:] - box[:3])).astype(np.float32)
    assert np.all(np.abs(gpu_scale.view(np.int32) - ieee.view(np.int32)) <= 2)
    keys, _ = oracle.morton(bmin, bmax, box, bits, scale=gpu_scale)
    np.testing.assert_array_equal(taps["morton_keys"].view(np.uint64), keys)
    sk, sr = oracle.sort(keys, bits)
    np.testing.assert_array_equal(taps["sorted_keys"].view(np.uint64), sk)
    np.testing.assert_array_equal(taps["sorted_refs"], sr)
    parent, left, right = oracle.karras(sk)
    np.testing.assert_array_equal(taps["node_parent"], parent)
    np.testing.assert_array_equal(taps["node_left"], left)
    np.testing.assert_array_equal(taps["node_right"], right)
    nbmin, nbmax, size, cost, state = oracle.refit(v, t, sr, parent, left, right)
    np.testing.assert_array_equal(taps["node_box_min"], nbmin)
    np.testing.assert_array_equal(taps["node_box_max"], nbmax)

    ref = oracle.build_lbvh(v, t, bits=bits, scale=gpu_scale)
    nodes, woop, tri = bvh.download()
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(woop.view(np.int32), ref["woop"].view(np.int32))
    assert bvh.validate(V, T)
    c_gpu = bvh.cost()
    c_ref = oracle.cost(ref["nodes"], ref["box"])
    assert c_gpu == pytest.approx(c_ref, rel=1e-12)


def test_rebuild_reuses_allocation(ctx):
    v, t = hp.gen.uniform_mesh(5, 20000)
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, hp.BuildParams(morton_bits=30))
    ptr = bvh.c.nodes
    v2, t2 = hp.gen.uniform_mesh(6, 15000)
    ctx.build(dev(v2), dev(t2), hp.BuildParams(morton_bits=30), bvh=bvh)
    assert bvh.c.nodes == ptr
    nodes, woop, tri = bvh.download()
    ref = oracle.build_lbvh(v2, t2, bits=30, scale=np.array(bvh.c.morton_scale, np.float32))
    np.testing.assert_array_equal(nodes, ref["nodes"])


def test_non_adaptive_leaf_size(ctx):
    v, t = hp.gen.uniform_mesh(8, 30000)
    p = hp.BuildParams(morton_bits=60, adaptive_leaf=0, max_leaf_size=4)
    bvh = ctx.build(dev(v), dev(t), p)
    nodes, woop, tri = bvh.download()
    ref = oracle.build_lbvh(v, t, bits=60, adaptive=0, max_leaf=4, scale=np.array(bvh.c.morton_scale, np.float32))
    np.testing.assert_array_equal(nodes, ref["nodes"])
    sizes = ~nodes[bvh.c.num_interior:, 14]
    assert sizes.max() <= 4


@pytest.mark.parametrize("n", [0, 1, 2, 3, 5])
def test_tiny_meshes(ctx, n):
    v, t = hp.gen.uniform_mesh(77, n)
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, hp.BuildParams(morton_bits=30))
    bvh.sync()
    ctx.check()
    ref = oracle.build_lbvh(v, t, bits=30, scale=np.array(bvh.c.morton_scale, np.float32))
    nodes, woop, tri = bvh.download()
    np.testing.assert_array_equal(nodes, ref["nodes"])
    if n:
        assert bvh.validate(V, T)
    rays = hp.gen.rays_targeted(3, 4096)
    res = ctx.trace(bvh, dev(rays), results=torch.zeros((4096, 4), dtype=torch.int32, device="cuda")).cpu().numpy()
    exp = oracle.trace(ref["nodes"], ref["woop"], ref["tri_idx"], rays)
    np.testing.assert_array_equal(res, exp)


def test_duplicate_centroids(ctx):
    n = 5000
    base = np.array([[0.5, 0.5, 0.5], [0.52, 0.5, 0.5], [0.5, 0.52, 0.5]], np.float32)
    v = np.tile(base, (n, 1))
    v[: 3 * 100] += 0.25  # a few elsewhere so the scene box is not degenerate
    t = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    bvh, taps, V, T = build_with_taps(ctx, v, t, hp.BuildParams(morton_bits=60))
    ref = oracle.build_lbvh(v, t, bits=60, scale=np.array(bvh.c.morton_scale, np.float32))
    nodes, woop, tri = bvh.download()
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    assert bvh.validate(V, T)


def test_bad_vertex_index_reported(ctx):
    v, t = hp.gen.uniform_mesh(1, 100)
    t = t.copy()
    t[10, 1] = 10 ** 6  # out of range: the kernels clamp the read and report it
    bvh = ctx.build(dev(v), dev(t), hp.BuildParams(morton_bits=30))
    with pytest.raises(hp.HPError) as ei:
        bvh.sync()
    assert ei.value.status == 5
