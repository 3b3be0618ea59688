"""GPU PLOC build against the CPU oracle: nodes, Woop triangles and triangle
order byte-identical; traversal of the PLOC BVH bit-identical (sm_100a)."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ploc(ctx, v, t, **kw):
    p = dict(method="ploc", morton_bits=60, ploc_radius=16, ploc_max_radius=256, ploc_adaptive=0)
    p.update(kw)
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, hp.BuildParams(**p))
    bvh.sync()
    ctx.check()
    ref = oracle.build_ploc(v, t, bits=p["morton_bits"], radius=p["ploc_radius"], max_radius=p["ploc_max_radius"],
                            adaptive_r=p["ploc_adaptive"], adaptive=p.get("adaptive_leaf", 1),
                            max_leaf=p.get("max_leaf_size", 8), scale=np.array(bvh.c.morton_scale, np.float32))
    return bvh, ref, V, T


@pytest.mark.parametrize("n", [2, 3, 100, 2048, 2049, 5000, 65536, 262144, 1 << 20])
def test_ploc_bit_exact(ctx, n):
    v, t = hp.gen.clustered_mesh(500 + n, n, clusters=max(1, min(1024, n // 64)))
    bvh, ref, V, T = _ploc(ctx, v, t)
    nodes, woop, tri = bvh.download()
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(woop.view(np.int32), ref["woop"].view(np.int32))
    assert bvh.validate(V, T)
    assert bvh.cost() == pytest.approx(oracle.cost(ref["nodes"], ref["box"]), rel=1e-12)


@pytest.mark.parametrize("n,radius,adaptive", [(1_500_000, 16, 0), (1_300_000, 2, 0), (1_250_000, 4, 0),
                                               (1_400_000, 7, 0), (1_300_000, 3, 1)])
def test_ploc_bit_exact_long_lists(ctx, n, radius, adaptive):
    """Lists of at least 148 * 4 * 512 clusters take the neighbour search with
    four clusters per thread (its run split for r >= 4, the tested path below);
    these builds run it down to that length and the one-cluster tiles after."""
    v, t = hp.gen.clustered_mesh(700 + n, n, clusters=1024)
    bvh, ref, V, T = _ploc(ctx, v, t, ploc_radius=radius, ploc_max_radius=max(radius, 9), ploc_adaptive=adaptive)
    nodes, woop, tri = bvh.download()
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    np.testing.assert_array_equal(nodes, ref["nodes"])


def test_ploc_adaptive_radius_and_fixed_leaves(ctx):
    v, t = hp.gen.uniform_mesh(9, 30000)
    bvh, ref, V, T = _ploc(ctx, v, t, ploc_radius=1, ploc_max_radius=24, ploc_adaptive=1)
    nodes, woop, tri = bvh.download()
    np.testing.assert_array_equal(nodes, ref["nodes"])
    bvh2, ref2, _, _ = _ploc(ctx, v, t, adaptive_leaf=0, max_leaf_size=3, morton_bits=30)
    nodes2, _, tri2 = bvh2.download()
    np.testing.assert_array_equal(nodes2, ref2["nodes"])
    np.testing.assert_array_equal(tri2, ref2["tri_idx"])


def test_ploc_trace_bit_exact(ctx):
    v, t = hp.gen.clustered_mesh(3, 200000, clusters=1024)
    bvh, ref, V, T = _ploc(ctx, v, t)
    box = np.concatenate([v.min(0), v.max(0)])
    rays = hp.gen.rays_sphere(4, 1 << 19, box)
    got = ctx.trace(bvh, dev(rays), results=torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda"))
    np.testing.assert_array_equal(got.cpu().numpy(), oracle.trace(ref["nodes"], ref["woop"], ref["tri_idx"], rays))


def test_ploc_beats_lbvh_cost(ctx):
    v, t = hp.gen.clustered_mesh(11, 300000, clusters=1024)
    bvh, ref, V, T = _ploc(ctx, v, t)
    lb = ctx.build(V, T, hp.BuildParams(morton_bits=60))
    assert bvh.cost() < lb.cost()
