"""Quad / Oct layouts on the GPU: the device collapse byte-identical to the
oracle's restatement of BVH::collapseAdaptiveWide + BVHConverter::convert (which
is pinned to the reference's own host code, tests/test_oracle_wide.py); the
wide tracer returning the binary tracer's hits (and the oracle's) bit for bit;
statistics and validation on the wide records (sm_100a)."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def trace(ctx, bvh, R, **kw):
    """Results with a zeroed buffer: a miss writes only {-1, tmax}."""
    res = torch.zeros((R.shape[0], 4), dtype=torch.int32, device="cuda")
    out = ctx.trace(bvh, R, results=res, **kw)
    return out


def build(ctx, v, t, method, layout, **kw):
    p = dict(method=method, morton_bits=60, layout=layout, atr_treelet=9, atr_iterations=2, ploc_radius=16,
             ploc_max_radius=256, ploc_adaptive=0)
    p.update(kw)
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, hp.BuildParams(**p))
    bvh.sync()
    ctx.check()
    return bvh, V, T


def oracle_wide(bvh, v, t, method, width, **kw):
    return oracle.build_wide(v, t, width, method=method, bits=kw.get("morton_bits", 60), treelet=9, iterations=2,
                             adaptive=kw.get("adaptive_leaf", 1), max_leaf=kw.get("max_leaf_size", 8),
                             scale=np.array(bvh.c.morton_scale, np.float32))


@pytest.mark.parametrize("method", ["lbvh", "ploc", "atr"])
@pytest.mark.parametrize("layout", [4, 8])
@pytest.mark.parametrize("n", [2, 3, 17, 1000, 40000])
def test_wide_build_bit_exact(ctx, method, layout, n):
    v, t = hp.gen.clustered_mesh(700 + n, n, clusters=max(1, min(256, n // 64)), sigma=0.05, half_extent=0.01)
    bvh, V, T = build(ctx, v, t, method, layout)
    ref = oracle_wide(bvh, v, t, method, layout)
    nodes, woop, tri = bvh.download()
    assert bvh.layout == layout and nodes.shape[1] == 8 * layout
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(woop.view(np.int32), ref["woop"].view(np.int32))
    assert bvh.validate(V, T)


@pytest.mark.parametrize("layout", [4, 8])
def test_wide_fixed_leaves(ctx, layout):
    v, t = hp.gen.uniform_mesh(31, 20000)
    kw = dict(adaptive_leaf=0, max_leaf_size=5)
    bvh, V, T = build(ctx, v, t, "lbvh", layout, **kw)
    ref = oracle_wide(bvh, v, t, "lbvh", layout, **kw)
    nodes, _, tri = bvh.download()
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(tri, ref["tri_idx"])


@pytest.mark.parametrize("layout", [4, 8])
def test_single_triangle(ctx, layout):
    v, t = hp.gen.uniform_mesh(2, 1)
    bvh, V, T = build(ctx, v, t, "lbvh", layout)
    ref = oracle_wide(bvh, v, t, "lbvh", layout)
    nodes, _, tri = bvh.download()
    np.testing.assert_array_equal(nodes, ref["nodes"])
    assert bvh.validate(V, T)
    rays = hp.gen.rays_sphere(1, 4096, np.concatenate([v.min(0) - 0.1, v.max(0) + 0.1]))
    bb, _, _ = build(ctx, v, t, "lbvh", 2)
    np.testing.assert_array_equal(trace(ctx, bvh, dev(rays)).cpu().numpy(), trace(ctx, bb, dev(rays)).cpu().numpy())


@pytest.mark.parametrize("method", ["lbvh", "ploc", "atr"])
@pytest.mark.parametrize("layout", [4, 8])
def test_wide_trace_matches_binary(ctx, method, layout):
    v, t = hp.gen.clustered_mesh(5, 120000, clusters=256)
    box = np.concatenate([v.min(0), v.max(0)])
    rays = np.concatenate([hp.gen.rays_sphere(6, 1 << 17, box), hp.gen.rays_targeted(7, 1 << 17)])
    R = dev(rays)
    wb, V, T = build(ctx, v, t, method, layout)
    bb, _, _ = build(ctx, v, t, method, 2)
    got = trace(ctx, wb, R).cpu().numpy()
    want = trace(ctx, bb, R).cpu().numpy()
    np.testing.assert_array_equal(got, want)
    # the oracle's binary traversal agrees as well
    nodes, woop, tri = bb.download()
    np.testing.assert_array_equal(got[:4096], oracle.trace(nodes, woop, tri, rays[:4096]))
    # any-hit finds a hit exactly where closest-hit does
    anyh = trace(ctx, wb, R, any_hit=True).cpu().numpy()
    np.testing.assert_array_equal(anyh[:, 0] >= 0, got[:, 0] >= 0)
    # statistics: nodes visited and triangles tested, zero for misses
    st = torch.zeros((R.shape[0], 2), dtype=torch.int32, device="cuda")
    res = trace(ctx, wb, R, stats=st)
    np.testing.assert_array_equal(res.cpu().numpy(), got)
    st = st.cpu().numpy()
    assert (st[got[:, 0] < 0] == 0).all() and (st[got[:, 0] >= 0] > 0).all()


@pytest.mark.parametrize("layout", [4, 8])
def test_wide_sorted_trace(ctx, layout):
    v, t = hp.gen.uniform_mesh(8, 50000)
    rays = hp.gen.rays_sphere(9, 1 << 18, np.concatenate([v.min(0), v.max(0)]))
    R = dev(rays)
    wb, _, _ = build(ctx, v, t, "ploc", layout)
    res = torch.zeros((R.shape[0], 4), dtype=torch.int32, device="cuda")
    np.testing.assert_array_equal(ctx.trace_sorted(wb, R, results=res).cpu().numpy(), trace(ctx, wb, R).cpu().numpy())


@pytest.mark.parametrize("layout", [4, 8])
def test_wide_stats_and_cost(ctx, layout):
    v, t = hp.gen.clustered_mesh(12, 30000, clusters=64, sigma=0.05, half_extent=0.01)
    bvh, V, T = build(ctx, v, t, "ploc", layout)
    st = bvh.stats()
    nodes, _, _ = bvh.download()
    N = layout
    ni = bvh.c.num_interior
    size = nodes[:, 8 * N - 5]
    sizes = ~size[ni:].astype(np.int64)
    assert st["sum_of_leaf_sizes"] == 30000 and st["avg_leaf_size"] == pytest.approx(sizes.mean(), rel=1e-15)
    hist = np.bincount(sizes[sizes <= 32], minlength=33)[:33] / len(sizes)
    np.testing.assert_array_equal(np.array(st["leaf_size_histogram"], np.float32), hist.astype(np.float32))
    # computeCost: union of the N stored boxes; leaves billed ceil(size/N)*N references
    f = nodes.view(np.float32).astype(np.float64)
    mnx = f[:, 0:4 * N:4].min(1); mxx = f[:, 1:4 * N:4].max(1)
    mny = f[:, 2:4 * N:4].min(1); mxy = f[:, 3:4 * N:4].max(1)
    mnz = f[:, 4 * N:8 * N:4].min(1); mxz = f[:, 4 * N + 1:8 * N:4].max(1)
    dx, dy, dz = mxx - mnx, mxy - mny, mxz - mnz
    area = 2 * (dx * dy + dy * dz + dz * dx)
    b = np.array(bvh.c.scene_box, np.float64)
    sd = b[3:] - b[:3]
    scene = 2 * (sd[0] * sd[1] + sd[1] * sd[2] + sd[2] * sd[0])
    billed = np.where(size < 0, (~size + N - 1) // N * N, 0)
    want = np.sum(np.where(size < 0, bvh.c.ci * area / scene * billed, bvh.c.ct * area / scene))
    assert st["sah_cost"] == pytest.approx(want, rel=1e-6)
    assert bvh.validate(V, T)
