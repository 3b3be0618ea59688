"""GPU closest-hit traversal against the CPU oracle: results bit-identical
(triangle id, t, u, v), stats identical, any-hit semantics (sm_100a)."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _setup(ctx, kind, n, n_rays, bits, seed=0):
    if kind == "uniform":
        v, t = hp.gen.uniform_mesh(seed + 1, n)
        rays = hp.gen.rays_targeted(seed + 2, n_rays)
    else:
        v, t = hp.gen.clustered_mesh(seed + 1, n, clusters=1024)
        lo, hi = v.min(0), v.max(0)
        rays = hp.gen.rays_sphere(seed + 2, n_rays, np.concatenate([lo, hi]))
    bvh = ctx.build(dev(v), dev(t), hp.BuildParams(morton_bits=bits))
    bvh.sync()
    return v, t, rays, bvh


@pytest.mark.parametrize("kind,n,n_rays,bits", [("uniform", 65536, 1 << 20, 30),
                                                ("clustered", 262144, 1 << 20, 60)])
def test_trace_bit_exact(ctx, kind, n, n_rays, bits):
    v, t, rays, bvh = _setup(ctx, kind, n, n_rays, bits)
    R = dev(rays)
    res = torch.zeros((n_rays, 4), dtype=torch.int32, device="cuda")
    st = torch.zeros((n_rays, 2), dtype=torch.int32, device="cuda")
    ctx.trace(bvh, R, results=res, stats=st)
    ctx.check()
    nodes, woop, tri = bvh.download()
    exp, est = oracle.trace(nodes, woop, tri, rays, stats=True)
    got = res.cpu().numpy()
    np.testing.assert_array_equal(got, exp)
    # Counters: postponed leaves make the GPU's visit order depend on the warp,
    # so node / triangle counts are compared in aggregate, not per ray.
    gst = st.cpu().numpy()
    hit = exp[:, 0] >= 0
    assert np.all(gst[~hit] == 0) and np.all(gst[hit] > 0)
    for k in range(2):
        assert abs(gst[hit, k].mean() / est[hit, k].mean() - 1.0) < 0.15
    hits = (got[:, 0] >= 0).mean()
    assert 0.05 < hits < 1.0
    # plain trace (no stats) gives the same results
    res2 = torch.zeros_like(res)
    ctx.trace(bvh, R, results=res2)
    assert torch.equal(res, res2)


def test_trace_vs_double_brute_force(ctx):
    v, t, rays, bvh = _setup(ctx, "uniform", 4000, 20000, 60, seed=5)
    got = ctx.trace(bvh, dev(rays)).cpu().numpy()
    bf = oracle.brute64(v, t, rays)
    hit = got[:, 0] >= 0
    both = hit & (bf[:, 0] >= 0)
    assert np.mean(hit == (bf[:, 0] >= 0)) > 0.999
    assert np.mean(got[both, 0] == bf[both, 0]) > 0.999
    tuv = got[both, 1:].view(np.float32).astype(np.float64)
    err = np.abs(tuv - bf[both, 1:]) / np.maximum(1.0, np.abs(bf[both, 1:]))
    # t is accurate to a few ulps; the FP32 Woop test computes u and v as a
    # difference of terms ~1/triangle size, so against exact barycentrics they
    # carry ~1e-5 absolute error (as the reference's own Woop test does).
    assert np.median(err[:, 0]) < 1e-6 and np.quantile(err[:, 0], 0.999) < 1e-4
    assert np.quantile(err[:, 1:], 0.99) < 1e-3


def test_any_hit_and_limits(ctx):
    v, t, rays, bvh = _setup(ctx, "uniform", 50000, 100000, 30, seed=9)
    R = dev(rays)
    closest = ctx.trace(bvh, R).cpu().numpy()
    anyh = torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda")
    ctx.trace(bvh, R, results=anyh, any_hit=True)
    anyh = anyh.cpu().numpy()
    np.testing.assert_array_equal(anyh[:, 0] >= 0, closest[:, 0] >= 0)
    # any hit: some intersected triangle, never closer than the closest one
    h = anyh[:, 0] >= 0
    assert np.all(anyh[h, 1].view(np.float32) >= closest[h, 1].view(np.float32))
    bf = oracle.brute64(v, t, rays[h][:2000])
    for i, row in enumerate(anyh[h][:2000]):
        p = v[t[row[0]]].astype(np.float64)
        ok, tuv = oracle.intersect64(p[0], p[1], p[2], rays[h][i, :3], rays[h][i, 4:7])
        assert ok and abs(tuv[0] - row[1:2].view(np.float32)[0]) <= 1e-4 * max(1.0, tuv[0]), i
    assert np.all(bf[:, 0] >= 0)
    nodes, woop, tri = bvh.download()
    # tmin / tmax windows
    r2 = rays.copy()
    r2[:, 3] = 0.3
    r2[:, 7] = 1.2
    got = ctx.trace(bvh, dev(r2), results=torch.zeros((r2.shape[0], 4), dtype=torch.int32, device="cuda"))
    exp = oracle.trace(nodes, woop, tri, r2)
    np.testing.assert_array_equal(got.cpu().numpy(), exp)
    tt = exp[exp[:, 0] >= 0, 1].view(np.float32)
    assert np.all((tt > 0.3) & (tt < 1.2))
    miss = exp[:, 0] < 0
    assert np.all(exp[miss, 1].view(np.float32) == np.float32(1.2))


def test_axis_aligned_rays(ctx):
    """Direction components of exactly zero take the 2^-80 reciprocal path."""
    v, t = hp.gen.uniform_mesh(3, 20000)
    bvh = ctx.build(dev(v), dev(t), hp.BuildParams(morton_bits=30))
    rng = np.random.default_rng(0)
    n = 30000
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = rng.uniform(0, 1, (n, 3))
    axis = rng.integers(0, 3, n)
    sign = rng.choice([-1.0, 1.0], n)
    rays[np.arange(n), 4 + axis] = sign
    rays[np.arange(n), axis] = np.where(sign > 0, -0.5, 1.5)
    rays[:, 7] = np.inf
    got = ctx.trace(bvh, dev(rays)).cpu().numpy()
    nodes, woop, tri = bvh.download()
    exp = oracle.trace(nodes, woop, tri, rays)
    np.testing.assert_array_equal(got[:, :2], exp[:, :2])
    h = exp[:, 0] >= 0
    np.testing.assert_array_equal(got[h], exp[h])
