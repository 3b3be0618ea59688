"""Primary rays, ray Morton keys and Morton-ordered tracing on the GPU against
the CPU oracle (bit-exact), sm_100a."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,sample,table", [(640, 320, 0, True), (257, 131, 5, True), (64, 64, 3, False)])
def test_primary_rays_vs_oracle(ctx, w, h, sample, table):
    pos = np.array([0.5, 0.5, -1.5], np.float32)
    m = hp.camera_screen_to_world(pos, [0, 0, 1], 45.0, w, h, 0.01, 100.0)
    tbl = hp.pixel_table(w, h) if table else None
    got = ctx.primary_rays(pos, m, w, h, max_dist=10.0, sample_index=sample,
                           index_to_pixel=None if tbl is None else torch.from_numpy(tbl).cuda())
    ctx.check()
    exp = oracle.primary_rays(pos, m, w, h, sample_index=sample, max_dist=10.0, index_to_pixel=tbl)
    np.testing.assert_array_equal(got.cpu().numpy(), exp)
    d = exp[:, 4:7]
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)


def test_ray_keys_vs_oracle(ctx):
    box = np.array([-0.5, -0.5, -0.5, 1.5, 1.5, 1.5], np.float32)
    rays = hp.gen.rays_sphere(21, 200000, box)
    R = torch.from_numpy(rays).cuda()
    for bits, b in [(30, None), (60, None), (64, box)]:
        got = ctx.ray_keys(R, bits=bits, box=b).cpu().numpy().view(np.uint64)
        exp = oracle.ray_keys(rays, bits=bits, box=(0, 0, 0, 1, 1, 1) if b is None else b)
        np.testing.assert_array_equal(got, exp)


def test_trace_sorted_equals_trace(ctx):
    v, t = hp.gen.clustered_mesh(31, 200000, 64)
    box = np.concatenate([v.min(0), v.max(0)])
    rays = hp.gen.rays_sphere(32, 1 << 19, box)
    V, T, R = (torch.from_numpy(x).cuda() for x in (v, t, rays))
    bvh = ctx.build(V, T, hp.BuildParams(morton_bits=60))
    a = ctx.trace(bvh, R, results=torch.zeros((R.shape[0], 4), dtype=torch.int32, device="cuda"))
    order = torch.empty(R.shape[0], dtype=torch.int32, device="cuda")
    b = ctx.trace_sorted(bvh, R, results=torch.zeros_like(a), bits=30, order=order)
    ctx.check()
    np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
    o = order.cpu().numpy()
    keys = oracle.ray_keys(rays, bits=30)
    assert np.array_equal(np.sort(o), np.arange(len(o)))
    np.testing.assert_array_equal(o, np.argsort(keys, kind="stable"))


def test_primary_rays_trace(ctx):
    v, t = hp.gen.uniform_mesh(41, 100000)
    V, T = torch.from_numpy(v).cuda(), torch.from_numpy(t).cuda()
    bvh = ctx.build(V, T, hp.BuildParams(morton_bits=60))
    w, h = 256, 128
    pos = np.array([0.5, 0.5, -1.5], np.float32)
    m = hp.camera_screen_to_world(pos, [0, 0, 1], 45.0, w, h, 0.01, 100.0)
    R = ctx.primary_rays(pos, m, w, h, index_to_pixel=torch.from_numpy(hp.pixel_table(w, h)).cuda())
    res = ctx.trace(bvh, R, results=torch.zeros((w * h, 4), dtype=torch.int32, device="cuda")).cpu().numpy()
    nodes, woop, tri = bvh.download()
    np.testing.assert_array_equal(res, oracle.trace(nodes, woop, tri, R.cpu().numpy()))
    # the unit box covers about 40 % of this 2:1 image
    assert 0.1 < (res[:, 0] >= 0).mean() < 0.6
