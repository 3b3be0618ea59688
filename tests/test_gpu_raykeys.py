"""Every ray Morton key method (RayBuffer::MortonCodeMethod) on the GPU against
the oracle, bit for bit, on incoherent, targeted and axis-aligned rays with
origins inside and outside the key box; sorted traces with each method give
the unsorted results (sm_100a)."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu

METHODS = ["two_point", "aila", "paraboloid", "octahedron", "origin", "costa", "reis"]


def _rays():
    box = np.array([-0.5, -0.5, -0.5, 1.5, 1.5, 1.5], np.float32)
    r = np.concatenate([hp.gen.rays_sphere(41, 100000, box), hp.gen.rays_targeted(42, 50000)])
    axis = r[:3000].copy()  # axis-aligned and coordinate-plane directions, zero components
    axis[:, 4:7] = 0.0
    axis[np.arange(3000), 4 + np.arange(3000) % 3] = np.where(np.arange(3000) % 2, 1.0, -1.0)
    axis[1000:2000, 4:7] = r[1000:2000, 4:7]
    axis[1000:2000, 4] = 0.0
    axis[2500:, 7] = 0.0  # zero tmax
    return np.concatenate([r, axis]).astype(np.float32)


@pytest.mark.parametrize("method", METHODS)
def test_keys_bit_exact(ctx, method):
    rays = _rays()
    R = torch.from_numpy(rays).cuda()
    box = np.array([-0.25, -0.5, 0.0, 1.25, 1.5, 1.0], np.float32)
    try:
        for bits, b, length in [(64, None, 0.25), (30, None, 0.7), (20, box, 0.1), (61, box, 3.0)]:
            ctx.set_ray_keys(method, length)
            got = ctx.ray_keys(R, bits=bits, box=b).cpu().numpy().view(np.uint64)
            exp = oracle.ray_keys(rays, bits=bits, box=(0, 0, 0, 1, 1, 1) if b is None else b, method=method,
                                  ray_length=length)
            np.testing.assert_array_equal(got, exp)
    finally:
        ctx.set_ray_keys("aila", 0.25)


@pytest.mark.parametrize("method", METHODS)
def test_sorted_trace_with_each_method(ctx, method):
    v, t = hp.gen.clustered_mesh(43, 100000, 64)
    box = np.concatenate([v.min(0), v.max(0)])
    rays = hp.gen.rays_sphere(44, 1 << 18, box)
    V, T, R = (torch.from_numpy(x).cuda() for x in (v, t, rays))
    bvh = ctx.build(V, T, hp.BuildParams(morton_bits=60))
    a = ctx.trace(bvh, R, results=torch.zeros((R.shape[0], 4), dtype=torch.int32, device="cuda"))
    order = torch.empty(R.shape[0], dtype=torch.int32, device="cuda")
    try:
        ctx.set_ray_keys(method, 0.5)
        b = ctx.trace_sorted(bvh, R, results=torch.zeros_like(a), bits=64, order=order)
    finally:
        ctx.set_ray_keys("aila", 0.25)
    ctx.check()
    np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
    keys = oracle.ray_keys(rays, bits=64, method=method, ray_length=0.5)
    np.testing.assert_array_equal(order.cpu().numpy(), np.argsort(keys, kind="stable"))
