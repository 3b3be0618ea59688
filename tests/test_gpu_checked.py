"""Checked mode (hp_ctx_set_checked): every call verifies its own output.

* With checked mode on, builds of every method and layout, a refit, the
  traces (device buffers, host buffers, the batch from a CUDA graph), the
  adjoint and the radix sort all pass their checks and return exactly what
  the same calls return with checked mode off.
* A failure surfaces from the call itself: a radix sort whose look-back
  waits may spin only once (the bounded-wait case of the spin-limit test,
  which stays inside its buffers) raises HP_ERR_DEVICE_STATUS from
  radix_sort, not from a later Context.check, and the context stays usable.
* HP_CHECKED=1 in the environment turns checked mode on for a new context.
"""
import numpy as np
import pytest
import torch

import hippie_b200 as hp

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def cctx():
    c = hp.Context(0)
    c.set_checked(True)
    assert c.checked
    yield c
    c.close()


@pytest.fixture(scope="module")
def scene():
    v, t = hp.gen.clustered_mesh(71, 60000, 64, 0.05, 0.004)
    box = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)
    rays = hp.gen.rays_sphere(72, 300000, box)
    return v, t, rays


@pytest.mark.parametrize("method,layout", [("lbvh", 2), ("ploc", 2), ("atr", 2), ("tr", 2), ("hlbvh", 2),
                                           ("lbvh", 4), ("ploc", 8)])
def test_checked_build_and_trace_equal_unchecked(ctx, cctx, scene, method, layout):
    v, t, rays = scene
    V, T, R = dev(v), dev(t), dev(rays)
    p = hp.BuildParams(method=method, morton_bits=60, layout=layout, ploc_radius=8)
    ref = ctx.build(V, T, p)
    got = cctx.build(V, T, p)
    for a, b in zip(ref.download(), got.download()):
        np.testing.assert_array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    np.testing.assert_array_equal(ctx.trace(ref, R).cpu().numpy(), cctx.trace(got, R).cpu().numpy())
    ctx.check()
    cctx.check()


def test_checked_refit_sort_adjoint_and_host_trace(ctx, cctx, scene):
    v, t, rays = scene
    V, T, R = dev(v), dev(t), dev(rays)
    p = hp.BuildParams(method="lbvh", morton_bits=30)
    a, b = ctx.build(V, T, p), cctx.build(V, T, p)
    V2 = dev(v + np.float32(0.001) * np.sin(np.arange(v.size, dtype=np.float32)).reshape(v.shape))
    ctx.refit(a, V2, T)
    cctx.refit(b, V2, T)
    for x, y in zip(a.download(), b.download()):
        np.testing.assert_array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
    res = ctx.trace(a, R)
    np.testing.assert_array_equal(res.cpu().numpy(), cctx.trace_host(b, R.cpu()).cpu().numpy())
    w = dev(np.random.default_rng(3).standard_normal((rays.shape[0], 3)).astype(np.float32))
    g0 = ctx.adjoint(V2, T, R, res, w)
    g1 = cctx.adjoint(V2, T, R, res, w)
    torch.testing.assert_close(g0, g1, rtol=0, atol=1e-4 * float(g0.abs().max()))
    keys = dev(np.random.default_rng(4).integers(0, 1 << 62, size=(1 << 21) + 5, dtype=np.uint64).view(np.int64))
    k0, v0 = ctx.radix_sort(keys, bits=62)
    k1, v1 = cctx.radix_sort(keys, bits=62)
    assert torch.equal(k0, k1) and torch.equal(v0, v1)
    ctx.check()


def test_checked_batch_from_graph(ctx, cctx):
    meshes, counts, rays = [], [], []
    box = np.array([-0.5, -0.5, -0.5, 1.5, 1.5, 1.5], np.float32)
    for m, n in enumerate([300, 5000, 40000, 1200]):
        v, t = hp.gen.uniform_mesh(90 + m, n, 0.01)
        meshes.append((dev(v), dev(t)))
        counts.append(2 * n)
        rays.append(hp.gen.rays_sphere(190 + m, 2 * n, box))
    R = dev(np.concatenate(rays))
    p = hp.BuildParams(method="lbvh", morton_bits=30)
    out = []
    for c in (ctx, cctx):
        batch = hp.Batch(c, meshes, counts, p)
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            res = batch.build_trace(R, results=torch.zeros((batch.num_rays, 4), dtype=torch.int32, device="cuda"))
        s.synchronize()
        out.append(res.cpu().numpy())
        batch.close()
    np.testing.assert_array_equal(out[0], out[1])
    ctx.check()


def test_checked_failure_comes_from_the_call(cctx):
    n = 1 << 24
    rng = np.random.default_rng(5)
    keys = torch.from_numpy(rng.integers(0, 1 << 60, size=n, dtype=np.uint64).view(np.int64)).cuda()
    cctx.check()
    cctx.set_sort_spin_limit(1)
    try:
        with pytest.raises(hp.HPError) as e:
            cctx.radix_sort(keys, bits=60)
        assert e.value.status == 5  # HP_ERR_DEVICE_STATUS
    finally:
        cctx.set_sort_spin_limit(0)
    torch.cuda.synchronize()
    cctx.check()  # the failing call cleared the error word
    ko, vo = cctx.radix_sort(keys, bits=60)
    order = np.argsort(keys.cpu().numpy().view(np.uint64), kind="stable")
    np.testing.assert_array_equal(vo.cpu().numpy(), order.astype(np.int32))


def test_checked_from_environment(monkeypatch):
    monkeypatch.setenv("HP_CHECKED", "1")
    c = hp.Context(0)
    try:
        assert c.checked
    finally:
        c.close()
    monkeypatch.setenv("HP_CHECKED", "0")
    c = hp.Context(0)
    try:
        assert not c.checked
    finally:
        c.close()
