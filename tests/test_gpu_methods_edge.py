"""Every builder (LBVH, PLOC, ATR, TRBVH, HLBVH) in every layout on tiny and
degenerate meshes against the oracle: empty, one to five triangles, and
triangles sharing one centroid (sm_100a)."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu

GPU = {"lbvh": {}, "ploc": dict(ploc_radius=16, ploc_max_radius=256, ploc_adaptive=0),
       "atr": dict(atr_treelet=9, atr_iterations=2), "tr": dict(atr_iterations=2), "hlbvh": dict(hlbvh_sah_bits=15)}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def oracle_build(method, v, t, scale, layout):
    if layout != 2:
        kw = dict(radius=16, max_radius=256, treelet=9, iterations=2, sah_bits=15)
        return oracle.build_wide(v, t, layout, method=method, bits=60, scale=scale, **kw)
    if method == "lbvh":
        return oracle.build_lbvh(v, t, bits=60, scale=scale)
    if method == "ploc":
        return oracle.build_ploc(v, t, bits=60, radius=16, max_radius=256, adaptive_r=0, scale=scale)
    if method == "atr":
        return oracle.build_atr(v, t, bits=60, treelet=9, iterations=2, scale=scale)
    if method == "tr":
        return oracle.build_tr(v, t, bits=60, iterations=2, scale=scale)
    return oracle.build_hlbvh(v, t, bits=60, sah_bits=15, scale=scale)


def check(ctx, method, layout, v, t, trace=True):
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, hp.BuildParams(method=method, morton_bits=60, layout=layout, **GPU[method]))
    bvh.sync()
    ctx.check()
    ref = oracle_build(method, v, t, np.array(bvh.c.morton_scale, np.float32), layout)
    nodes, woop, tri = bvh.download()
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    if t.shape[0]:
        assert bvh.validate(V, T)
    if trace and layout == 2:
        rays = hp.gen.rays_targeted(3, 4096)
        res = ctx.trace(bvh, dev(rays), results=torch.zeros((4096, 4), dtype=torch.int32, device="cuda"))
        np.testing.assert_array_equal(res.cpu().numpy(), oracle.trace(ref["nodes"], ref["woop"], ref["tri_idx"], rays))


@pytest.mark.parametrize("method", list(GPU))
@pytest.mark.parametrize("layout", [2, 4, 8])
@pytest.mark.parametrize("n", [0, 1, 2, 3, 5])
def test_tiny_meshes(ctx, method, layout, n):
    v, t = hp.gen.uniform_mesh(90 + n, n)
    check(ctx, method, layout, v, t)


@pytest.mark.parametrize("method", list(GPU))
@pytest.mark.parametrize("layout", [2, 8])
def test_shared_centroids(ctx, method, layout):
    """2,000 triangles around one centroid plus 50 elsewhere: long runs of equal
    Morton keys (index tie-break), treelets of equal boxes, one HLBVH cell
    holding almost everything."""
    n = 2050
    base = np.array([[0.5, 0.5, 0.5], [0.52, 0.5, 0.5], [0.5, 0.52, 0.5]], np.float32)
    v = np.tile(base, (n, 1))
    v[: 3 * 50] += np.repeat(np.linspace(0.1, 0.4, 50, dtype=np.float32), 3)[:, None]
    t = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    check(ctx, method, layout, v, t, trace=False)
