"""HLBVH (LBVH clusters below the top Morton bits, a binned-SAH top tree over
them: HLBVHBuilder) on the GPU against the CPU oracle (bit-exact nodes,
triangle order and Woop triangles) and against the reference's own HLBVH
kernels where the reference harness is built (sm_100a)."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle
from oracle import ref_harness as R
from hlbvh_cases import canonical

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _mesh(kind, n, seed):
    if kind == "uniform":
        return hp.gen.uniform_mesh(seed, n)
    if kind == "clustered":
        return hp.gen.clustered_mesh(seed, n, clusters=max(1, n // 4096))
    v1, t1 = hp.gen.uniform_mesh(seed, n // 2)
    v2, t2 = hp.gen.clustered_mesh(seed + 1, n - n // 2, clusters=max(1, n // 8192))
    return np.concatenate([v1, v2]), np.concatenate([t1, t2 + v1.shape[0]]).astype(np.int32)


def _normalised(v):
    """The reference's scene loader scales scenes into [0, 1]^3 (SceneLoader.cpp:136-140)."""
    lo, hi = v.min(0), v.max(0)
    return ((v - lo) / (hi - lo).max()).astype(np.float32)


def oracle_singleton_scene():
    """A uniform scene plus one triangle alone far beyond its maximum corner."""
    v, t = hp.gen.uniform_mesh(5, 400)
    lo, hi = v.min(0), v.max(0)
    far = hi + 0.5 * (hi - lo) + np.array([[0, 0, 0], [0.01, 0, 0], [0, 0.01, 0]], np.float32)
    v = np.concatenate([v, far.astype(np.float32)])
    t = np.concatenate([t, np.array([[len(v) - 3, len(v) - 2, len(v) - 1]], np.int32)])
    return v, t


def build(ctx, v, t, **kw):
    bvh = ctx.build(dev(v), dev(t), hp.BuildParams(method="hlbvh", **kw))
    bvh.sync()
    ctx.check()
    return bvh


@pytest.mark.parametrize("kind,n,bits,sah", [
    ("uniform", 2, 60, 15), ("uniform", 3, 60, 15), ("clustered", 17, 60, 6), ("uniform", 100, 60, 9),
    ("clustered", 1000, 60, 15), ("uniform", 50000, 30, 12), ("clustered", 131072, 60, 15),
    ("mixed", 200000, 60, 9), ("mixed", 300000, 60, 15), ("uniform", 40000, 60, 6),
])
def test_hlbvh_bit_exact_vs_oracle(ctx, kind, n, bits, sah):
    v, t = _mesh(kind, n, 400 + n)
    bvh = build(ctx, v, t, morton_bits=bits, hlbvh_sah_bits=sah)
    nodes, woop, tri = bvh.download()
    ref = oracle.build_hlbvh(v, t, bits=bits, sah_bits=sah, scale=np.array(bvh.c.morton_scale, np.float32))
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(woop.view(np.int32), ref["woop"].view(np.int32))
    assert bvh.validate(dev(v), dev(t))


def test_hlbvh_singleton_last_cell(ctx):
    """A leaf cluster at the last sorted position bins with key 0's cell and ends
    paired with the first cluster by the object-median fallback."""
    v, t = oracle_singleton_scene()
    bvh = build(ctx, v, t, morton_bits=60, hlbvh_sah_bits=15)
    ref = oracle.build_hlbvh(v, t, bits=60, sah_bits=15, scale=np.array(bvh.c.morton_scale, np.float32))
    nodes, _, tri = bvh.download()
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(tri, ref["tri_idx"])


def test_hlbvh_root_in_one_cell_keeps_lbvh(ctx):
    """Every key sharing the top SAH bits: the LBVH is kept."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.001, 0.001, 0], [1.001, 0, 0], [0, 1.001, 0]], np.float32)
    t = np.array([[0, 1, 2], [3, 4, 5]], np.int32)
    hl = build(ctx, v, t, morton_bits=60, hlbvh_sah_bits=15)
    lb = ctx.build(dev(v), dev(t), hp.BuildParams(method="lbvh", morton_bits=60))
    lb.sync()
    np.testing.assert_array_equal(hl.download()[0], lb.download()[0])


def test_hlbvh_traces_like_lbvh(ctx):
    v, t = _mesh("mixed", 300000, 7)
    V, T = dev(v), dev(t)
    lb = ctx.build(V, T, hp.BuildParams(method="lbvh", morton_bits=60))
    hl = ctx.build(V, T, hp.BuildParams(method="hlbvh", morton_bits=60))
    assert hl.validate(V, T)
    rays = hp.gen.rays_sphere(8, 1 << 17, np.concatenate([v.min(0), v.max(0)]))
    R_ = dev(rays)
    r1 = ctx.trace(lb, R_, results=torch.zeros((R_.shape[0], 4), dtype=torch.int32, device="cuda")).cpu().numpy()
    r2 = ctx.trace(hl, R_, results=torch.zeros((R_.shape[0], 4), dtype=torch.int32, device="cuda")).cpu().numpy()
    np.testing.assert_array_equal(r1, r2)
    nodes, woop, tri = hl.download()
    np.testing.assert_array_equal(r2[:4096], oracle.trace(nodes, woop, tri, rays[:4096]))


def test_hlbvh_from_env(ctx):
    p = hp.Env().read_string("Bvh { method hlbvh\n hlbvhMortonCodeBits 30\n hlbvhMortonCodeSAHBits 12 }").build_params()
    v, t = _mesh("uniform", 20000, 9)
    bvh = ctx.build(dev(v), dev(t), p)
    bvh.sync()
    ref = oracle.build_hlbvh(v, t, bits=30, sah_bits=12, scale=np.array(bvh.c.morton_scale, np.float32))
    np.testing.assert_array_equal(bvh.download()[0], ref["nodes"])


def test_hlbvh_rejects_sah_bits(ctx):
    v, t = _mesh("uniform", 1000, 3)
    for sah, status in ((7, 6), (16, 2), (5, 2)):
        with pytest.raises(hp.HPError) as ei:
            ctx.build(dev(v), dev(t), hp.BuildParams(method="hlbvh", hlbvh_sah_bits=sah))
        assert ei.value.status == status
    with pytest.raises(hp.HPError):
        ctx.build(dev(v), dev(t), hp.BuildParams(method="hlbvh", morton_bits=12, hlbvh_sah_bits=15))


@pytest.mark.parametrize("layout", [4, 8])
def test_hlbvh_wide_layouts(ctx, layout):
    v, t = _mesh("clustered", 30000, 11)
    bvh = build(ctx, v, t, morton_bits=60, layout=layout)
    ref = oracle.build_wide(v, t, layout, method="hlbvh", bits=60, sah_bits=15,
                            scale=np.array(bvh.c.morton_scale, np.float32))
    np.testing.assert_array_equal(bvh.download()[0], ref["nodes"])
    assert bvh.validate(dev(v), dev(t))


@pytest.mark.skipif(not R.available(), reason="reference harness not built (needs the reference sources)")
@pytest.mark.parametrize("kind,n,bits,sah", [("uniform", 65536, 60, 15), ("clustered", 131072, 60, 15),
                                             ("mixed", 100000, 60, 9), ("uniform", 30000, 30, 12),
                                             ("clustered", 5000, 60, 6), ("singleton", 401, 60, 15)])
def test_hlbvh_matches_reference_kernels(ctx, kind, n, bits, sah):
    v, t = oracle_singleton_scene() if kind == "singleton" else _mesh(kind, n, 500 + n)
    v = _normalised(v)
    V, T = dev(v), dev(t)
    bvh = build(ctx, v, t, morton_bits=bits, hlbvh_sah_bits=sah)
    box = np.array(bvh.c.scene_box, np.float32)
    ref = R.build(V, T, box, method="hlbvh", bits=bits, sah_bits=sah)
    nodes, woop, tri = bvh.download()
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    order = oracle.binary_tree(v, t, method="lbvh", bits=bits, scale=np.array(bvh.c.morton_scale, np.float32))
    assert canonical(nodes, tri, order["sorted_tri"]) == canonical(ref["nodes"], ref["tri_idx"], order["sorted_tri"])
