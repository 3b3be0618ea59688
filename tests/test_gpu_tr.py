"""TRBVH (treelet restructuring by dynamic programming over 7-leaf treelets,
TRBuilder) on the GPU against the CPU oracle: bit-exact nodes, triangle order
and Woop triangles, sm_100a. (The reference's own TRBVH kernels are not run:
see the parity notes of the design document.)"""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def canonical(nodes, tri_idx):
    out = []
    stack = [0]
    while stack:
        i = stack.pop()
        c0, c1, size, _ = nodes[i, 12:16]
        if size < 0:
            out.append(("L", tuple(nodes[i, :12].tolist()), tuple(sorted(tri_idx[c0:c1].tolist()))))
        else:
            out.append(("I", tuple(nodes[i, :12].tolist()), int(size)))
            stack.append(~c1 if c1 < 0 else c1)
            stack.append(~c0 if c0 < 0 else c0)
    return out


def _mesh(kind, n, seed):
    if kind == "uniform":
        return hp.gen.uniform_mesh(seed, n)
    if kind == "clustered":
        return hp.gen.clustered_mesh(seed, n, clusters=max(1, n // 4096))
    v1, t1 = hp.gen.uniform_mesh(seed, n // 2)
    v2, t2 = hp.gen.clustered_mesh(seed + 1, n - n // 2, clusters=max(1, n // 8192))
    return np.concatenate([v1, v2]), np.concatenate([t1, t2 + v1.shape[0]]).astype(np.int32)


@pytest.mark.parametrize("kind,n,bits,iters", [
    ("uniform", 8, 60, 2), ("clustered", 100, 60, 2), ("uniform", 50000, 30, 2), ("clustered", 131072, 60, 2),
    ("mixed", 200000, 60, 3), ("clustered", 20000, 60, 0), ("uniform", 30000, 60, 1),
])
def test_tr_bit_exact_vs_oracle(ctx, kind, n, bits, iters):
    v, t = _mesh(kind, n, 300 + n)
    bvh = ctx.build(dev(v), dev(t), hp.BuildParams(method="tr", morton_bits=bits, atr_iterations=iters))
    bvh.sync()
    ctx.check()
    nodes, woop, tri = bvh.download()
    ref = oracle.build_tr(v, t, bits=bits, iterations=iters, scale=np.array(bvh.c.morton_scale, np.float32))
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(woop.view(np.int32), ref["woop"].view(np.int32))


def test_tr_lowers_cost_and_traces(ctx):
    v, t = _mesh("mixed", 300000, 7)
    V, T = dev(v), dev(t)
    lb = ctx.build(V, T, hp.BuildParams(method="lbvh", morton_bits=60))
    tr = ctx.build(V, T, hp.BuildParams(method="tr", morton_bits=60))
    assert tr.cost() < lb.cost()
    assert tr.validate(V, T)
    rays = dev(hp.gen.rays_sphere(8, 1 << 17, np.concatenate([v.min(0), v.max(0)])))
    r1 = ctx.trace(lb, rays, results=torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda"))
    r2 = ctx.trace(tr, rays, results=torch.zeros((rays.shape[0], 4), dtype=torch.int32, device="cuda"))
    np.testing.assert_array_equal(r1.cpu().numpy(), r2.cpu().numpy())


def test_tr_from_env(ctx):
    p = hp.Env().read_string("Bvh { method tr\n trIterations 3\n trMortonCodeBits 30 }").build_params()
    assert (p.method, p.atr_iterations, p.morton_bits) == (3, 3, 30)
    v, t = _mesh("uniform", 20000, 9)
    bvh = ctx.build(dev(v), dev(t), p)
    bvh.sync()
    ref = oracle.build_tr(v, t, bits=30, iterations=3, scale=np.array(bvh.c.morton_scale, np.float32))
    np.testing.assert_array_equal(bvh.download()[0], ref["nodes"])


@pytest.mark.parametrize("layout", [4, 8])
def test_tr_wide_layouts(ctx, layout):
    v, t = _mesh("clustered", 30000, 11)
    bvh = ctx.build(dev(v), dev(t), hp.BuildParams(method="tr", morton_bits=60, layout=layout))
    bvh.sync()
    ref = oracle.build_wide(v, t, layout, method="tr", bits=60, iterations=2,
                            scale=np.array(bvh.c.morton_scale, np.float32))
    np.testing.assert_array_equal(bvh.download()[0], ref["nodes"])
