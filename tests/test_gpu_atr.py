"""ATR treelet restructuring on the GPU against the CPU oracle (bit-exact nodes,
triangle order and Woop triangles) and against the reference's own ATR kernels
(canonical trees), sm_100a."""
import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle
from oracle import ref_harness as R

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


@pytest.mark.parametrize("kind,n,bits,treelet,iters", [
    ("uniform", 50000, 30, 9, 2),
    ("clustered", 131072, 60, 9, 2),
    ("mixed", 200000, 60, 9, 2),
    ("uniform", 30000, 60, 20, 2),
    ("clustered", 40000, 60, 4, 3),
    ("uniform", 20000, 30, 30, 1),
    ("clustered", 20000, 60, 9, 0),
])
def test_atr_bit_exact_vs_oracle(ctx, kind, n, bits, treelet, iters):
    v, t = _mesh(kind, n, 100 + n)
    bvh = ctx.build(dev(v), dev(t), hp.BuildParams(method="atr", morton_bits=bits, atr_treelet=treelet,
                                                   atr_iterations=iters))
    bvh.sync()
    ctx.check()
    nodes, woop, tri = bvh.download()
    ref = oracle.build_atr(v, t, bits=bits, treelet=treelet, iterations=iters,
                           scale=np.array(bvh.c.morton_scale, np.float32))
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    np.testing.assert_array_equal(nodes, ref["nodes"])
    np.testing.assert_array_equal(tri, ref["tri_idx"])
    np.testing.assert_array_equal(woop, ref["woop"])
    assert bvh.validate(dev(v), dev(t))


def test_atr_lowers_cost_and_traces(ctx):
    v, t = _mesh("mixed", 262144, 7)
    V, T = dev(v), dev(t)
    lb = ctx.build(V, T, hp.BuildParams(method="lbvh", morton_bits=60))
    at = ctx.build(V, T, hp.BuildParams(method="atr", morton_bits=60, atr_treelet=9, atr_iterations=2))
    assert at.cost() < lb.cost()
    rays = hp.gen.rays_sphere(8, 1 << 18, np.concatenate([v.min(0), v.max(0)]))
    got = ctx.trace(at, dev(rays)).cpu().numpy()
    nodes, woop, tri = at.download()
    np.testing.assert_array_equal(got, oracle.trace(nodes, woop, tri, rays))
    ref_lb = ctx.trace(lb, dev(rays)).cpu().numpy()
    # same closest hits through either tree, up to ties in t
    same = (got[:, 0] == ref_lb[:, 0]) | (got[:, 1] == ref_lb[:, 1])
    assert np.mean(same) > 0.9999


def test_atr_from_env(ctx):
    env = hp.Env().read_string("Bvh {\n method atr\n atrMortonCodeBits 60\n atrIterations 2\n atrTreeletSize 9\n}\n")
    p = env.build_params()
    assert p.method == hp.HP_METHOD_ATR and p.atr_treelet == 9 and p.atr_iterations == 2
    v, t = _mesh("uniform", 10000, 9)
    bvh = ctx.build(dev(v), dev(t), p)
    bvh.sync()
    ref = oracle.build_atr(v, t, bits=60, treelet=9, iterations=2, scale=np.array(bvh.c.morton_scale, np.float32))
    np.testing.assert_array_equal(bvh.download()[0], ref["nodes"])


@pytest.mark.skipif(not R.available(), reason="reference harness not built (needs the reference sources)")
@pytest.mark.parametrize("kind,n,bits,treelet", [("uniform", 65536, 30, 9), ("clustered", 131072, 60, 9),
                                                 ("mixed", 100000, 60, 20)])
def test_atr_matches_reference_kernels(ctx, kind, n, bits, treelet):
    v, t = _mesh(kind, n, 200 + n)
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, hp.BuildParams(method="atr", morton_bits=bits, atr_treelet=treelet, atr_iterations=2))
    bvh.sync()
    box = np.array(bvh.c.scene_box, np.float32)
    ref = R.build(V, T, box, method="atr", bits=bits, treelet=treelet, iterations=2)
    nodes, woop, tri = bvh.download()
    assert (bvh.c.num_interior, bvh.c.num_leaf) == tuple(ref["counts"].tolist())
    assert canonical(nodes, tri) == canonical(ref["nodes"], ref["tri_idx"])
