"""Device BVH statistics and validation (HipBVH::getCost, getAvgLeafSize,
getLeafSizeHistogram and validate, rt/bvh/HipBVH.cpp:157-442): statistics
against the downloaded nodes and the oracle's cost; validation accepts every
built BVH and rejects copies with planted faults (all indices kept in range)."""
import ctypes as C

import numpy as np
import pytest
import torch

import hippie_b200 as hp
import oracle
from hippie_b200 import _lib

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def leaf_stats(nodes, num_interior):
    sizes = ~nodes[num_interior:, 14].astype(np.int64)
    hist = np.bincount(sizes[sizes <= 32], minlength=33)[:33] / len(sizes)
    return int(sizes.sum()), sizes.sum() / len(sizes), hist.astype(np.float32)


@pytest.mark.parametrize("method", ["lbvh", "ploc", "atr"])
@pytest.mark.parametrize("n", [1, 2, 1000, 100000])
def test_stats_match_nodes(ctx, method, n):
    v, t = hp.gen.clustered_mesh(11, n, 64, 0.05, 0.01) if n > 2 else hp.gen.uniform_mesh(11, n)
    p = hp.BuildParams(method=method, morton_bits=60)
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, p)
    st = bvh.stats()
    nodes, _, _ = bvh.download()
    ni = bvh.c.num_interior
    s, avg, hist = leaf_stats(nodes, ni)
    assert (st["num_interior"], st["num_leaf"]) == (ni, bvh.c.num_leaf)
    assert st["sum_of_leaf_sizes"] == s == n
    assert st["avg_leaf_size"] == pytest.approx(avg, rel=1e-15)
    assert np.array_equal(np.array(st["leaf_size_histogram"], np.float32), hist)
    want = oracle.cost(nodes, np.array(bvh.c.scene_box[:], np.float32), bvh.c.ct, bvh.c.ci)
    assert st["sah_cost"] == pytest.approx(want, rel=1e-12)
    assert bvh.stats() == st  # fixed summation order: repeated calls agree bit for bit
    assert bvh.cost() == st["sah_cost"]
    assert bvh.validate(V, T)


def test_large_leaves_leave_the_histogram(ctx):
    v, t = hp.gen.clustered_mesh(5, 50000, 16, 0.02, 0.002)
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, hp.BuildParams(method="lbvh", morton_bits=60, ct=60.0, ci=1.0, max_leaf_size=256))
    st = bvh.stats()
    nodes, _, _ = bvh.download()
    sizes = ~nodes[bvh.c.num_interior:, 14]
    assert sizes.max() > 32  # the case under test
    s, avg, hist = leaf_stats(nodes, bvh.c.num_interior)
    assert np.array_equal(np.array(st["leaf_size_histogram"], np.float32), hist)
    assert sum(st["leaf_size_histogram"]) < 1.0 and st["avg_leaf_size"] == pytest.approx(avg, rel=1e-15)
    assert bvh.validate(V, T)


def _validate_copy(ctx, bvh, nodes, tri, V, T):
    """hp_bvh_validate on a copy of the BVH whose nodes and triangle indices live in
    the given host arrays (uploaded); returns (valid, message)."""
    dn, dt = dev(nodes), dev(tri)
    c2 = _lib.hp_bvh()
    C.memmove(C.addressof(c2), C.addressof(bvh.c), C.sizeof(_lib.hp_bvh))
    c2.nodes = dn.data_ptr()
    c2.tri_indices = dt.data_ptr()
    m = hp._mesh(V, T)
    ok = C.c_int32()
    hp.check(hp.load().hp_bvh_validate(ctx.h, C.byref(c2), C.byref(m), C.byref(ok), None))
    torch.cuda.synchronize()
    return bool(ok.value), (hp.load().hp_last_error() or b"").decode()


def test_validate_rejects_planted_faults(ctx):
    v, t = hp.gen.uniform_mesh(3, 5000)
    V, T = dev(v), dev(t)
    bvh = ctx.build(V, T, hp.BuildParams(method="lbvh", morton_bits=30))
    nodes, _, tri = bvh.download()
    ni = bvh.c.num_interior
    assert _validate_copy(ctx, bvh, nodes, tri, V, T)[0]
    interior_child = next(i for i in range(1, ni) if nodes[0, 12] == i or nodes[0, 13] == i)
    leaf = ni + 3

    def wrong_parent(nd, tr):
        nd[interior_child, 15] = (nodes[interior_child, 15] + 1) % ni

    def size_off(nd, tr):
        nd[interior_child, 14] += 1

    def leaf_box(nd, tr):
        for k in (1, 5):  # max x of both stored boxes below the min x
            nd[leaf, k] = np.float32(nd[leaf, k - 1].view(np.float32) - 1.0).view(np.int32)

    def dup_ref(nd, tr):
        tr[0] = tr[1]

    def flag(nd, tr):
        nd[0, 12] = ~nd[0, 12] if nd[0, 12] >= 0 else nd[0, 12]
        nd[0, 13] = ~nd[0, 13] if nd[0, 13] >= 0 else nd[0, 13]

    def twice(nd, tr):
        nd[0, 13] = nd[0, 12]

    cases = [
        (wrong_parent, {"invalid parent index"}),
        (size_off, {"invalid node size"}),
        (leaf_box, {"triangle is not in its leaf box"}),
        (dup_ref, {"triangle not referenced exactly once", "triangle is not in its leaf box"}),
        (flag, {"child leaf flag mismatch"}),
        (twice, {"invalid node size", "node not referenced exactly once", "root size is not the reference count",
                 "child box not enclosed"}),
    ]
    for mutate, messages in cases:
        nd, tr = nodes.copy(), tri.copy()
        mutate(nd, tr)
        ok, msg = _validate_copy(ctx, bvh, nd, tr, V, T)
        assert not ok, mutate.__name__
        assert any(m in msg for m in messages), (mutate.__name__, msg)
    # the original is still valid
    assert bvh.validate(V, T)
