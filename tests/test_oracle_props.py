"""Properties of the CPU oracle on synthetic scenes (CPU only)."""
import numpy as np
import pytest

import hippie_b200 as hp
import oracle


def _mesh(n, seed=1):
    return hp.gen.uniform_mesh(seed, n)


def test_sort_is_stable_sort():
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 12, size=20000).astype(np.uint64)  # many duplicates
    sk, sr = oracle.sort(keys, 12)
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(sr, order)
    np.testing.assert_array_equal(sk, keys[order])


@pytest.mark.parametrize("n", [2, 3, 7, 100, 1000])
def test_karras_topology_invariants(n):
    v, t = _mesh(n, seed=n)
    bmin, bmax, box = oracle.tri_boxes(v, t)
    keys, _ = oracle.morton(bmin, bmax, box, 30)
    sk, sr = oracle.sort(keys, 30)
    parent, left, right = oracle.karras(sk)
    nn = 2 * n - 1
    assert parent[0] == -1
    counts = np.zeros(nn, int)
    for i in range(n - 1):
        for c in (left[i], right[i]):
            assert 0 < c < nn
            assert parent[c] == i
            counts[c] += 1
    assert counts[0] == 0 and np.all(counts[1:] == 1)
    # leaves in order: an in-order walk visits leaves 0..n-1
    out = []
    stack = [0]
    while stack:
        x = stack.pop()
        if x >= n - 1:
            out.append(x - (n - 1))
        else:
            stack += [right[x], left[x]]
    assert out == list(range(n))


def test_duplicate_keys_tree():
    """All triangles at the same place: every key equal, ties broken by index."""
    n = 64
    v = np.tile(np.array([[0.5, 0.5, 0.5], [0.51, 0.5, 0.5], [0.5, 0.51, 0.5]], np.float32), (n, 1))
    t = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    r = oracle.build_lbvh(v, t, bits=30)
    assert r["counts"].sum() == r["nodes"].shape[0]
    _check_bin_tree(r["nodes"], r["counts"], r["tri_idx"], v, t)


def _check_bin_tree(nodes, counts, tri_idx, v, t):
    n_int, n_leaf = int(counts[0]), int(counts[1])
    assert nodes.shape[0] == n_int + n_leaf
    f = nodes[:, :12].view(np.float32)
    seen = np.zeros(nodes.shape[0], int)
    seen[0] = 1
    tris_seen = np.zeros(t.shape[0], int)
    stack = [0]
    while stack:
        i = stack.pop()
        c0, c1, size, par = nodes[i, 12:16]
        if size >= 0:
            assert i < n_int
            s = 0
            for raw, slot in ((c0, 0), (c1, 1)):
                c = ~raw if raw < 0 else raw
                assert nodes[c, 15] == i
                s += ~nodes[c, 14] if nodes[c, 14] < 0 else nodes[c, 14]
                seen[c] += 1
                stack.append(c)
            assert s == size
        else:
            assert i >= n_int
            b, e = c0, c1
            assert e - b == ~size
            mn = np.array([f[i, 0], f[i, 2], f[i, 8]])
            mx = np.array([f[i, 1], f[i, 3], f[i, 9]])
            for r in range(b, e):
                tris_seen[tri_idx[r]] += 1
                p = v[t[tri_idx[r]]]
                assert np.all(p >= mn) and np.all(p <= mx)
    assert np.all(seen == 1)
    assert np.all(tris_seen == 1)


@pytest.mark.parametrize("n,bits", [(2, 30), (3, 60), (50, 30), (2000, 60), (5000, 30)])
def test_lbvh_build_valid(n, bits):
    v, t = _mesh(n, seed=11 + n)
    r = oracle.build_lbvh(v, t, bits=bits)
    _check_bin_tree(r["nodes"], r["counts"], r["tri_idx"], v, t)
    c = oracle.cost(r["nodes"], r["box"])
    assert c > 0


def test_refit_matches_brute_force_boxes():
    n = 500
    v, t = _mesh(n, seed=5)
    bmin, bmax, box = oracle.tri_boxes(v, t)
    keys, _ = oracle.morton(bmin, bmax, box, 60)
    sk, sr = oracle.sort(keys, 60)
    parent, left, right = oracle.karras(sk)
    nbmin, nbmax, size, cost, state = oracle.refit(v, t, sr, parent, left, right)
    # brute force: box of node = union of the triangle boxes of its leaves
    def leaves(x):
        if x >= n - 1:
            return [x - (n - 1)]
        return leaves(left[x]) + leaves(right[x])
    for x in [0, 1, 5, n // 2, n - 2]:
        ls = leaves(x)
        tb = np.concatenate([v[t[sr[p]]] for p in ls])
        np.testing.assert_array_equal(nbmin[x, :3], tb.min(0))
        np.testing.assert_array_equal(nbmax[x, :3], tb.max(0))
        assert size[x] == len(ls)


def test_trace_matches_brute_force_double():
    n = 3000
    v, t = _mesh(n, seed=9)
    r = oracle.build_lbvh(v, t, bits=30)
    rays = hp.gen.rays_targeted(21, 4000)
    res = oracle.trace(r["nodes"], r["woop"], r["tri_idx"], rays)
    bf = oracle.brute64(v, t, rays)
    hit = res[:, 0] >= 0
    bhit = bf[:, 0] >= 0
    # hit/miss agreement except grazing rays
    assert np.mean(hit == bhit) > 0.999
    both = hit & bhit
    same = res[both, 0] == bf[both, 0].astype(np.int32)
    assert np.mean(same) > 0.999
    t32 = res[both, 1].view(np.float32)
    rel = np.abs(t32 - bf[both, 1]) / np.maximum(1.0, np.abs(bf[both, 1]))
    assert np.median(rel) < 1e-6


def test_trace_stats_and_any_hit():
    v, t = _mesh(500, seed=2)
    r = oracle.build_lbvh(v, t, bits=30)
    rays = hp.gen.rays_targeted(4, 1000)
    res, st = oracle.trace(r["nodes"], r["woop"], r["tri_idx"], rays, stats=True)
    hit = res[:, 0] >= 0
    assert np.all(st[hit, 0] > 0) and np.all(st[hit, 1] > 0)
    assert np.all(st[~hit] == 0)
    anyres = oracle.trace(r["nodes"], r["woop"], r["tri_idx"], rays, any_hit=True)
    np.testing.assert_array_equal(anyres[:, 0] >= 0, hit)


def test_empty_and_single():
    v = np.zeros((0, 3), np.float32)
    t = np.zeros((0, 3), np.int32)
    r = oracle.build_lbvh(v, t)
    assert r["nodes"].shape[0] == 0
    rays = hp.gen.rays_targeted(1, 10)
    res = oracle.trace(r["nodes"], np.zeros((0, 12), np.float32), np.zeros(0, np.int32), rays)
    assert np.all(res[:, 0] == -1)
    v1 = np.array([[0, 0, 0.5], [1, 0, 0.5], [0, 1, 0.5]], np.float32)
    t1 = np.array([[0, 1, 2]], np.int32)
    r1 = oracle.build_lbvh(v1, t1)
    assert r1["counts"].tolist() == [1, 2]
    ray = np.array([[0.2, 0.2, 2.0, 0.0, 0.0, 0.0, -1.0, np.inf]], np.float32)
    res1 = oracle.trace(r1["nodes"], r1["woop"], r1["tri_idx"], ray)
    assert res1[0, 0] == 0


@pytest.mark.parametrize("n", [2, 3, 64, 3000])
def test_ploc_oracle_tree_valid(n):
    v, t = hp.gen.clustered_mesh(n, n, clusters=max(1, n // 64))
    r = oracle.build_ploc(v, t, radius=4, max_radius=64)
    _check_bin_tree(r["nodes"], r["counts"], r["tri_idx"], v, t)
    # preorder: the left child of an interior node is the next node
    nodes, n_int = r["nodes"], r["counts"][0]
    for i in range(n_int):
        c0 = nodes[i, 12]
        if c0 >= 0:
            assert c0 == i + 1
    if n > 100:
        lb = oracle.build_lbvh(v, t, bits=60)
        assert oracle.cost(r["nodes"], r["box"]) < oracle.cost(lb["nodes"], lb["box"])


def test_canonical_form_ignores_numbering():
    """oracle.canonical: the depth-first form of a collapsed tree does not change
    when interior nodes are renumbered or a leaf's triangles are reordered, and
    it matches a direct walk of the tree."""
    import hippie_b200 as hp
    v, t = hp.gen.clustered_mesh(21, 5000, clusters=16)
    r = oracle.build_ploc(v, t, radius=4, max_radius=64)
    nodes, tri = r["nodes"], r["tri_idx"]
    rows, tris = oracle.canonical(nodes, tri)
    assert rows.shape[0] == nodes.shape[0]
    assert sorted(tris.tolist()) == list(range(t.shape[0]))
    # renumber interior nodes 1.. in reverse and reverse every leaf's triangles
    n_int = int(r["counts"][0])
    perm = np.arange(nodes.shape[0])
    perm[1:n_int] = perm[1:n_int][::-1]
    new = np.empty_like(nodes)
    new[perm] = nodes
    for i in range(new.shape[0]):
        for k in (12, 13):
            c = new[i, k]
            if new[i, 14] >= 0 and 0 <= c < n_int:
                new[i, k] = perm[c]
        if new[i, 15] >= 0:
            new[i, 15] = perm[new[i, 15]]
    tri2 = tri.copy()
    for i in range(new.shape[0]):
        if new[i, 14] < 0:
            b, e = new[i, 12], new[i, 13]
            tri2[b:e] = tri2[b:e][::-1]
    rows2, tris2 = oracle.canonical(new, tri2)
    np.testing.assert_array_equal(rows, rows2)
    np.testing.assert_array_equal(tris, tris2)
    with pytest.raises(ValueError):
        bad = nodes.copy()
        bad[0, 12] = nodes.shape[0] + 5
        oracle.canonical(bad, tri)
