"""The oracle's N-wide collapse (Quad / Oct layouts) against the reference's own
host code (BVH::collapseAdaptiveWide / collapseWide, rt/bvh/BVH.h, with the
breadth-first numbering of BVHConverter::convert): the committed fixtures from
tests/golden/make_wide_fixtures.py always, the live harness (oracle/_ref) on
more cases where it is built. CPU only."""
from pathlib import Path

import numpy as np
import pytest

import hippie_b200 as hp
import oracle
from oracle import ref_harness as R

FIX = Path(__file__).resolve().parent / "golden" / "wide_ref_fixtures.npz"
CASES = {
    "lbvh_quad": (lambda: hp.gen.uniform_mesh(81, 600), "lbvh", 4, 1, 8),
    "lbvh_oct": (lambda: hp.gen.clustered_mesh(82, 700, 16, 0.05, 0.01), "lbvh", 8, 1, 8),
    "ploc_quad": (lambda: hp.gen.clustered_mesh(83, 700, 16, 0.05, 0.01), "ploc", 4, 1, 8),
    "ploc_oct": (lambda: hp.gen.uniform_mesh(84, 600), "ploc", 8, 1, 8),
    "atr_oct": (lambda: hp.gen.clustered_mesh(85, 700, 8, 0.05, 0.01), "atr", 8, 1, 8),
    "lbvh_quad_maxleaf": (lambda: hp.gen.clustered_mesh(86, 700, 8, 0.05, 0.01), "lbvh", 4, 0, 6),
}


def check_tree(nodes, tri, counts, n, width):
    """Structure: every node reached once from the root, parents, sizes, child counts,
    leaf ranges tiling the reference order, each triangle once."""
    ni, nl = counts
    assert nodes.shape[0] == ni + nl
    N = width
    seen = np.zeros(ni + nl, np.int32)
    seen[0] = 1
    covered = np.zeros(n, np.int32)
    stack = [0]
    while stack:
        i = stack.pop()
        nd = nodes[i]
        if nd[8 * N - 5] < 0:
            b, e = nd[4 * N + 2], nd[4 * N + 3]
            assert i >= ni and 0 <= b < e <= n and e - b == ~nd[8 * N - 5]
            covered[b:e] += 1
            continue
        assert i < ni
        k = nd[8 * N - 9]
        assert (1 if n == 1 else 2) <= k <= N
        total = 0
        for c in range(k):
            raw = nd[4 * (N + c) + 2]
            ch = ~raw if raw < 0 else raw
            assert (raw < 0) == (ch >= ni) and nodes[ch, 8 * N - 1] == i
            seen[ch] += 1
            s = nodes[ch, 8 * N - 5]
            total += ~s if s < 0 else s
            stack.append(ch)
        assert total == nd[8 * N - 5]
    assert (seen == 1).all() and (covered == 1).all()
    assert np.array_equal(np.sort(tri), np.arange(n))


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_reference_fixtures(name):
    fx = np.load(FIX)
    mesh, method, width, adaptive, max_leaf = CASES[name]
    v, t = mesh()
    d = oracle.binary_tree(v, t, method)
    nodes, tri, counts = oracle.collapse_wide(t.shape[0], d["left"], d["right"], d["bmin4"], d["bmax4"],
                                              d["sorted_tri"], width, adaptive=adaptive, max_leaf=max_leaf)
    assert counts == tuple(fx[name + "_counts"].tolist())
    assert np.array_equal(nodes, fx[name + "_nodes"])
    assert np.array_equal(tri, fx[name + "_tri"])
    check_tree(nodes, tri, counts, t.shape[0], width)


@pytest.mark.skipif(not R.available(), reason="reference harness not built here")
@pytest.mark.parametrize("method", ["lbvh", "ploc", "atr"])
@pytest.mark.parametrize("width", [4, 8])
def test_oracle_matches_live_reference(method, width):
    rng = np.random.default_rng(7)
    for case in range(4):
        n = int(rng.integers(40, 6000))
        v, t = (hp.gen.uniform_mesh(100 + case, n) if case % 2 else
                hp.gen.clustered_mesh(100 + case, n, int(rng.integers(1, 64)), 0.05, 0.005))
        d = oracle.binary_tree(v, t, method)
        for adaptive, max_leaf in ((1, 8), (0, int(rng.integers(1, 16)))):
            args = (n, d["left"], d["right"], d["bmin4"], d["bmax4"], d["sorted_tri"], width)
            ref = R.wide_collapse(*args, adaptive=adaptive, max_leaf=max_leaf)
            if ref is None:  # root best as a leaf: undefined in the reference
                continue
            got = oracle.collapse_wide(*args, adaptive=adaptive, max_leaf=max_leaf)
            assert got[2] == ref[2]
            assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 17])
def test_small_meshes(width, n):
    v, t = hp.gen.uniform_mesh(9, n)
    b = oracle.build_wide(v, t, width)
    check_tree(b["nodes"], b["tri_idx"], tuple(b["counts"].tolist()), n, width)
