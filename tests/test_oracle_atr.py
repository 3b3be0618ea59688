"""CPU oracle of ATR treelet restructuring (ATRBuilder, rt/bvh/ATRBuilder.cpp:80-236):
structural properties and the reduction tie rules it restates."""
import numpy as np
import pytest

import hippie_b200 as hp
import oracle


def _leaf_sets(nodes, tri_idx):
    sets = []
    for row in nodes:
        if row[14] < 0:
            sets.append(tuple(sorted(tri_idx[row[12]:row[13]].tolist())))
    return sets


def _check_bvh(r, n):
    nodes, tri = r["nodes"], r["tri_idx"]
    ni, nl = r["counts"]
    assert nodes.shape[0] == ni + nl
    assert sorted(tri.tolist()) == list(range(n))
    # every node but the root is referenced exactly once; leaf ranges tile [0, n)
    seen = np.zeros(ni + nl, np.int32)
    covered = 0
    for i in range(ni):
        for c in nodes[i, 12:14]:
            seen[~c if c < 0 else c] += 1
    assert seen[0] == 0 and np.all(seen[1:] == 1)
    for row in nodes[ni:]:
        covered += row[13] - row[12]
        assert row[14] == ~(row[13] - row[12])
    assert covered == n


@pytest.mark.parametrize("treelet", [4, 9, 20, 30])
def test_atr_valid_and_not_worse(treelet):
    v, t = hp.gen.uniform_mesh(11, 6000)
    base = oracle.build_lbvh(v, t, bits=60)
    r = oracle.build_atr(v, t, bits=60, treelet=treelet, iterations=2)
    _check_bvh(r, t.shape[0])
    box = base["box"]
    assert oracle.cost(r["nodes"], box) <= oracle.cost(base["nodes"], box) * (1 + 1e-6)


def test_atr_zero_iterations_is_lbvh():
    v, t = hp.gen.clustered_mesh(12, 5000, 16)
    base = oracle.build_lbvh(v, t, bits=30)
    r = oracle.build_atr(v, t, bits=30, treelet=9, iterations=0)
    assert tuple(r["counts"]) == tuple(base["counts"])
    assert sorted(_leaf_sets(r["nodes"], r["tri_idx"])) == sorted(_leaf_sets(base["nodes"], base["tri_idx"]))
    assert oracle.cost(r["nodes"], base["box"]) == pytest.approx(oracle.cost(base["nodes"], base["box"]), rel=1e-12)


def test_atr_improves_clustered_scene():
    v, t = hp.gen.clustered_mesh(13, 20000, 64)
    base = oracle.build_lbvh(v, t, bits=60)
    r = oracle.build_atr(v, t, bits=60, treelet=9, iterations=2)
    box = base["box"]
    assert oracle.cost(r["nodes"], box) < 0.99 * oracle.cost(base["nodes"], box)


def test_atr_duplicate_triangles():
    """Equal boxes make equal union areas: the warp reductions' tie rules decide."""
    v, t = hp.gen.uniform_mesh(14, 1000)
    v = np.concatenate([v, v, v])
    t = np.concatenate([t, t + 3000, t + 6000]).astype(np.int32)
    r = oracle.build_atr(v, t, bits=30, treelet=9, iterations=3)
    _check_bvh(r, t.shape[0])
    r2 = oracle.build_atr(v, t, bits=30, treelet=9, iterations=3)
    np.testing.assert_array_equal(r["nodes"], r2["nodes"])


def test_atr_small_meshes():
    for n in (2, 3, 5, 9, 17):
        v, t = hp.gen.uniform_mesh(15 + n, n)
        r = oracle.build_atr(v, t, bits=60, treelet=9, iterations=2)
        _check_bvh(r, n)
