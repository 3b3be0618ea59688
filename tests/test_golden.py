"""Oracle against the hand-derived known-answer vectors in tests/golden/ (CPU only).

The reference has no tests or fixtures of its own; tests/golden/make_golden.py
derives these vectors from the reference's formulas and from Karras 2012.
"""
import json
from pathlib import Path

import numpy as np

import oracle

G = Path(__file__).resolve().parent / "golden"
UNIT_BOX = np.array([0, 0, 0, 1, 1, 1], np.float32)


def _key_of_point(x, y, z, bits=60):
    """Morton key the oracle assigns to integer grid point (x, y, z) of the 20-bit grid.

    The centroid (q + 0.25) / 1048575 in a unit scene box with scale 1 quantises to q:
    every rounding error is below 0.1 of a grid cell, so truncation is unambiguous.
    """
    c = ((np.array([x, y, z], np.float64) + 0.25) / 1048575.0).astype(np.float32)
    box = np.array([[c[0], c[1], c[2], 0]], np.float32)
    keys, _ = oracle.morton(box, box.copy(), UNIT_BOX, bits, scale=[1.0, 1.0, 1.0])
    return int(keys[0])


def test_morton_codes_vs_table():
    kat = json.loads((G / "morton_kat.json").read_text())
    checked = 0
    for e in kat["codes"]:
        x, y, z = e["xyz"]
        if max(x, y, z) > 1048575:
            continue
        assert _key_of_point(x, y, z) == e["code60"], e
        assert _key_of_point(x, y, z, bits=30) == e["code60"] >> 30, e
        assert _key_of_point(x, y, z, bits=17) == e["code60"] >> 43, e
        checked += 1
    assert checked >= 70


def test_morton_quantisation():
    kat = json.loads((G / "morton_kat.json").read_text())
    codes = {}
    for e in kat["codes"]:
        codes[tuple(e["xyz"])] = e["code60"]
    for q in kat["quant"]:
        c = np.float32(q["centroid"])
        box = np.array([[c, c, c, 0]], np.float32)
        keys, _ = oracle.morton(box, box.copy(), UNIT_BOX, 60, scale=[1.0, 1.0, 1.0])
        v = q["q"]
        expect = 0
        for b in range(20):
            expect |= ((v >> b) & 1) * (0b111 << (3 * b))
        assert int(keys[0]) == expect, q


def test_karras_paper_example():
    kat = json.loads((G / "karras_kat.json").read_text())
    keys = np.array(kat["keys"], np.uint64)
    parent, left, right = oracle.karras(keys)
    assert parent.tolist() == kat["parent"]
    assert left.tolist() == kat["left"]
    assert right.tolist() == kat["right"]


def test_woop_known_answers():
    kat = json.loads((G / "woop_kat.json").read_text())
    verts = np.array([p for t in kat["triangles"] for p in t["v"]], np.float32)
    tris = np.arange(verts.shape[0], dtype=np.int32).reshape(-1, 3)
    tri_idx = np.arange(tris.shape[0], dtype=np.int32)
    woop = np.zeros((tris.shape[0], 12), np.float32)
    oracle.load().or_woopify(tris.shape[0], verts.ctypes.data, tris.ctypes.data, tri_idx.ctypes.data,
                             woop.ctypes.data)
    for i, t in enumerate(kat["triangles"]):
        np.testing.assert_array_equal(woop[i], np.array(t["w"], np.float32).reshape(-1))


def test_ray_known_answers():
    """Woop traversal of each known-answer triangle gives the exact (t, u, v)."""
    kat = json.loads((G / "woop_kat.json").read_text())
    for r in kat["rays"]:
        v = np.array(kat["triangles"][r["tri"]]["v"], np.float32)
        hit, tuv = oracle.intersect64(v[0], v[1], v[2], r["o"], r["d"])
        assert hit
        np.testing.assert_allclose(tuv, r["tuv"], rtol=0, atol=1e-12)
        tris = np.array([[0, 1, 2]], np.int32)
        bvh = oracle.build_lbvh(v, tris)
        ray = np.array([[*r["o"], 0.0, *r["d"], np.inf]], np.float32)
        res = oracle.trace(bvh["nodes"], bvh["woop"], bvh["tri_idx"], ray)
        assert res[0, 0] == 0
        got = res[0, 1:].view(np.float32)
        np.testing.assert_array_equal(got, np.array(r["tuv"], np.float32))
