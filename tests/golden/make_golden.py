"""Generates the known-answer vectors in this folder.

The reference ships no tests, fixtures or golden vectors, so these vectors are
derived by hand from the reference's formulas, written here as plain Python
that shares no code with the oracle or the library:

* morton_kat.json   Morton codes (rt/HipUtil.h:35-106): 20-bit integer
  coordinates interleaved bit by bit with x in the least significant position
  of each triple; bits 10..19 of every axis form key bits 30..59. Plus the
  centroid quantisation of computeMortonCodes60 (rt/bvh/LBVHBuilderKernels.cu:131-160)
  for boxes whose centroids sit on exact binary fractions of the scene box.
* karras_kat.json   The 8-key example of Karras 2012 ("Maximizing parallelism
  in the construction of BVHs, octrees, and k-d trees", Fig. 3/4) with the
  tree that paper shows: interior node i covers a range starting or ending at
  key i; leaf j is node n-1+j.
* woop_kat.json     Woop transforms of axis-aligned right triangles whose
  inverse matrices are exact in binary floating point
  (rt/bvh/HipBVHKernels.cu:12-65), and rays with exactly known (t, u, v).

Run: python tests/golden/make_golden.py
"""
import json
import random
from pathlib import Path

HERE = Path(__file__).resolve().parent


def interleave60(x, y, z):
    code = 0
    for b in range(20):
        code |= ((x >> b) & 1) << (3 * b)
        code |= ((y >> b) & 1) << (3 * b + 1)
        code |= ((z >> b) & 1) << (3 * b + 2)
    return code


def morton60_ref(x, y, z):
    # mortonCode64 splits each 20-bit coordinate into its low and high 10 bits
    lo = interleave60(x & 1023, y & 1023, z & 1023)
    hi = interleave60(x >> 10, y >> 10, z >> 10)
    return (hi << 30) | lo


def morton_kat():
    rnd = random.Random(20150101)
    cases = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1), (2, 0, 0), (1023, 1023, 1023),
             (1024, 0, 0), (0, 1024, 0), (0, 0, 1024), (1048575, 1048575, 1048575), (1048575, 0, 0),
             (524288, 524288, 524288), (1048576, 0, 0)]
    cases += [(rnd.randrange(1 << 20), rnd.randrange(1 << 20), rnd.randrange(1 << 20)) for _ in range(64)]
    codes = [{"xyz": list(c), "code60": morton60_ref(*c)} for c in cases]
    # Quantisation: scene box [0,1]^3 (scale exactly 1), boxes of zero extent at
    # binary fractions k/2^m, so (c - 0) * 1 * 1048575 is exact and truncation is clear.
    quant = []
    for k, m in [(0, 1), (1, 1), (1, 2), (3, 4), (1, 10), (1023, 10), (1, 20), (5, 3)]:
        c = k / 2 ** m
        q = int(c * 1048575)  # exact product of a dyadic fraction and an integer, truncated
        quant.append({"centroid": c, "q": q})
    return {"codes": codes, "quant": quant}


def karras_kat():
    keys = [0b00001, 0b00010, 0b00100, 0b00101, 0b10011, 0b11000, 0b11001, 0b11110]
    n = len(keys)
    L = lambda j: n - 1 + j  # leaf node index
    # interior node -> (left, right) as drawn in the paper
    tree = {0: (3, 4), 3: (1, 2), 1: (L(0), L(1)), 2: (L(2), L(3)), 4: (L(4), 5), 5: (6, L(7)), 6: (L(5), L(6))}
    left = [0] * (2 * n - 1)
    right = [0] * (2 * n - 1)
    parent = [0] * (2 * n - 1)
    parent[0] = -1
    for i, (l, r) in tree.items():
        left[i], right[i] = l, r
        parent[l] = parent[r] = i
    for j in range(n):
        left[L(j)], right[L(j)] = j, j + 1
    return {"bits": 5, "keys": keys, "left": left, "right": right, "parent": parent}


def woop_kat():
    tris = [
        # v0, v1, v2, expected rows w0 (normal/t), w1 (u), w2 (v)
        {"v": [[1, 0, 0], [0, 1, 0], [0, 0, 0]],
         "w": [[0, 0, 1, 0], [1, 0, 0, 0], [0, 1, 0, 0]]},
        {"v": [[2, 0, 0], [0, 4, 0], [0, 0, 0]],
         "w": [[0, 0, 0.125, 0], [0.5, 0, 0, 0], [0, 0.25, 0, 0]]},
        {"v": [[3, 1, 1], [1, 5, 1], [1, 1, 1]],
         "w": [[0, 0, 0.125, 0.125], [0.5, 0, 0, -0.5], [0, 0.25, 0, -0.25]]},
    ]
    rays = [
        # triangle index, origin, direction, expected (t, u, v)
        {"tri": 0, "o": [0.25, 0.25, 1.0], "d": [0, 0, -1], "tuv": [1.0, 0.25, 0.25]},
        {"tri": 1, "o": [0.5, 1.0, 2.0], "d": [0, 0, -1], "tuv": [2.0, 0.25, 0.25]},
        {"tri": 2, "o": [1.5, 2.0, 5.0], "d": [0, 0, -1], "tuv": [4.0, 0.25, 0.25]},
        {"tri": 2, "o": [2.0, 1.0, -3.0], "d": [0, 0, 1], "tuv": [4.0, 0.5, 0.0]},
    ]
    return {"triangles": tris, "rays": rays}


def main():
    (HERE / "morton_kat.json").write_text(json.dumps(morton_kat(), indent=1))
    (HERE / "karras_kat.json").write_text(json.dumps(karras_kat(), indent=1))
    (HERE / "woop_kat.json").write_text(json.dumps(woop_kat(), indent=1))


if __name__ == "__main__":
    main()
