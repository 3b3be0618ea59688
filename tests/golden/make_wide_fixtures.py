"""Writes tests/golden/wide_ref_fixtures.npz: N-wide collapses computed by the
REFERENCE's own host code (BVH::collapseAdaptiveWide / collapseWide of
rt/bvh/BVH.h, built into oracle/_ref by oracle/ref/Makefile) on the binary
trees the oracle builds for seeded meshes. Run where the reference sources are
present: python tests/golden/make_wide_fixtures.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import hippie_b200 as hp  # noqa: E402
import oracle  # noqa: E402
from oracle import ref_harness as R  # noqa: E402

# name -> (mesh, method, width, adaptive, max_leaf)
CASES = {
    "lbvh_quad": (lambda: hp.gen.uniform_mesh(81, 600), "lbvh", 4, 1, 8),
    "lbvh_oct": (lambda: hp.gen.clustered_mesh(82, 700, 16, 0.05, 0.01), "lbvh", 8, 1, 8),
    "ploc_quad": (lambda: hp.gen.clustered_mesh(83, 700, 16, 0.05, 0.01), "ploc", 4, 1, 8),
    "ploc_oct": (lambda: hp.gen.uniform_mesh(84, 600), "ploc", 8, 1, 8),
    "atr_oct": (lambda: hp.gen.clustered_mesh(85, 700, 8, 0.05, 0.01), "atr", 8, 1, 8),
    "lbvh_quad_maxleaf": (lambda: hp.gen.clustered_mesh(86, 700, 8, 0.05, 0.01), "lbvh", 4, 0, 6),
}


def main():
    out = {}
    for name, (mesh, method, width, adaptive, max_leaf) in CASES.items():
        v, t = mesh()
        d = oracle.binary_tree(v, t, method)
        r = R.wide_collapse(t.shape[0], d["left"], d["right"], d["bmin4"], d["bmax4"], d["sorted_tri"], width,
                            adaptive=adaptive, max_leaf=max_leaf)
        assert r is not None, name
        out[name + "_nodes"], out[name + "_tri"], out[name + "_counts"] = r[0], r[1], np.array(r[2], np.int32)
    np.savez_compressed(Path(__file__).resolve().parent / "wide_ref_fixtures.npz", **out)


if __name__ == "__main__":
    main()
