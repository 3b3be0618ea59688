"""Generates tests/golden/ref_fixtures.npz from the REFERENCE's own kernels.

Runs on a GPU machine in a checkout where oracle/_ref/libhipref.so was built
from the reference sources (oracle/ref/Makefile). For two small synthetic
meshes it records what the reference's kernels produce: Morton keys, the
sorted reference order, the pre-collapse LBVH topology and refitted boxes,
the collapsed binary BVH (nodes, triangle order, Woop triangles), a PLOC BVH,
an ATR BVH (treelet 9, 2 iterations) and closest hits of the reference tracer. The scene box and the Morton scale
(the approximate reciprocal the reference's fast-math build uses) are stored
with them, so the CPU oracle can be compared against the reference offline.

Run: python tests/golden/make_ref_fixtures.py <output.npz>
"""
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import hippie_b200 as hp  # noqa: E402
from oracle import ref_harness as R  # noqa: E402


def main(out):
    ctx = hp.Context(0)
    data = {}
    cases = [("uniform", hp.gen.uniform_mesh(71, 3000), 30), ("clustered", hp.gen.clustered_mesh(72, 4000, 16), 60)]
    for name, (v, t), bits in cases:
        V, T = torch.from_numpy(v).cuda(), torch.from_numpy(t).cuda()
        bvh = ctx.build(V, T, hp.BuildParams(morton_bits=bits))
        bvh.sync()
        box = np.array(bvh.c.scene_box, np.float32)
        data[f"{name}_box"] = box
        data[f"{name}_scale"] = np.array(bvh.c.morton_scale, np.float32)
        ref = R.build(V, T, box, method="lbvh", bits=bits, taps=True)
        for k in ("keys", "sorted", "refs", "parent", "left", "right", "bmin", "bmax", "nodes", "tri_idx", "woop",
                  "counts"):
            data[f"{name}_lbvh_{k}"] = ref[k]
        p = R.build(V, T, box, method="ploc", bits=bits, radius=4, max_radius=64)
        for k in ("nodes", "tri_idx", "counts"):
            data[f"{name}_ploc_{k}"] = p[k]
        a = R.build(V, T, box, method="atr", bits=bits, treelet=9, iterations=2)
        for k in ("nodes", "tri_idx", "counts"):
            data[f"{name}_atr_{k}"] = a[k]
        rays = hp.gen.rays_targeted(73, 2000) if name == "uniform" else \
            hp.gen.rays_sphere(74, 2000, np.concatenate([v.min(0), v.max(0)]))
        res, _ = R.trace(torch.from_numpy(ref["nodes"]).cuda(), torch.from_numpy(ref["woop"]).cuda(),
                         torch.from_numpy(ref["tri_idx"]).cuda(), torch.from_numpy(rays).cuda())
        data[f"{name}_trace"] = res
    np.savez_compressed(out, **data)
    print("wrote", out, sum(a.nbytes for a in data.values()), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).resolve().parent / "ref_fixtures.npz"))
