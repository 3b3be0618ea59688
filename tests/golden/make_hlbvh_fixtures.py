"""Writes hlbvh_ref_fixtures.npz: HLBVH builds by the REFERENCE's own kernels
(rt/bvh/HLBVHBuilderKernels.cu with the LBVH and collapser kernels, sequenced
as HLBVHBuilder::build; built into oracle/_ref by oracle/ref/Makefile) for
seeded meshes scaled into [0, 1]^3 as the reference's scene loader does.
Records the collapsed nodes, triangle order and node counts, with the scene
box and Morton scale of this library's build of the same mesh, so the CPU
oracle can be compared against the reference offline (tests/test_oracle_hlbvh.py).

Runs on a GPU machine in a checkout where oracle/_ref/libhipref.so was built
from the reference sources: python tests/golden/make_hlbvh_fixtures.py <out.npz>
"""
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
import hippie_b200 as hp  # noqa: E402
from oracle import ref_harness as R  # noqa: E402
from hlbvh_cases import CASES, mesh  # noqa: E402


def main(out):
    ctx = hp.Context(0)
    data = {}
    for name, (_, bits, sah) in CASES.items():
        v, t = mesh(name)
        V, T = torch.from_numpy(v).cuda(), torch.from_numpy(t).cuda()
        bvh = ctx.build(V, T, hp.BuildParams(method="hlbvh", morton_bits=bits, hlbvh_sah_bits=sah))
        bvh.sync()
        box = np.array(bvh.c.scene_box, np.float32)
        ref = R.build(V, T, box, method="hlbvh", bits=bits, sah_bits=sah)
        data[f"{name}_box"] = box
        data[f"{name}_scale"] = np.array(bvh.c.morton_scale, np.float32)
        for k in ("nodes", "tri_idx", "counts"):
            data[f"{name}_{k}"] = ref[k]
    np.savez_compressed(out, **data)
    print("wrote", out, sum(a.nbytes for a in data.values()), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).resolve().parent / "hlbvh_ref_fixtures.npz"))
