"""The C++ bench CLI on the GPU: the BVH it builds from an env file and the
primary rays it traces agree with the same build and trace through the
Python binding (sm_100a)."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

import hippie_b200 as hp

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "hippie_b200" / "hippie_b200_bench"

ENV = """Bvh {{
 method {method}
 plocRadius 16
 plocMaxRadius 256
 plocMortonCodeBits 60
 lbvhMortonCodeBits 30
}}
Scene {{
 filename {scene}
}}
Resolution {{
 width 256
 height 128
}}
Camera {{
 position 0.5 0.5 -1.5
 direction 0.0 0.0 1.0
 nearPlane 0.01
 farPlane 100.0
}}
Renderer {{
 numberOfPrimarySamples 2
}}
"""


@pytest.mark.parametrize("method", ["lbvh", "ploc", "atr", "tr", "hlbvh"])
def test_cli_matches_python(ctx, tmp_path, method):
    v, t = hp.gen.uniform_mesh(5, 3000)
    obj = tmp_path / "m.obj"
    lines = [f"v {x!r} {y!r} {z!r}" for x, y, z in v.tolist()] + [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in t]
    obj.write_text("\n".join(lines) + "\n")
    env = tmp_path / "s.env"
    env.write_text(ENV.format(method=method, scene=obj))
    r = subprocess.run([str(CLI), str(env), "--steps", "2"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout)
    assert d["triangles"] == 3000 and d["valid"] is True
    # the same build through the Python binding, on the scene as the CLI loaded it
    # (vertices round-trip exactly through repr; then SceneLoader's normalisation)
    scene = hp.load_scene(obj)
    assert np.array_equal(scene.triangles, t)
    assert np.array_equal(scene.vertices, hp.Scene(v, t).normalized().vertices)
    p = hp.Env().read_string(env.read_text()).build_params()
    V, T = torch.from_numpy(scene.vertices).cuda(), torch.from_numpy(scene.triangles).cuda()
    bvh = ctx.build(V, T, p)
    bvh.sync()
    assert d["nodes"] == bvh.num_nodes
    st = bvh.stats()
    assert d["sah_cost"] == st["sah_cost"]
    assert d["avg_leaf_size"] == st["avg_leaf_size"]
    assert d["leaf_size_histogram"] == pytest.approx(st["leaf_size_histogram"], rel=1e-8)
    pos = np.array([0.5, 0.5, -1.5], np.float32)
    m = hp.camera_screen_to_world(pos, [0, 0, 1], 45.0, 256, 128, 0.01, 100.0)
    tbl = torch.from_numpy(hp.pixel_table(256, 128)).cuda()
    hits = 0
    for s in range(2):
        R = ctx.primary_rays(pos, m, 256, 128, max_dist=100.0, sample_index=s, index_to_pixel=tbl)
        hits += int((ctx.trace(bvh, R)[:, 0] >= 0).sum())
    assert d["hits"] == hits


def test_cli_synthetic_scene(tmp_path):
    env = tmp_path / "s.env"
    env.write_text(ENV.format(method="ploc", scene="synthetic:clustered:100000"))
    r = subprocess.run([str(CLI), str(env)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout)
    assert d["triangles"] == 100000 and d["valid"] is True and d["build_mtris_s"] > 0 and d["trace_mrays_s"] > 0
