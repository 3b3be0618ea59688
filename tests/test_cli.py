"""The C++ bench CLI (hippie_b200_bench) on the host: env files in the
reference's format resolve to the expected build, camera and scene settings;
OBJ scenes load (polygons fanned into triangles, negative indices); bad input
is reported with a non-zero exit."""
import json
import subprocess
from pathlib import Path

import pytest

import hippie_b200 as hp

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "hippie_b200" / "hippie_b200_bench"


@pytest.fixture(scope="module", autouse=True)
def built():
    from hippie_b200 import build
    build.build()
    assert CLI.exists()


def run(*args):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, timeout=120)


ENV = """Bvh {{
 method {method}
 plocRadius 8
 plocMortonCodeBits 60
 atrIterations 3
 atrTreeletSize 9
 ct 3.0
 ci 2.0
}}
Scene {{
 filename {scene}
}}
Resolution {{
 width 320
 height 200
}}
Camera {{
 position 0.5 0.5 -1.5
 direction 0.0 0.0 1.0
 fieldOfView 50.0
 nearPlane 0.01
 farPlane 100.0
}}
Renderer {{
 numberOfPrimarySamples 3
}}
"""


def test_help():
    r = run("--help")
    assert r.returncode == 0 and "usage" in r.stdout


def test_dry_run_env(tmp_path):
    env = tmp_path / "a.env"
    env.write_text(ENV.format(method="atr", scene="synthetic:uniform:1000"))
    r = run(env, "--dry-run")
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout)
    assert (d["method"], d["atr_iterations"], d["atr_treelet"], d["triangles"]) == ("atr", 3, 9, 1000)
    assert (d["width"], d["height"], d["samples"], d["fov"]) == (320, 200, 3, 50)
    assert d["camera"] == [0.5, 0.5, -1.5, 0, 0, 1]


def test_obj_scene(tmp_path):
    obj = tmp_path / "quad.obj"
    obj.write_text("# two quads and a triangle\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 1\n"
                   "f 1 2 3 4\nf 1/1/1 2/2/2 5/3/3\nf -1 -2 -3 -4\n")
    env = tmp_path / "b.env"
    env.write_text(ENV.format(method="lbvh", scene=obj))
    d = json.loads(run(env, "--dry-run").stdout)
    assert (d["triangles"], d["vertices"]) == (5, 5)
    # loaded as SceneLoader does: the geometry is cached beside the scene file
    cached = hp.read_scene_bin(tmp_path / "quad.obj.bin")
    assert cached.triangles.shape == (5, 3)


def test_bad_input(tmp_path):
    env = tmp_path / "c.env"
    env.write_text(ENV.format(method="ploc", scene=tmp_path / "missing.obj"))
    r = run(env, "--dry-run")
    assert r.returncode != 0 and "cannot open" in r.stderr
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nf 1 2 3\n")
    env.write_text(ENV.format(method="ploc", scene=bad))
    r = run(env, "--dry-run")
    assert r.returncode != 0 and "bad face index" in r.stderr
    env.write_text(ENV.format(method="bogus", scene="synthetic:uniform:10"))
    assert run(env, "--dry-run").returncode != 0
