"""Scene files on the host: the binary cache format of BinImporter / BinExporter
(util/BinImporter.cpp:16-84, util/BinExporter.cpp:14-70), the OBJ geometry the
importer returns, and SceneLoader::loadStaticScene's normalisation
(rt/scene/SceneLoader.cpp:103-160). No GPU."""
import os
import struct

import numpy as np
import pytest

import hippie_b200 as hp


def _write_reference_bin(path, verts, tris, box, materials=2, textures=("a.png", "tex/b.jpg")):
    """The file layout BinExporter::exportScene writes, produced independently here:
    header, box, vertices, normals, texture coordinates, triangles, material
    indices, materials (opaque bytes here) and QDataStream texture names."""
    nv, nt = len(verts), len(tris)
    rng = np.random.default_rng(3)
    with open(path, "wb") as f:
        f.write(struct.pack("<4i", nv, nt, materials, len(textures)))
        f.write(np.asarray(box, np.float32).tobytes())
        f.write(np.asarray(verts, np.float32).tobytes())
        f.write(rng.standard_normal((nv, 3)).astype(np.float32).tobytes())  # normals
        f.write(rng.random((nv, 2)).astype(np.float32).tobytes())  # texture coordinates
        f.write(np.asarray(tris, np.int32).tobytes())
        f.write(rng.integers(0, max(materials, 1), nt).astype(np.int32).tobytes())
        f.write(bytes(rng.integers(0, 256, 96 * materials, dtype=np.uint8)))
        for name in textures:  # QDataStream QString: uint32 byte length (big endian), UTF-16BE
            b = name.encode("utf-16-be")
            f.write(struct.pack(">I", len(b)) + b)


def test_read_bin_matches_reference_layout(tmp_path):
    v, t = hp.gen.uniform_mesh(7, 500)
    box = np.concatenate([v.min(0), v.max(0)])
    p = tmp_path / "s.obj.bin"
    _write_reference_bin(p, v, t, box)
    s = hp.read_scene_bin(p)
    assert np.array_equal(s.vertices, v) and np.array_equal(s.triangles, t)
    assert np.array_equal(s.box, box.astype(np.float32))


def test_write_bin_layout(tmp_path):
    v, t = hp.gen.clustered_mesh(2, 300, 8, 0.05, 0.01)
    box = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)
    p = tmp_path / "w.bin"
    hp.Scene(v, t, box).write_bin(p)
    raw = p.read_bytes()
    nv, nt = len(v), len(t)
    assert len(raw) == 16 + 24 + nv * 12 + nv * 12 + nv * 8 + nt * 12 + nt * 4
    assert struct.unpack("<4i", raw[:16]) == (nv, nt, 0, 0)
    assert np.array_equal(np.frombuffer(raw[16:40], np.float32), box)
    off = 40
    assert np.array_equal(np.frombuffer(raw[off:off + nv * 12], np.float32).reshape(-1, 3), v)
    off += nv * 12 + nv * 20  # normals and texture coordinates are zero
    assert not np.frombuffer(raw[40 + nv * 12:off], np.uint8).any()
    assert np.array_equal(np.frombuffer(raw[off:off + nt * 12], np.int32).reshape(-1, 3), t)
    # and the round trip
    s = hp.read_scene_bin(p)
    assert np.array_equal(s.vertices, v) and np.array_equal(s.triangles, t) and np.array_equal(s.box, box)


def test_read_obj_fans_negative_indices_and_degenerates(tmp_path):
    p = tmp_path / "q.obj"
    p.write_text("# quad, a degenerate face, a relative-index triangle and a pentagon\n"
                 "v 0 0 0\nv 2 0 0\nv 2 1 0\nv 0 1 0\nv 5 5 5\n"
                 "vn 0 0 1\nvt 0 0\n"
                 "f 1/1/1 2/1/1 3/1/1 4/1/1\n"
                 "f 1 1 2\n"
                 "f -1 -2 -3\n"
                 "f 1 2 3 4 5\n")
    s = hp.read_scene_obj(p)
    assert s.triangles.tolist() == [[0, 1, 2], [0, 2, 3], [4, 3, 2], [0, 1, 2], [0, 2, 3], [0, 3, 4]]
    assert s.vertices.shape == (5, 3)
    assert s.box.tolist() == [0, 0, 0, 5, 5, 5]


def test_normalize_is_bitwise_the_reference_formula():
    v, t = hp.gen.clustered_mesh(4, 2000, 16, 0.3, 0.05)
    v = (v * np.float32(7.5) - np.float32(3.0)).astype(np.float32)
    box = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)
    s = hp.Scene(v, t, box).normalized()
    diag = box[3:] - box[:3]
    scale = np.float32(1.0) / np.float32(max(diag))
    want = (v - box[:3]).astype(np.float32) * scale
    assert np.array_equal(s.vertices, want.astype(np.float32))
    assert s.vertices.min() == 0.0 and s.vertices.max() <= 1.0


def test_load_scene_caches_and_prefers_the_cache(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text("v 0 0 0\nv 4 0 0\nv 0 2 0\nv 0 0 1\nf 1 2 3\nf 1 2 4\n")
    s = hp.load_scene(p)
    cache = tmp_path / "m.obj.bin"
    assert cache.exists()
    assert s.triangles.tolist() == [[0, 1, 2], [0, 1, 3]]
    assert np.array_equal(s.vertices, np.array([[0, 0, 0], [1, 0, 0], [0, .5, 0], [0, 0, .25]], np.float32))
    # the cache wins over the (changed) OBJ file, as in SceneLoader::loadScene
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    s2 = hp.load_scene(p)
    assert np.array_equal(s2.vertices, s.vertices) and np.array_equal(s2.triangles, s.triangles)
    os.remove(cache)
    s3 = hp.load_scene(p, write_cache=False)
    assert len(s3.triangles) == 1 and not cache.exists()
    # a ".bin" path is read directly
    s4 = hp.load_scene(tmp_path / "m.obj", write_cache=True)
    s5 = hp.load_scene(cache)
    assert np.array_equal(s4.vertices, s5.vertices)


def test_scene_errors(tmp_path):
    with pytest.raises(hp.HPError):
        hp.read_scene_bin(tmp_path / "missing.bin")
    with pytest.raises(hp.HPError):
        hp.load_scene(tmp_path / "missing.obj")
    bad = tmp_path / "trunc.bin"
    bad.write_bytes(struct.pack("<4i", 10, 5, 0, 0) + bytes(24) + bytes(40))
    with pytest.raises(hp.HPError):
        hp.read_scene_bin(bad)
    idx = tmp_path / "idx.bin"
    _write_reference_bin(idx, np.zeros((3, 3), np.float32), np.array([[0, 1, 3]], np.int32), np.zeros(6), 0, ())
    with pytest.raises(hp.HPError):
        hp.read_scene_bin(idx)
    obj = tmp_path / "bad.obj"
    obj.write_text("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(hp.HPError):
        hp.read_scene_obj(obj)
