"""Ray generation on the host side (CPU): the pixel table against the oracle's
literal walk of PixelTable::recalculate, the camera matrix against an
independent double-precision construction, the Halton points."""
import math

import numpy as np
import pytest

import hippie_b200 as hp
import oracle


@pytest.mark.parametrize("w,h", [(8, 8), (16, 8), (13, 11), (100, 37), (64, 64), (1921, 1081), (7, 5), (1, 1)])
def test_pixel_table_matches_reference_walk(w, h):
    a = hp.pixel_table(w, h)
    np.testing.assert_array_equal(a, oracle.pixel_table(w, h))
    assert np.array_equal(np.sort(a), np.arange(w * h))


def test_pixel_table_block_order():
    t = hp.pixel_table(16, 16)
    # first block: the 8x8 pixels at the origin, x and y bits interleaved
    assert t[:4].tolist() == [0, 1, 16, 17]
    assert set(t[:64].tolist()) == {y * 16 + x for y in range(8) for x in range(8)}
    assert set(t[64:128].tolist()) == {y * 16 + x for y in range(8) for x in range(8, 16)}


def _rot(angle, axis):
    x, y, z = axis
    c, s, t = math.cos(angle), math.sin(angle), 1 - math.cos(angle)
    return np.array([[c + x * x * t, x * y * t - z * s, x * z * t + y * s, 0],
                     [x * y * t + z * s, c + y * y * t, y * z * t - x * s, 0],
                     [z * x * t - y * s, z * y * t + x * s, c + z * z * t, 0],
                     [0, 0, 0, 1]])


def test_camera_matrix():
    pos, d = np.array([0.3, 0.7, -1.5]), np.array([0.1, -0.2, 1.0])
    w, h, fov, near, far = 640, 320, 45.0, 0.01, 50.0
    got = hp.camera_screen_to_world(pos, d, fov, w, h, near, far).astype(np.float64)
    dn = d / np.linalg.norm(d)
    elev, view = math.asin(dn[1]), math.atan2(dn[0], -dn[2])
    T = np.eye(4)
    T[:3, 3] = -pos
    V = _rot(-elev, (1, 0, 0)) @ _rot(view, (0, 1, 0)) @ T
    fy = 1 / math.tan(math.radians(fov) / 2)
    P = np.array([[fy / (w / h), 0, 0, 0], [0, fy, 0, 0],
                  [0, 0, (near + far) / (near - far), 2 * near * far / (near - far)], [0, 0, -1, 0]])
    exp = np.linalg.inv(P @ V)
    np.testing.assert_allclose(got, exp, rtol=1e-5, atol=1e-5 * np.abs(exp).max())
    # the centre of the screen looks along the camera direction
    p = got @ np.array([0, 0, 0, 1.0])
    v = p[:3] / p[3] - pos
    assert np.allclose(v / np.linalg.norm(v), dn, atol=1e-5)


def test_camera_rejects_bad_input():
    with pytest.raises(hp.HPError):
        hp.camera_screen_to_world([0, 0, 0], [0, 0, 0], 45.0, 64, 64)
    with pytest.raises(hp.HPError):
        hp.camera_screen_to_world([0, 0, 0], [0, 0, 1], 0.0, 64, 64)


def test_halton():
    assert oracle.halton(1, 2) == np.float32(0.5)
    assert oracle.halton(2, 2) == np.float32(0.25)
    assert oracle.halton(3, 2) == np.float32(0.75)
    assert oracle.halton(1, 3) == np.float32(1 / 3)
    assert oracle.halton(0, 2) == 0


def test_oracle_generators_equal_library_generators():
    """The CPU arm of bench.py makes its inputs with oracle.gen (no GPU library);
    they are the same bytes as hippie_b200.gen's."""
    import oracle
    for seed in (0xC0FFEE, 0xC0FFEE + 1, 7):
        a, b = hp.gen.uniform_mesh(seed, 5003, 0.01), oracle.gen.uniform_mesh(seed, 5003, 0.01)
        np.testing.assert_array_equal(a[0].view(np.int32), b[0].view(np.int32))
        np.testing.assert_array_equal(a[1], b[1])
        a, b = hp.gen.clustered_mesh(seed, 7001, 64, 0.02, 0.005), oracle.gen.clustered_mesh(seed, 7001, 64, 0.02, 0.005)
        np.testing.assert_array_equal(a[0].view(np.int32), b[0].view(np.int32))
        np.testing.assert_array_equal(a[1], b[1])
        box = np.concatenate([a[0].min(0), a[0].max(0)]).astype(np.float32)
        np.testing.assert_array_equal(hp.gen.rays_sphere(seed + 1, 9999, box).view(np.int32),
                                      oracle.gen.rays_sphere(seed + 1, 9999, box).view(np.int32))
        np.testing.assert_array_equal(hp.gen.rays_targeted(seed + 1, 9999, -0.5, 1.5).view(np.int32),
                                      oracle.gen.rays_targeted(seed + 1, 9999, -0.5, 1.5).view(np.int32))
