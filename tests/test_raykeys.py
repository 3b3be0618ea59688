"""Ray Morton key methods on the CPU: the renderer's method names
(Renderer::stringToMortonCodeMethod), and the oracle's keys against a float64
restatement of the reference formulas (exact atan2 / acos; the keys may differ
only where a quantised coordinate sits at a step)."""
import numpy as np
import pytest

import hippie_b200 as hp
from hippie_b200._lib import load
import oracle


def test_method_names():
    lib = load()
    want = {"aila": 1, "paraboloid": 2, "octahedron": 3, "origin": 4, "costa": 5, "reise": 6,
            "reis": 0, "twopoint": 0, "": 0}
    for name, m in want.items():
        assert lib.hp_ray_keys_method(name.encode()) == m, name


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.2, 1.2, (n, 3))
    d = rng.normal(size=(n, 3))
    d[: n // 8, 0] = 0.0  # directions in a coordinate plane
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3], r[:, 4:7], r[:, 7] = o, d, rng.uniform(0.0, 2.0, n)
    return r


def _spherical_f64(r):
    d = r[:, 4:7].astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    bx = np.arctan2(d[:, 1], d[:, 0]) / (2 * np.pi) + 0.5
    by = np.arccos(np.clip(d[:, 2], -1, 1)) / np.pi
    return bx, by


@pytest.mark.parametrize("method,scale,shift", [("costa", 32767, 49), ("reis", 2097151, 1)])
def test_spherical_direction_bits(method, scale, shift):
    """The direction part of the Costa / Reis keys against float64 atan2 / acos."""
    r = _rays(20000, 3)
    keys = oracle.ray_keys(r, bits=64, method=method)
    bx, by = _spherical_f64(r)
    qx, qy = np.floor(bx * scale).astype(np.int64), np.floor(by * scale).astype(np.int64)
    if method == "costa":  # direction bits 14..11 of x and y at 2i+35 / 2i+34
        got_x = sum(((keys >> np.uint64(2 * i + 35)) & np.uint64(1)).astype(np.int64) << i for i in range(11, 15))
        got_y = sum(((keys >> np.uint64(2 * i + 34)) & np.uint64(1)).astype(np.int64) << i for i in range(11, 15))
        want_x, want_y = qx & 0x7800, qy & 0x7800
    else:  # all 21 bits at 2i+1 / 2i
        got_x = sum(((keys >> np.uint64(2 * i + 1)) & np.uint64(1)).astype(np.int64) << i for i in range(21))
        got_y = sum(((keys >> np.uint64(2 * i)) & np.uint64(1)).astype(np.int64) << i for i in range(21))
        want_x, want_y = qx, qy
    dx = np.abs(got_x - want_x)
    dy = np.abs(got_y - want_y)
    if method == "costa":  # 4 bits per axis: equal but where the value sits at a step
        assert np.all(dx <= 0x800) and np.all(dy <= 0x800)
        assert (dx > 0).mean() < 0.01 and (dy > 0).mean() < 0.01
    else:  # 21 bits per axis: float32 rounding moves a few percent by a step; acos near the
        # poles (|z| -> 1, an infinite slope) by a few steps
        assert np.all(dx <= 1) and (dx > 0).mean() < 0.1
        assert np.mean(dy <= 1) > 0.99 and np.mean(dy <= 16) == 1.0


def test_origin_keys_ignore_direction_and_default_is_aila():
    r = _rays(4096, 5)
    r2 = r.copy()
    r2[:, 4:7] = -r2[:, 4:7]
    np.testing.assert_array_equal(oracle.ray_keys(r, bits=64, method="origin"),
                                  oracle.ray_keys(r2, bits=64, method="origin"))
    a = oracle.ray_keys(r, bits=30)
    np.testing.assert_array_equal(a, oracle.ray_keys(r, bits=30, method="aila"))
    # two-point keys depend on the ray length: a zero length puts both points at the origin
    t0 = oracle.ray_keys(r, bits=64, method="two_point", ray_length=0.0)
    t1 = oracle.ray_keys(r, bits=64, method="two_point", ray_length=0.25)
    assert (t0 != t1).mean() > 0.5
