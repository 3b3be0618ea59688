"""CPU oracle — test infrastructure only (see oracle.cpp).

ctypes access to liboracle.so, a C++/OpenMP restatement of the reference's
build-and-trace path. Only the tests, __graft_entry__.smoke() and the CPU
baseline leg of bench.py use it; the shipped library never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None

_P = C.c_void_p
_SIGS = {
    "or_tri_boxes": (None, [_P, _P, C.c_int64, _P, _P, _P]),
    "or_morton": (None, [C.c_int64, _P, _P, _P, _P, C.c_int, _P, _P]),
    "or_sort": (None, [C.c_int64, _P, C.c_int, _P, _P]),
    "or_karras": (None, [C.c_int, _P, _P, _P, _P]),
    "or_refit": (None, [C.c_int, _P, _P, _P, _P, _P, _P, C.c_float, C.c_float, C.c_int, C.c_int,
                        _P, _P, _P, _P, _P]),
    "or_collapse": (C.c_int64, [C.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "or_woopify": (None, [C.c_int64, _P, _P, _P, _P]),
    "or_build_lbvh": (C.c_int64, [_P, _P, C.c_int64, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int,
                                  _P, _P, _P, _P, _P, _P, _P]),
    "or_cost": (C.c_double, [_P, C.c_int64, _P, C.c_float, C.c_float]),
    "or_build_ploc": (C.c_int64, [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                  C.c_int, C.c_int, _P, _P, _P, _P, _P, _P, _P, _P]),
    "or_build_atr": (C.c_int64, [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                                 C.c_int, _P, _P, _P, _P, _P, _P, _P]),
    "or_atr": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _P, _P, _P, _P, _P]),
    "or_pixel_table": (C.c_int32, [C.c_int32, C.c_int32, _P]),
    "or_primary_rays": (None, [_P, _P, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float, _P, _P]),
    "or_ray_keys": (None, [_P, C.c_int64, _P, C.c_int32, _P]),
    "or_ray_keys_method": (None, [_P, C.c_int64, _P, C.c_int32, C.c_int32, C.c_float, _P]),
    "or_build_hlbvh": (C.c_int64, [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, _P,
                                   _P, _P, _P, _P, _P, _P]),
    "or_tr": (C.c_int, [C.c_int, C.c_int, C.c_float, C.c_float, _P, _P, _P, _P, _P]),
    "or_build_tr": (C.c_int64, [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, _P, _P,
                                _P, _P, _P, _P, _P]),
    "or_collapse_wide": (C.c_int64, [C.c_int, _P, _P, _P, _P, _P, C.c_int, C.c_float, C.c_float, C.c_int, _P, _P,
                                      _P]),
    "or_binary_tree": (None, [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                              C.c_int, C.c_float, C.c_float, _P, _P, _P, _P, _P, _P, _P, _P]),
    "or_build_wide": (C.c_int64, [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P,
                                  _P]),
    "or_trace": (None, [_P, _P, _P, C.c_int64, _P, C.c_int64, _P, _P, C.c_int]),
    "or_intersect64": (C.c_int, [_P, _P, _P, _P, _P, C.c_double, _P]),
    "or_brute64": (None, [_P, _P, C.c_int64, _P, C.c_int64, _P]),
    "or_adjoint64": (None, [_P, _P, _P, _P, _P, C.c_int64, _P]),
    "or_canonical": (C.c_int64, [_P, C.c_int64, _P, C.c_int64, _P, _P]),
    "or_gen_uniform_mesh": (None, [C.c_uint64, C.c_int64, C.c_float, _P, _P]),
    "or_gen_clustered_mesh": (None, [C.c_uint64, C.c_int64, C.c_int32, C.c_float, C.c_float, _P, _P]),
    "or_gen_rays_targeted": (None, [C.c_uint64, C.c_int64, C.c_float, C.c_float, _P]),
    "or_gen_rays_sphere": (None, [C.c_uint64, C.c_int64, _P, _P]),
}


def load():
    global _lib
    if _lib is not None:
        return _lib
    src = HERE / "oracle.cpp"
    if not LIB.exists() or (src.exists() and src.stat().st_mtime > LIB.stat().st_mtime):
        subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, capture_output=True)
    lib = C.CDLL(str(LIB))
    for k, (res, args) in _SIGS.items():
        f = getattr(lib, k)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


def tri_boxes(verts, tris):
    n = tris.shape[0]
    bmin = np.zeros((n, 4), np.float32)
    bmax = np.zeros((n, 4), np.float32)
    box = np.zeros(6, np.float32)
    load().or_tri_boxes(_p(verts), _p(tris), n, _p(bmin), _p(bmax), _p(box))
    return bmin, bmax, box


def morton(bmin, bmax, scene_box, bits, scale=None):
    n = bmin.shape[0]
    keys = np.zeros(n, np.uint64)
    sc = np.zeros(3, np.float32)
    s_in = None if scale is None else np.ascontiguousarray(scale, np.float32)
    load().or_morton(n, _p(bmin), _p(bmax), _p(np.ascontiguousarray(scene_box, np.float32)), _p(s_in), bits,
                     _p(keys), _p(sc))
    return keys, sc


def sort(keys, bits):
    n = keys.shape[0]
    sk = np.zeros(n, np.uint64)
    sr = np.zeros(n, np.int32)
    load().or_sort(n, _p(np.ascontiguousarray(keys, np.uint64)), bits, _p(sk), _p(sr))
    return sk, sr


def karras(skeys):
    n = skeys.shape[0]
    nn = 2 * n - 1
    parent = np.zeros(nn, np.int32)
    left = np.zeros(nn, np.int32)
    right = np.zeros(nn, np.int32)
    load().or_karras(n, _p(skeys), _p(parent), _p(left), _p(right))
    return parent, left, right


def refit(verts, tris, sorted_tri, parent, left, right, ct=3.0, ci=2.0, adaptive=1, max_leaf=8):
    n = sorted_tri.shape[0]
    nn = 2 * n - 1
    bmin = np.zeros((nn, 4), np.float32)
    bmax = np.zeros((nn, 4), np.float32)
    size = np.zeros(nn, np.int32)
    cost = np.zeros(nn, np.float32)
    state = np.zeros(nn, np.int32)
    load().or_refit(n, _p(verts), _p(tris), _p(sorted_tri), _p(parent), _p(left), _p(right), ct, ci, adaptive,
                    max_leaf, _p(bmin), _p(bmax), _p(size), _p(cost), _p(state))
    return bmin, bmax, size, cost, state


def build_lbvh(verts, tris, bits=60, ct=3.0, ci=2.0, adaptive=1, max_leaf=8, scale=None):
    """Full LBVH build; returns dict with nodes (N,16) int32, woop (n,12), tri_idx, counts, box, scale."""
    n = tris.shape[0]
    cap = max(2 * n - 1, 3)
    nodes = np.zeros((cap, 16), np.int32)
    woop = np.zeros((max(n, 1), 12), np.float32)
    tri = np.zeros(max(n, 1), np.int32)
    counts = np.zeros(2, np.int32)
    box = np.zeros(6, np.float32)
    sc = np.zeros(3, np.float32)
    s_in = None if scale is None else np.ascontiguousarray(scale, np.float32)
    cnt = load().or_build_lbvh(_p(verts), _p(tris), n, bits, ct, ci, adaptive, max_leaf, _p(s_in), _p(nodes),
                               _p(woop), _p(tri), _p(counts), _p(box), _p(sc))
    return dict(nodes=nodes[:cnt], woop=woop[:n], tri_idx=tri[:n], counts=counts, box=box, scale=sc)


def build_ploc(verts, tris, bits=60, radius=16, max_radius=256, adaptive_r=0, ct=3.0, ci=2.0, adaptive=1,
               max_leaf=8, scale=None):
    """Full PLOC build with depth-first collapse numbering; also returns the iteration count."""
    n = tris.shape[0]
    cap = max(2 * n - 1, 3)
    nodes = np.zeros((cap, 16), np.int32)
    woop = np.zeros((max(n, 1), 12), np.float32)
    tri = np.zeros(max(n, 1), np.int32)
    counts = np.zeros(2, np.int32)
    box = np.zeros(6, np.float32)
    sc = np.zeros(3, np.float32)
    it = np.zeros(1, np.int32)
    s_in = None if scale is None else np.ascontiguousarray(scale, np.float32)
    cnt = load().or_build_ploc(_p(verts), _p(tris), n, bits, radius, max_radius, adaptive_r, ct, ci, adaptive,
                               max_leaf, _p(s_in), _p(nodes), _p(woop), _p(tri), _p(counts), _p(box), _p(sc),
                               _p(it))
    return dict(nodes=nodes[:cnt], woop=woop[:n], tri_idx=tri[:n], counts=counts, box=box, scale=sc,
                iterations=int(it[0]))


def build_atr(verts, tris, bits=60, treelet=9, iterations=2, ct=3.0, ci=2.0, adaptive=1, max_leaf=8, scale=None):
    """LBVH + ATR treelet restructuring + depth-first collapse (ATRBuilder::build)."""
    n = tris.shape[0]
    cap = max(2 * n - 1, 3)
    nodes = np.zeros((cap, 16), np.int32)
    woop = np.zeros((max(n, 1), 12), np.float32)
    tri = np.zeros(max(n, 1), np.int32)
    counts = np.zeros(2, np.int32)
    box = np.zeros(6, np.float32)
    sc = np.zeros(3, np.float32)
    s_in = None if scale is None else np.ascontiguousarray(scale, np.float32)
    cnt = load().or_build_atr(_p(verts), _p(tris), n, bits, treelet, iterations, ct, ci, adaptive, max_leaf,
                              _p(s_in), _p(nodes), _p(woop), _p(tri), _p(counts), _p(box), _p(sc))
    return dict(nodes=nodes[:cnt], woop=woop[:n], tri_idx=tri[:n], counts=counts, box=box, scale=sc)


def build_tr(verts, tris, bits=60, iterations=2, ct=3.0, ci=2.0, adaptive=1, max_leaf=8, scale=None):
    """LBVH + TRBVH treelet restructuring (treelet 7) + depth-first collapse (TRBuilder::build)."""
    n = tris.shape[0]
    cap = max(2 * n - 1, 3)
    nodes = np.zeros((cap, 16), np.int32)
    woop = np.zeros((max(n, 1), 12), np.float32)
    tri = np.zeros(max(n, 1), np.int32)
    counts = np.zeros(2, np.int32)
    box = np.zeros(6, np.float32)
    sc = np.zeros(3, np.float32)
    s_in = None if scale is None else np.ascontiguousarray(scale, np.float32)
    cnt = load().or_build_tr(_p(verts), _p(tris), n, bits, iterations, ct, ci, adaptive, max_leaf, _p(s_in),
                             _p(nodes), _p(woop), _p(tri), _p(counts), _p(box), _p(sc))
    return dict(nodes=nodes[:cnt], woop=woop[:n], tri_idx=tri[:n], counts=counts, box=box, scale=sc)


def build_hlbvh(verts, tris, bits=60, sah_bits=15, ct=3.0, ci=2.0, adaptive=1, max_leaf=8, scale=None):
    """HLBVH (HLBVHBuilder::build): LBVH clusters below the top sah_bits Morton bits, a
    binned-SAH top tree above them, then the depth-first collapse."""
    n = tris.shape[0]
    cap = max(2 * n - 1, 3)
    nodes = np.zeros((cap, 16), np.int32)
    woop = np.zeros((max(n, 1), 12), np.float32)
    tri = np.zeros(max(n, 1), np.int32)
    counts = np.zeros(2, np.int32)
    box = np.zeros(6, np.float32)
    sc = np.zeros(3, np.float32)
    s_in = None if scale is None else np.ascontiguousarray(scale, np.float32)
    cnt = load().or_build_hlbvh(_p(verts), _p(tris), n, bits, sah_bits, ct, ci, adaptive, max_leaf, _p(s_in),
                                _p(nodes), _p(woop), _p(tri), _p(counts), _p(box), _p(sc))
    if cnt < 0:
        raise ValueError("sah_bits must be a multiple of 3 in [6, 15] and at most bits")
    return dict(nodes=nodes[:cnt], woop=woop[:n], tri_idx=tri[:n], counts=counts, box=box, scale=sc)


def tr(n, parent, left, right, bmin4, bmax4, iterations=2, ct=3.0, ci=2.0):
    """TRBVH iterations in place on a refitted binary tree (arrays over 2n-1 nodes)."""
    return load().or_tr(n, iterations, ct, ci, _p(parent), _p(left), _p(right), _p(bmin4), _p(bmax4))


def atr(n, parent, left, right, bmin4, bmax4, treelet=9, iterations=2, ct=3.0, ci=2.0):
    """ATR iterations in place on a refitted binary tree (arrays over 2n-1 nodes)."""
    return load().or_atr(n, treelet, iterations, ct, ci, _p(parent), _p(left), _p(right), _p(bmin4), _p(bmax4))


def pixel_table(width, height):
    t = np.empty(width * height, np.int32)
    k = load().or_pixel_table(width, height, _p(t))
    assert k == width * height
    return t


def halton(i, base):
    """Radical inverse as the library computes it (double, then rounded to float)."""
    r, f = 0.0, 1.0 / base
    while i > 0:
        r += f * (i % base)
        i //= base
        f /= base
    return np.float32(r)


def primary_rays(origin, m, width, height, sample_index=0, max_dist=np.inf, index_to_pixel=None):
    rays = np.empty((width * height, 8), np.float32)
    o = np.ascontiguousarray(origin, np.float32)
    mm = np.ascontiguousarray(m, np.float32).reshape(16)
    tbl = None if index_to_pixel is None else np.ascontiguousarray(index_to_pixel, np.int32)
    load().or_primary_rays(_p(o), _p(mm), width, height, float(halton(sample_index, 2)),
                           float(halton(sample_index, 3)), max_dist, _p(tbl), _p(rays))
    return rays


RAY_KEY_METHODS = {"two_point": 0, "aila": 1, "paraboloid": 2, "octahedron": 3, "origin": 4, "costa": 5, "reis": 6}


def ray_keys(rays, bits=30, box=(0, 0, 0, 1, 1, 1), method="aila", ray_length=0.25):
    """Ray Morton keys of RayBuffer::computeMortonCodes (the 64-bit kernels) by method."""
    keys = np.empty(rays.shape[0], np.uint64)
    b = np.ascontiguousarray(box, np.float32)
    m = RAY_KEY_METHODS[method] if isinstance(method, str) else int(method)
    load().or_ray_keys_method(_p(np.ascontiguousarray(rays, np.float32)), rays.shape[0], _p(b), bits, m,
                              float(ray_length), _p(keys))
    return keys


METHODS = {"lbvh": 0, "ploc": 1, "atr": 2, "tr": 3, "hlbvh": 4}


def binary_tree(verts, tris, method="lbvh", bits=60, radius=16, max_radius=256, adaptive_r=0, treelet=9,
                iterations=2, ct=3.0, ci=2.0, scale=None, sah_bits=15):
    """The binary tree a build collapses: dict of left, right, bmin4, bmax4 (2n-1 nodes),
    sorted_tri, scene_box, scale."""
    n = tris.shape[0]
    nn = max(2 * n - 1, 1)
    d = dict(left=np.zeros(nn, np.int32), right=np.zeros(nn, np.int32), bmin4=np.zeros((nn, 4), np.float32),
             bmax4=np.zeros((nn, 4), np.float32), sorted_tri=np.zeros(n, np.int32), scene_box=np.zeros(6, np.float32),
             scale=np.zeros(3, np.float32))
    s_in = None if scale is None else np.ascontiguousarray(scale, np.float32)
    load().or_binary_tree(_p(verts), _p(tris), n, METHODS[method], bits, radius, max_radius, adaptive_r, treelet,
                          iterations, sah_bits, ct, ci, _p(s_in), _p(d["left"]), _p(d["right"]), _p(d["bmin4"]),
                          _p(d["bmax4"]), _p(d["sorted_tri"]), _p(d["scene_box"]), _p(d["scale"]))
    return d


def collapse_wide(n, left, right, bmin4, bmax4, sorted_tri, width, ct=3.0, ci=2.0, adaptive=1, max_leaf=8):
    """BVH::collapseAdaptiveWide / collapseWide + BVHConverter::convert, restated:
    (nodes [count, 8*width] int32, triangle order, (interior, leaves))."""
    nodes = np.zeros((max(2 * n - 1, 2), 8 * width), np.int32)
    tri = np.zeros(max(n, 1), np.int32)
    counts = np.zeros(2, np.int32)
    c = load().or_collapse_wide(n, _p(np.ascontiguousarray(sorted_tri, np.int32)),
                                _p(np.ascontiguousarray(left, np.int32)), _p(np.ascontiguousarray(right, np.int32)),
                                _p(np.ascontiguousarray(bmin4, np.float32)),
                                _p(np.ascontiguousarray(bmax4, np.float32)), width, ct, ci,
                                0x7FFFFFFF if adaptive else max_leaf, _p(nodes), _p(tri), _p(counts))
    return nodes[:c], tri[:n], (int(counts[0]), int(counts[1]))


def build_wide(verts, tris, width, method="lbvh", bits=60, radius=16, max_radius=256, adaptive_r=0, treelet=9,
               iterations=2, ct=3.0, ci=2.0, adaptive=1, max_leaf=8, scale=None, sah_bits=15):
    """Whole build into the Quad (4) or Oct (8) layout: dict of nodes, woop, tri_idx, counts, box, scale."""
    n = tris.shape[0]
    nodes = np.zeros((max(2 * n - 1, 2), 8 * width), np.int32)
    woop = np.zeros((max(n, 1), 12), np.float32)
    tri = np.zeros(max(n, 1), np.int32)
    counts = np.zeros(2, np.int32)
    box = np.zeros(6, np.float32)
    sc = np.zeros(3, np.float32)
    s_in = None if scale is None else np.ascontiguousarray(scale, np.float32)
    c = load().or_build_wide(_p(verts), _p(tris), n, METHODS[method], bits, radius, max_radius, adaptive_r, treelet,
                             iterations, sah_bits, ct, ci, adaptive, max_leaf, width, _p(s_in), _p(nodes), _p(woop), _p(tri),
                             _p(counts), _p(box), _p(sc))
    return dict(nodes=nodes[:c], woop=woop[:n], tri_idx=tri[:n], counts=counts, box=box, scale=sc)


def cost(nodes, scene_box, ct=3.0, ci=2.0):
    return load().or_cost(_p(np.ascontiguousarray(nodes)), nodes.shape[0],
                          _p(np.ascontiguousarray(scene_box, np.float32)), ct, ci)


def trace(nodes, woop, tri_idx, rays, any_hit=False, stats=False):
    r = rays.shape[0]
    res = np.zeros((r, 4), np.int32)
    st = np.zeros((r, 2), np.int32) if stats else None
    load().or_trace(_p(np.ascontiguousarray(nodes)), _p(np.ascontiguousarray(woop)),
                    _p(np.ascontiguousarray(tri_idx)), tri_idx.shape[0], _p(np.ascontiguousarray(rays)), r,
                    _p(res), _p(st), int(any_hit))
    return (res, st) if stats else res


def brute64(verts, tris, rays):
    out = np.zeros((rays.shape[0], 4), np.float64)
    load().or_brute64(_p(verts), _p(tris), tris.shape[0], _p(np.ascontiguousarray(rays)), rays.shape[0], _p(out))
    return out


def adjoint64(verts, tris, rays, results, dl):
    out = np.zeros(verts.shape, np.float64)
    load().or_adjoint64(_p(verts), _p(tris), _p(np.ascontiguousarray(rays)), _p(np.ascontiguousarray(results)),
                        _p(np.ascontiguousarray(dl, np.float32)), rays.shape[0], _p(out))
    return out


def intersect64(v0, v1, v2, o, d, tmin=0.0):
    tuv = np.zeros(3, np.float64)
    a = [np.ascontiguousarray(x, np.float64) for x in (v0, v1, v2, o, d)]
    hit = load().or_intersect64(*[_p(x) for x in a], tmin, _p(tuv))
    return bool(hit), tuv


def canonical(nodes, tri_idx):
    """Canonical form of a collapsed binary BVH (node numbering and the order of
    triangles inside a leaf removed): (rows [count, 13] int32 = 12 child-box
    words + size word per node in depth-first order, leaf triangle ids sorted
    per leaf in visit order)."""
    nodes = np.ascontiguousarray(nodes, np.int32)
    tri_idx = np.ascontiguousarray(tri_idx, np.int32)
    rows = np.zeros((max(nodes.shape[0], 1), 13), np.int32)
    tris = np.zeros(max(tri_idx.shape[0], 1), np.int32)
    c = load().or_canonical(_p(nodes), nodes.shape[0], _p(tri_idx), tri_idx.shape[0], _p(rows), _p(tris))
    if c < 0:
        raise ValueError("not a tree over these node and triangle arrays")
    return rows[:c], tris[:tri_idx.shape[0]]


class gen:
    """The benchmark's synthetic inputs, generated without the GPU library (the
    same streams as hippie_b200.gen, checked equal byte for byte)."""

    @staticmethod
    def uniform_mesh(seed, n, half_extent=0.01):
        v = np.empty((3 * n, 3), np.float32)
        t = np.empty((n, 3), np.int32)
        load().or_gen_uniform_mesh(seed, n, half_extent, _p(v), _p(t))
        return v, t

    @staticmethod
    def clustered_mesh(seed, n, clusters=1024, sigma=0.02, half_extent=0.005):
        v = np.empty((3 * n, 3), np.float32)
        t = np.empty((n, 3), np.int32)
        load().or_gen_clustered_mesh(seed, n, clusters, sigma, half_extent, _p(v), _p(t))
        return v, t

    @staticmethod
    def rays_targeted(seed, n, lo=-0.5, hi=1.5):
        r = np.empty((n, 8), np.float32)
        load().or_gen_rays_targeted(seed, n, lo, hi, _p(r))
        return r

    @staticmethod
    def rays_sphere(seed, n, box):
        r = np.empty((n, 8), np.float32)
        load().or_gen_rays_sphere(seed, n, _p(np.ascontiguousarray(box, np.float32)), _p(r))
        return r
