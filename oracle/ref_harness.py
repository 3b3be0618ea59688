"""ctypes access to oracle/_ref/libhipref.so: the reference's own CUDA kernels
driven by a restatement of its host sequences (test infrastructure only).

Built from the reference sources by oracle/ref/Makefile where they are
present; the library then travels with the repository. Tests skip when it is
absent.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libhipref.so"
_lib = None
_P = C.c_void_p


def available() -> bool:
    return LIB.exists()


def load():
    global _lib
    if _lib is None:
        lib = C.CDLL(str(LIB))
        lib.hpref_build.restype = C.c_int
        lib.hpref_build.argtypes = [C.c_int, _P, _P, C.c_int, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                    C.c_float, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                    C.POINTER(C.c_double), _P]
        lib.hpref_trace.restype = C.c_int
        lib.hpref_trace.argtypes = [_P, _P, _P, _P, C.c_int, _P, C.c_int, C.POINTER(C.c_double)]
        lib.hpref_last_error.restype = C.c_char_p
        lib.hpref_last_error.argtypes = []
        lib.hpref_wide_collapse.restype = C.c_int
        lib.hpref_wide_collapse.argtypes = [C.c_int, _P, _P, _P, _P, _P, C.c_int, C.c_float, C.c_float, C.c_int,
                                            C.c_int, _P, _P, _P]
        lib.hpref_bvh_cost.restype = C.c_float
        lib.hpref_bvh_cost.argtypes = [_P, C.c_int, C.c_float, C.c_float, C.c_float]
        _lib = lib
    return _lib


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def build(V, T, scene_box, method="lbvh", bits=60, radius=16, max_radius=256, adaptive_r=0, ct=3.0, ci=2.0,
          taps=False, treelet=20, iterations=2, sah_bits=15):
    """Run the reference's build on device tensors V (float32 [v,3]) and T (int32 [n,3]).

    method: "lbvh", "ploc" (radius / max_radius / adaptive_r), "atr" (treelet /
    iterations) or "hlbvh" (sah_bits)."""
    import torch
    n = T.shape[0]
    nn = 2 * n - 1
    dev = V.device
    nodes = torch.zeros((nn, 16), dtype=torch.int32, device=dev)
    woop = torch.zeros((n, 12), dtype=torch.float32, device=dev)
    tri = torch.zeros(n, dtype=torch.int32, device=dev)
    tp = {}
    if taps:
        tp = dict(keys=torch.zeros(n, dtype=torch.int64, device=dev), sorted=torch.zeros(n, dtype=torch.int64, device=dev),
                  refs=torch.zeros(n, dtype=torch.int32, device=dev), parent=torch.zeros(nn, dtype=torch.int32, device=dev),
                  left=torch.zeros(nn, dtype=torch.int32, device=dev), right=torch.zeros(nn, dtype=torch.int32, device=dev),
                  bmin=torch.zeros((nn, 4), dtype=torch.float32, device=dev),
                  bmax=torch.zeros((nn, 4), dtype=torch.float32, device=dev))
    counts = np.zeros(2, np.int32)
    secs = C.c_double()
    iters = np.zeros(1, np.int32)
    box = np.ascontiguousarray(scene_box, np.float32)
    code = {"lbvh": 0, "ploc": 1, "atr": 2, "hlbvh": 3}[method]
    if method == "atr":
        radius, max_radius = treelet, iterations
    elif method == "hlbvh":
        radius = sah_bits
    rc = load().hpref_build(code, _p(V), _p(T), n, box.ctypes.data, bits, radius, max_radius,
                            adaptive_r, ct, ci, _p(nodes), _p(woop), _p(tri), _p(tp.get("keys")), _p(tp.get("sorted")),
                            _p(tp.get("refs")), _p(tp.get("parent")), _p(tp.get("left")), _p(tp.get("right")),
                            _p(tp.get("bmin")), _p(tp.get("bmax")), counts.ctypes.data, C.byref(secs),
                            iters.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"reference build failed ({rc}): {load().hpref_last_error().decode()}")
    cnt = int(counts.sum())
    out = dict(nodes=nodes[:cnt].cpu().numpy(), woop=woop.cpu().numpy(), tri_idx=tri.cpu().numpy(),
               counts=counts, seconds=secs.value, iterations=int(iters[0]))
    out.update({k: v.cpu().numpy() for k, v in tp.items()})
    return out


def trace(nodes, woop, tri_idx, R, any_hit=False):
    """Run the reference tracer; nodes/woop/tri_idx/R are device tensors."""
    import torch
    res = torch.zeros((R.shape[0], 4), dtype=torch.int32, device=R.device)
    secs = C.c_double()
    rc = load().hpref_trace(_p(nodes), _p(woop), _p(tri_idx), _p(R), R.shape[0], _p(res), int(any_hit), C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"reference trace failed ({rc})")
    return res.cpu().numpy(), secs.value


def cost(nodes, num_nodes, scene_area, ct=3.0, ci=2.0):
    return float(load().hpref_bvh_cost(_p(nodes), num_nodes, scene_area, ct, ci))


def wide_collapse(n, left, right, bmin4, bmax4, sorted_tri, width, ct=3.0, ci=2.0, adaptive=1, max_leaf=8):
    """BVH::collapseAdaptiveWide / collapseWide of the reference (host code, rt/bvh/BVH.h)
    on a binary tree given as host arrays; returns (nodes [count, 8*width] int32,
    triangle order, (interior, leaves)), or None when the root's best choice is a leaf."""
    def p(a):
        return np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)
    arrs = [np.ascontiguousarray(a) for a in (left, right, bmin4, bmax4, sorted_tri)]
    nodes = np.zeros((max(2 * n - 1, 2), 8 * width), np.int32)
    tri = np.zeros(max(n, 1), np.int32)
    counts = np.zeros(2, np.int32)
    c = load().hpref_wide_collapse(n, *[a.ctypes.data_as(C.c_void_p) for a in arrs], width, ct, ci, adaptive,
                                   max_leaf, nodes.ctypes.data_as(C.c_void_p), tri.ctypes.data_as(C.c_void_p),
                                   counts.ctypes.data_as(C.c_void_p))
    if c < 0:
        return None
    return nodes[:c], tri[:n], (int(counts[0]), int(counts[1]))
