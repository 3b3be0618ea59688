"""hippie_b200 — B200-native LBVH/PLOC BVH construction and closest-hit traversal.

Python access to the C ABI (include/hippie_b200.h) for tests and benchmarks.
Device buffers are torch CUDA tensors (plumbing only); all computation happens
in the CUDA kernels of libhippie_b200.so.

Mirrors the reference's builder / tracer objects (src/hippie/rt/bvh/BVHBuilder.h,
rt/bvh/HipBVH.h, rt/tracer/HipTracer.h) as `Context.build`, `BVH`, `Context.trace`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (HP_BATCH_NO_GRAPH, HP_METHOD_ATR, HP_METHOD_LBVH, HP_METHOD_PLOC, HP_TRACE_ANY_HIT,
                   HP_TRACE_STATS, HPError, check, hp_build_params, hp_build_taps, hp_bvh, hp_bvh_stats, hp_host_scene,
                   hp_mesh, hp_tune, load)

__all__ = ["Context", "BVH", "Batch", "BuildParams", "Env", "HPError", "gen", "pixel_table", "Scene",
           "load_scene", "read_scene_bin", "read_scene_obj",
           "camera_screen_to_world", "HP_METHOD_LBVH", "HP_METHOD_PLOC",
           "HP_METHOD_ATR", "HP_TRACE_ANY_HIT", "HP_TRACE_STATS", "load"]


def _ptr(t):
    return C.c_void_p(0) if t is None else C.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


class BuildParams:
    """hp_build_params with the reference's defaults (environment/AppEnvironment.cpp:52-75)."""

    def __init__(self, **kw):
        self.c = hp_build_params()
        load().hp_build_params_default(C.byref(self.c))
        for k, v in kw.items():
            if k == "method" and isinstance(v, str):
                v = {"lbvh": HP_METHOD_LBVH, "ploc": HP_METHOD_PLOC, "atr": HP_METHOD_ATR, "tr": 3, "hlbvh": 4}[v]
            if k == "layout" and isinstance(v, str):
                v = {"bin": 2, "quad": 4, "oct": 8}[v]
            setattr(self.c, k, v)

    def __getattr__(self, k):
        return getattr(self.__dict__["c"], k)


class Env:
    """Environment file (Environment / AppEnvironment) with the reference's keys."""

    def __init__(self):
        self.h = C.c_void_p()
        check(load().hp_env_create(C.byref(self.h)))

    def __del__(self):
        # At interpreter shutdown module globals may already be gone.
        if getattr(self, "h", None) and load is not None:
            load().hp_env_destroy(self.h)
            self.h = None

    def read_string(self, text: str):
        check(load().hp_env_read_string(self.h, text.encode()))
        return self

    def read_file(self, path: str):
        check(load().hp_env_read_file(self.h, str(path).encode()))
        return self

    def get_int(self, name):
        v = C.c_int32()
        check(load().hp_env_get_int(self.h, name.encode(), C.byref(v)))
        return v.value

    def get_float(self, name):
        v = C.c_float()
        check(load().hp_env_get_float(self.h, name.encode(), C.byref(v)))
        return v.value

    def get_bool(self, name):
        v = C.c_int32()
        check(load().hp_env_get_bool(self.h, name.encode(), C.byref(v)))
        return bool(v.value)

    def get_string(self, name):
        buf = C.create_string_buffer(4096)
        check(load().hp_env_get_string(self.h, name.encode(), buf, 4096))
        return buf.value.decode()

    def build_params(self) -> BuildParams:
        p = BuildParams()
        check(load().hp_env_build_params(self.h, C.byref(p.c)))
        return p


class BVH:
    """A built BVH (HipBVH): nodes of its layout (64-byte binary, or Quad / Oct
    records of 32 * N bytes), Woop triangles, triangle indices."""

    def __init__(self, ctx: "Context"):
        self.ctx = ctx
        self.c = hp_bvh()

    def __del__(self):
        if getattr(self, "c", None) is not None and self.c.impl and load is not None and C is not None:
            load().hp_bvh_free(self.ctx.h, C.byref(self.c))

    def sync(self, stream=None):
        check(load().hp_bvh_sync(self.ctx.h, C.byref(self.c), _stream_ptr(stream)))
        return self

    @property
    def num_nodes(self):
        return self.c.num_interior + self.c.num_leaf

    @property
    def layout(self) -> int:
        """Children per node: 2 (bin), 4 (quad) or 8 (oct)."""
        return self.c.layout or 2

    def cost(self, stream=None) -> float:
        v = C.c_double()
        check(load().hp_bvh_cost(self.ctx.h, C.byref(self.c), C.byref(v), _stream_ptr(stream)))
        return v.value

    def stats(self, stream=None) -> dict:
        """HipBVH::getCost / getAvgLeafSize / getLeafSizeHistogram in one device pass."""
        st = hp_bvh_stats()
        check(load().hp_bvh_stats_get(self.ctx.h, C.byref(self.c), C.byref(st), _stream_ptr(stream)))
        return {"sah_cost": st.sah_cost, "avg_leaf_size": st.avg_leaf_size,
                "sum_of_leaf_sizes": st.sum_of_leaf_sizes, "num_interior": st.num_interior,
                "num_leaf": st.num_leaf, "leaf_size_histogram": list(st.leaf_size_histogram)}

    def validate(self, verts, tris, stream=None) -> bool:
        m = _mesh(verts, tris)
        ok = C.c_int32()
        check(load().hp_bvh_validate(self.ctx.h, C.byref(self.c), C.byref(m), C.byref(ok), _stream_ptr(stream)))
        return bool(ok.value)

    @classmethod
    def reserve(cls, ctx: "Context", num_refs: int, layout: int = 2) -> "BVH":
        """Storage for a BVH of num_refs references, to be filled by a copy or
        broadcast of another BVH's arrays and then set_info (hp_bvh_reserve)."""
        b = cls(ctx)
        check(load().hp_bvh_reserve(ctx.h, C.byref(b.c), int(num_refs), int(layout)))
        return b

    def set_info(self, num_interior, num_leaf, scene_box, morton_scale, stream=None):
        box = np.ascontiguousarray(scene_box, np.float32)
        sc = np.ascontiguousarray(morton_scale, np.float32)
        check(load().hp_bvh_set_info(self.ctx.h, C.byref(self.c), int(num_interior), int(num_leaf),
                                     box.ctypes.data, sc.ctypes.data, _stream_ptr(stream)))

    def info(self) -> dict:
        """Node counts, scene box and Morton scale (after sync)."""
        return {"num_interior": self.c.num_interior, "num_leaf": self.c.num_leaf,
                "scene_box": list(self.c.scene_box), "morton_scale": list(self.c.morton_scale)}

    def arrays(self):
        """torch views (no copy) of the device arrays: nodes (capacity rows of
        8 * layout int32), Woop rows (num_refs x 12 float32), triangle indices."""
        import torch
        cap = max(2 * max(self.c.capacity_refs, 2) - 1, 3)
        n = self.c.num_refs
        dev = torch.device("cuda", self.ctx.device)
        return (torch.as_tensor(_DeviceArray(self.c.nodes, (cap, 8 * self.layout), "<i4"), device=dev),
                torch.as_tensor(_DeviceArray(self.c.woop, (n, 12), "<f4"), device=dev),
                torch.as_tensor(_DeviceArray(self.c.tri_indices, (n,), "<i4"), device=dev))

    def download(self, stream=None):
        """Copy nodes (N x 16 int32), woop (n x 12 float32) and triangle indices to the host."""
        self.sync(stream)
        nodes = np.zeros((self.num_nodes, 8 * self.layout), np.int32)
        woop = np.zeros((self.c.num_refs, 12), np.float32)
        tri = np.zeros(self.c.num_refs, np.int32)
        check(load().hp_bvh_download(self.ctx.h, C.byref(self.c), nodes.ctypes.data, woop.ctypes.data,
                                     tri.ctypes.data, _stream_ptr(stream)))
        return nodes, woop, tri


class _DeviceArray:
    """A device buffer of the library described by __cuda_array_interface__ (so
    torch.as_tensor can view it without a copy); the owner must outlive it."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"data": (int(ptr or 0), False), "shape": tuple(shape),
                                         "typestr": typestr, "version": 3}


def _mesh(verts, tris) -> hp_mesh:
    m = hp_mesh()
    m.vertices = verts.data_ptr() if verts is not None and verts.numel() else None
    m.triangles = tris.data_ptr() if tris is not None and tris.numel() else None
    m.num_vertices = verts.shape[0] if verts is not None else 0
    m.num_triangles = tris.shape[0] if tris is not None else 0
    return m


class Context:
    """One hp_ctx per device and host thread (library scratch arena + error words)."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        check(load().hp_ctx_create(C.byref(self.h), device))
        self.device = device

    def close(self):
        if getattr(self, "h", None) and load is not None:
            load().hp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def check(self, stream=None):
        check(load().hp_ctx_check(self.h, _stream_ptr(stream)))

    def build(self, verts, tris, params: BuildParams | None = None, bvh: BVH | None = None, taps=None,
              stream=None) -> BVH:
        """Build (or rebuild into `bvh`) over float32 (V,3) vertices and int32 (T,3) triangles."""
        params = params or BuildParams()
        bvh = bvh or BVH(self)
        m = _mesh(verts, tris)
        tp = None
        if taps is not None:
            tp = hp_build_taps()
            for k, v in taps.items():
                setattr(tp, k, v.data_ptr())
        check(load().hp_build(self.h, C.byref(m), C.byref(params.c), C.byref(bvh.c),
                              C.byref(tp) if tp is not None else None, _stream_ptr(stream)))
        return bvh

    def refit(self, bvh: BVH, verts, tris, stream=None):
        m = _mesh(verts, tris)
        check(load().hp_refit(self.h, C.byref(bvh.c), C.byref(m), _stream_ptr(stream)))

    def trace(self, bvh: BVH, rays, results=None, stats=None, any_hit=False, stream=None):
        """rays: float32 (R, 8) CUDA tensor. Returns int32 (R, 4) results (and stats if given).
        A miss writes only {-1, tmax}; a buffer allocated here starts zeroed."""
        import torch
        n = rays.shape[0]
        if results is None:
            results = torch.zeros((n, 4), dtype=torch.int32, device=rays.device)
        flags = (HP_TRACE_ANY_HIT if any_hit else 0) | (HP_TRACE_STATS if stats is not None else 0)
        check(load().hp_trace(self.h, C.byref(bvh.c), _ptr(rays), n, _ptr(results), _ptr(stats), flags,
                              _stream_ptr(stream)))
        return results

    def trace_host(self, bvh: BVH, rays, results=None, stats=None, any_hit=False, chunk=0, stream=None):
        """hp_trace_host: rays, results and stats in HOST memory (CPU tensors, pinned for
        overlap); chunked uploads, traces and downloads overlap. Every result record is
        written in full (a miss reads {-1, tmax, 0, 0}). Synchronises `stream` before
        returning, so the results are complete."""
        import torch
        n = rays.shape[0]
        assert not rays.is_cuda, "trace_host takes host tensors"
        if results is None:
            results = torch.empty((n, 4), dtype=torch.int32, pin_memory=rays.is_pinned())
        flags = (HP_TRACE_ANY_HIT if any_hit else 0) | (HP_TRACE_STATS if stats is not None else 0)
        check(load().hp_trace_host(self.h, C.byref(bvh.c), _ptr(rays), n, _ptr(results), _ptr(stats), flags,
                                   chunk, _stream_ptr(stream)))
        (torch.cuda.current_stream() if stream is None else stream).synchronize()
        return results

    def trace_sorted(self, bvh: BVH, rays, results=None, stats=None, any_hit=False, bits=30, order=None,
                     stream=None):
        """HipTracer::traceSort: trace in ray Morton order; results at each ray's own index."""
        import torch
        n = rays.shape[0]
        if results is None:
            results = torch.zeros((n, 4), dtype=torch.int32, device=rays.device)
        flags = (HP_TRACE_ANY_HIT if any_hit else 0) | (HP_TRACE_STATS if stats is not None else 0)
        check(load().hp_trace_sorted(self.h, C.byref(bvh.c), _ptr(rays), n, _ptr(results), _ptr(stats), flags,
                                     bits, _ptr(order), _stream_ptr(stream)))
        return results

    RAY_KEY_METHODS = {"two_point": 0, "aila": 1, "paraboloid": 2, "octahedron": 3, "origin": 4, "costa": 5,
                       "reis": 6}

    def set_ray_keys(self, method="aila", ray_length=0.25):
        """RayBuffer::setMortonCodeMethod / setRayLength for this context's ray keys and
        sorted traces: a name of RAY_KEY_METHODS, a renderer env value (hp_ray_keys_method)
        or a method number."""
        if isinstance(method, str):
            m = self.RAY_KEY_METHODS.get(method)
            if m is None:
                m = load().hp_ray_keys_method(method.encode())
        else:
            m = int(method)
        check(load().hp_ctx_set_ray_keys(self.h, m, float(ray_length)))

    def ray_keys(self, rays, bits=30, box=None, stream=None):
        import torch
        keys = torch.empty(rays.shape[0], dtype=torch.int64, device=rays.device)
        b = None if box is None else np.ascontiguousarray(box, np.float32)
        check(load().hp_ray_keys(self.h, _ptr(rays), rays.shape[0], None if b is None else b.ctypes.data, bits,
                                 _ptr(keys), _stream_ptr(stream)))
        return keys

    def primary_rays(self, position, screen_to_world, width, height, max_dist=float("inf"), sample_index=0,
                     index_to_pixel=None, out=None, stream=None):
        """RayGen::primary: width*height pinhole rays (8 floats each) in pixel-table order."""
        import torch
        rays = out if out is not None else torch.empty((width * height, 8), dtype=torch.float32,
                                                       device=f"cuda:{self.device}")
        pos = np.ascontiguousarray(position, np.float32)
        m = np.ascontiguousarray(screen_to_world, np.float32).reshape(16)
        check(load().hp_gen_primary_rays(self.h, pos.ctypes.data, m.ctypes.data, width, height, max_dist,
                                         sample_index, _ptr(index_to_pixel), _ptr(rays), _stream_ptr(stream)))
        return rays

    _TUNE_FIELDS = ("sort_block", "trace_ctas_per_sm", "trace_stack", "trace_sorted", "ploc_radius",
                    "ploc_adaptive", "ploc_max_radius", "build_ms", "trace_ms")

    def get_tune(self) -> dict:
        t = hp_tune()
        check(load().hp_ctx_get_tune(self.h, C.byref(t)))
        return {k: getattr(t, k) for k in self._TUNE_FIELDS}

    def set_tune(self, **kw):
        """Set launch choices (sort_block, trace_ctas_per_sm, trace_stack, trace_sorted); others keep theirs."""
        t = hp_tune()
        check(load().hp_ctx_get_tune(self.h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        check(load().hp_ctx_set_tune(self.h, C.byref(t)))

    def reset_tune(self):
        t = hp_tune()
        load().hp_tune_default(C.byref(t))
        check(load().hp_ctx_set_tune(self.h, C.byref(t)))

    def autotune(self, verts, tris, rays, params: BuildParams | None = None, ploc_radius=False, stream=None) -> dict:
        """hp_autotune on this mesh and rays; applies the result-neutral choices, returns all of them."""
        params = params or BuildParams()
        m = _mesh(verts, tris)
        t = hp_tune()
        check(load().hp_autotune(self.h, C.byref(m), C.byref(params.c), _ptr(rays), rays.shape[0],
                                 1 if ploc_radius else 0, C.byref(t), _stream_ptr(stream)))
        return {k: getattr(t, k) for k in self._TUNE_FIELDS}

    def adjoint(self, verts, tris, rays, results, dl_dtuv, dl_dverts=None, stream=None):
        import torch
        if dl_dverts is None:
            dl_dverts = torch.zeros_like(verts)
        m = _mesh(verts, tris)
        check(load().hp_trace_adjoint(self.h, C.byref(m), _ptr(rays), _ptr(results), _ptr(dl_dtuv),
                                      rays.shape[0], _ptr(dl_dverts), _stream_ptr(stream)))
        return dl_dverts

    def set_arithmetic(self, mode: str = "ieee"):
        """"ieee" (default) or "reference": the reciprocals of the reference's
        fast-math build in Woop rows and in the binary tracer (hp_ctx_set_arithmetic)."""
        check(load().hp_ctx_set_arithmetic(self.h, {"ieee": 0, "reference": 1}[mode]))

    def set_sort_spin_limit(self, spins: int = 0):
        """Spins of one radix-sort look-back wait before it gives up (0: the default)."""
        check(load().hp_ctx_set_sort_spin_limit(self.h, int(spins)))

    def set_checked(self, on: bool = True):
        """Checked mode (hp_ctx_set_checked): every call synchronises and verifies
        its output (BVH validation after build and refit, sortedness after a
        sort, the device error words after a trace), raising HippieError."""
        check(load().hp_ctx_set_checked(self.h, 1 if on else 0))

    @property
    def checked(self) -> bool:
        return bool(load().hp_ctx_get_checked(self.h))

    def radix_sort(self, keys, vals=None, bits=None, stream=None):
        import torch
        kb = keys.element_size()
        bits = bits or 8 * kb
        ko = torch.empty_like(keys)
        vo = torch.empty(keys.shape[0], dtype=torch.int32, device=keys.device)
        check(load().hp_radix_sort(self.h, _ptr(keys), _ptr(vals), _ptr(ko), _ptr(vo), keys.shape[0], kb, bits,
                                   _stream_ptr(stream)))
        return ko, vo


class Batch:
    """Many meshes built (LBVH) and traced in a fixed number of launches (hp_batch_*).

    meshes: list of (vertices, triangles) CUDA tensors, kept alive by the batch.
    rays_per_mesh: ray count of every mesh; the rays of mesh m are rows
    [ray_offset(m), ray_offset(m+1)) of the ray tensor given to trace().
    With graph=True (default) launches replay a CUDA graph, which needs a
    non-default stream (torch.cuda.stream(...))."""

    def __init__(self, ctx: Context, meshes, rays_per_mesh, params: BuildParams | None = None):
        self.ctx = ctx
        self.meshes = list(meshes)
        self.h = C.c_void_p()
        params = params or BuildParams()
        arr = (hp_mesh * max(len(self.meshes), 1))()
        for i, (v, t) in enumerate(self.meshes):
            arr[i] = _mesh(v, t)
        rc = (C.c_int64 * max(len(self.meshes), 1))(*[int(r) for r in rays_per_mesh])
        check(load().hp_batch_create(ctx.h, arr, len(self.meshes), rc, C.byref(params.c), C.byref(self.h)))
        m, n, r = C.c_int32(), C.c_int64(), C.c_int64()
        check(load().hp_batch_info(self.h, C.byref(m), C.byref(n), C.byref(r)))
        self.num_meshes, self.num_triangles, self.num_rays = m.value, n.value, r.value

    def close(self):
        if getattr(self, "h", None) and load is not None:
            load().hp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def ray_offset(self, m: int) -> int:
        v = C.c_int64()
        check(load().hp_batch_ray_offset(self.h, m, C.byref(v)))
        return v.value

    @staticmethod
    def _flags(graph, any_hit=False, stats=None):
        return (0 if graph else HP_BATCH_NO_GRAPH) | (HP_TRACE_ANY_HIT if any_hit else 0) | \
            (HP_TRACE_STATS if stats is not None else 0)

    @staticmethod
    def _stream(stream, graph):
        s = _stream_ptr(stream)
        if graph and not s.value:
            raise ValueError("graph launches need a non-default CUDA stream")
        return s

    def build(self, graph=True, stream=None):
        check(load().hp_batch_build(self.ctx.h, self.h, self._flags(graph), self._stream(stream, graph)))

    def trace(self, rays, results=None, stats=None, any_hit=False, graph=True, stream=None):
        import torch
        if results is None:
            results = torch.empty((self.num_rays, 4), dtype=torch.int32, device=rays.device)
        check(load().hp_batch_trace(self.ctx.h, self.h, _ptr(rays), _ptr(results), _ptr(stats),
                                    self._flags(graph, any_hit, stats), self._stream(stream, graph)))
        return results

    def build_trace(self, rays, results=None, stats=None, any_hit=False, graph=True, stream=None):
        import torch
        if results is None:
            results = torch.empty((self.num_rays, 4), dtype=torch.int32, device=rays.device)
        check(load().hp_batch_build_trace(self.ctx.h, self.h, _ptr(rays), _ptr(results), _ptr(stats),
                                          self._flags(graph, any_hit, stats), self._stream(stream, graph)))
        return results

    def bvh(self, m: int) -> BVH:
        """A non-owning BVH view of mesh m (sync / download / cost / validate / Context.trace)."""
        b = BVH(self.ctx)
        check(load().hp_batch_bvh(self.h, m, C.byref(b.c)))
        b.batch = self  # keeps the batch's storage alive
        return b


class Scene:
    """A host triangle mesh: vertices (V x 3 float32), triangles (T x 3 int32) and
    the box stored with it (min xyz, max xyz, before any normalisation)."""

    def __init__(self, vertices, triangles, box=None):
        self.vertices = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        self.triangles = np.ascontiguousarray(triangles, np.int32).reshape(-1, 3)
        if box is None:
            box = np.concatenate([self.vertices.min(0), self.vertices.max(0)]) if len(self.vertices) else \
                np.zeros(6, np.float32)
        self.box = np.asarray(box, np.float32).copy()

    def _c(self) -> hp_host_scene:
        c = hp_host_scene()
        c.vertices = self.vertices.ctypes.data_as(C.POINTER(C.c_float))
        c.triangles = self.triangles.ctypes.data_as(C.POINTER(C.c_int32))
        c.num_vertices = len(self.vertices)
        c.num_triangles = len(self.triangles)
        c.box[:] = self.box.tolist()
        return c

    @staticmethod
    def _take(c: hp_host_scene) -> "Scene":
        try:
            v = np.ctypeslib.as_array(c.vertices, (c.num_vertices * 3,)).copy() if c.num_vertices else \
                np.zeros(0, np.float32)
            t = np.ctypeslib.as_array(c.triangles, (c.num_triangles * 3,)).copy() if c.num_triangles else \
                np.zeros(0, np.int32)
            return Scene(v, t, np.array(c.box[:], np.float32))
        finally:
            load().hp_scene_free(C.byref(c))

    def write_bin(self, path) -> None:
        """BinExporter::exportScene (zero normals, texture coordinates, material indices)."""
        c = self._c()
        check(load().hp_scene_write_bin(str(path).encode(), C.byref(c)))

    def normalized(self) -> "Scene":
        """SceneLoader::loadStaticScene's normalisation, done by the library."""
        out = Scene(self.vertices.copy(), self.triangles, self.box)
        c = out._c()
        check(load().hp_scene_normalize(C.byref(c)))
        return out


def read_scene_bin(path) -> Scene:
    """BinImporter::importScene: geometry of a scene in the binary cache format."""
    c = hp_host_scene()
    check(load().hp_scene_read_bin(str(path).encode(), C.byref(c)))
    return Scene._take(c)


def read_scene_obj(path) -> Scene:
    """Geometry of a Wavefront OBJ file (polygon fans, degenerate triangles dropped)."""
    c = hp_host_scene()
    check(load().hp_scene_read_obj(str(path).encode(), C.byref(c)))
    return Scene._take(c)


def load_scene(path, write_cache: bool = True) -> Scene:
    """SceneLoader::loadStaticScene: path + ".bin" if present, else the OBJ file
    (cached to path + ".bin" when write_cache), normalised to the unit box."""
    c = hp_host_scene()
    check(load().hp_scene_load(str(path).encode(), 1 if write_cache else 0, C.byref(c)))
    return Scene._take(c)


def pixel_table(width: int, height: int):
    """PixelTable::recalculate: pixel index of every ray slot (host int32 array)."""
    t = np.empty(width * height, np.int32)
    check(load().hp_pixel_table(width, height, t.ctypes.data))
    return t


def camera_screen_to_world(position, direction, fov_deg, width, height, near=0.01, far=100.0):
    """inverse(projection * view) of the reference's Camera, row-major 4x4 (float32)."""
    out = np.empty(16, np.float32)
    p = np.ascontiguousarray(position, np.float32)
    d = np.ascontiguousarray(direction, np.float32)
    check(load().hp_camera_screen_to_world(p.ctypes.data, d.ctypes.data, fov_deg, width, height, near, far,
                                           out.ctypes.data))
    return out.reshape(4, 4)


class gen:
    """Synthetic inputs (host numpy arrays) from the library's deterministic generators."""

    @staticmethod
    def uniform_mesh(seed, n, half_extent=0.01):
        v = np.empty((3 * n, 3), np.float32)
        t = np.empty((n, 3), np.int32)
        check(load().hp_gen_uniform_mesh(seed, n, half_extent, v.ctypes.data, t.ctypes.data))
        return v, t

    @staticmethod
    def clustered_mesh(seed, n, clusters=1024, sigma=0.02, half_extent=0.005):
        v = np.empty((3 * n, 3), np.float32)
        t = np.empty((n, 3), np.int32)
        check(load().hp_gen_clustered_mesh(seed, n, clusters, sigma, half_extent, v.ctypes.data, t.ctypes.data))
        return v, t

    @staticmethod
    def heightfield(seed, nx=512, ny=1024, sx=1.0, sy=2.0, waves=16):
        v = np.empty((nx * ny, 3), np.float32)
        t = np.empty((2 * (nx - 1) * (ny - 1), 3), np.int32)
        check(load().hp_gen_heightfield(seed, nx, ny, sx, sy, waves, v.ctypes.data, t.ctypes.data))
        return v, t

    @staticmethod
    def rays_targeted(seed, n, lo=-0.5, hi=1.5):
        r = np.empty((n, 8), np.float32)
        check(load().hp_gen_rays_targeted(seed, n, lo, hi, r.ctypes.data))
        return r

    @staticmethod
    def rays_sphere(seed, n, box):
        r = np.empty((n, 8), np.float32)
        b = np.ascontiguousarray(box, np.float32)
        check(load().hp_gen_rays_sphere(seed, n, b.ctypes.data, r.ctypes.data))
        return r

    @staticmethod
    def rays_grid_down(seed, nx, ny, sx=1.0, sy=2.0, z0=1.0):
        r = np.empty((nx * ny, 8), np.float32)
        check(load().hp_gen_rays_grid_down(seed, nx, ny, sx, sy, z0, r.ctypes.data))
        return r
