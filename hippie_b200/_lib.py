"""ctypes bindings of include/hippie_b200.h (libhippie_b200.so, built in-tree).

Loading fails loudly when the library is missing: there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libhippie_b200.so"

HP_OK = 0
STATUS_NAMES = {0: "HP_OK", 1: "HP_ERR_CUDA", 2: "HP_ERR_ARG", 3: "HP_ERR_OOM", 4: "HP_ERR_TIMEOUT",
                5: "HP_ERR_DEVICE_STATUS", 6: "HP_ERR_UNSUPPORTED", 7: "HP_ERR_PARSE"}

HP_METHOD_LBVH, HP_METHOD_PLOC, HP_METHOD_ATR = 0, 1, 2
HP_TRACE_ANY_HIT, HP_TRACE_STATS = 1, 2
HP_BATCH_NO_GRAPH = 0x100
HP_LAYOUT_BIN, HP_LAYOUT_QUAD, HP_LAYOUT_OCT = 2, 4, 8
HP_METHOD_TR = 3
HP_METHOD_HLBVH = 4


class hp_mesh(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("triangles", C.c_void_p),
                ("num_vertices", C.c_int64), ("num_triangles", C.c_int64)]


class hp_build_params(C.Structure):
    _fields_ = [("method", C.c_int32), ("morton_bits", C.c_int32), ("ploc_radius", C.c_int32),
                ("ploc_max_radius", C.c_int32), ("ploc_adaptive", C.c_int32),
                ("atr_iterations", C.c_int32), ("atr_treelet", C.c_int32), ("ct", C.c_float),
                ("ci", C.c_float), ("max_leaf_size", C.c_int32), ("adaptive_leaf", C.c_int32),
                ("layout", C.c_int32), ("hlbvh_sah_bits", C.c_int32), ("reserved", C.c_int32 * 3)]


class hp_bvh(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("woop", C.c_void_p), ("tri_indices", C.c_void_p),
                ("num_refs", C.c_int64), ("capacity_refs", C.c_int64), ("num_interior", C.c_int32),
                ("num_leaf", C.c_int32), ("scene_box", C.c_float * 6), ("morton_scale", C.c_float * 3),
                ("method", C.c_int32), ("ct", C.c_float), ("ci", C.c_float), ("impl", C.c_void_p),
                ("layout", C.c_int32), ("node_bytes", C.c_int32)]


class hp_bvh_stats(C.Structure):
    _fields_ = [("sah_cost", C.c_double), ("avg_leaf_size", C.c_double), ("sum_of_leaf_sizes", C.c_int64),
                ("num_interior", C.c_int32), ("num_leaf", C.c_int32),
                ("leaf_size_histogram", C.c_float * 33), ("pad", C.c_int32)]


class hp_host_scene(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("triangles", C.POINTER(C.c_int32)),
                ("num_vertices", C.c_int64), ("num_triangles", C.c_int64), ("box", C.c_float * 6)]


class hp_tune(C.Structure):
    _fields_ = [("sort_block", C.c_int32), ("trace_ctas_per_sm", C.c_int32), ("trace_stack", C.c_int32),
                ("trace_sorted", C.c_int32), ("ploc_radius", C.c_int32), ("ploc_adaptive", C.c_int32),
                ("ploc_max_radius", C.c_int32), ("build_ms", C.c_float), ("trace_ms", C.c_float),
                ("reserved", C.c_int32 * 7)]


class hp_build_taps(C.Structure):
    _fields_ = [("morton_keys", C.c_void_p), ("sorted_keys", C.c_void_p), ("sorted_refs", C.c_void_p),
                ("node_parent", C.c_void_p), ("node_left", C.c_void_p), ("node_right", C.c_void_p),
                ("node_box_min", C.c_void_p), ("node_box_max", C.c_void_p), ("scene_box", C.c_void_p)]


# name -> (restype, argtypes)
_P = C.c_void_p
_SIGS = {
    "hp_ctx_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32]),
    "hp_ctx_destroy": (C.c_int, [_P]),
    "hp_ctx_check": (C.c_int, [_P, _P]),
    "hp_last_error": (C.c_char_p, []),
    "hp_abi_version": (C.c_int32, []),
    "hp_profile_enable": (C.c_int, [_P, C.c_int32]),
    "hp_profile_reset": (C.c_int, [_P]),
    "hp_profile_count": (C.c_int32, [_P]),
    "hp_profile_get": (C.c_int, [_P, C.c_int32, C.c_char_p, C.c_int64, C.POINTER(C.c_float)]),
    "hp_launch_count": (C.c_int64, []),
    "hp_build_params_default": (None, [C.POINTER(hp_build_params)]),
    "hp_build": (C.c_int, [_P, C.POINTER(hp_mesh), C.POINTER(hp_build_params), C.POINTER(hp_bvh),
                           C.POINTER(hp_build_taps), _P]),
    "hp_bvh_sync": (C.c_int, [_P, C.POINTER(hp_bvh), _P]),
    "hp_bvh_free": (C.c_int, [_P, C.POINTER(hp_bvh)]),
    "hp_bvh_download": (C.c_int, [_P, C.POINTER(hp_bvh), _P, _P, _P, _P]),
    "hp_bvh_cost": (C.c_int, [_P, C.POINTER(hp_bvh), C.POINTER(C.c_double), _P]),
    "hp_bvh_validate": (C.c_int, [_P, C.POINTER(hp_bvh), C.POINTER(hp_mesh), C.POINTER(C.c_int32), _P]),
    "hp_bvh_stats_get": (C.c_int, [_P, C.POINTER(hp_bvh), C.POINTER(hp_bvh_stats), _P]),
    "hp_refit": (C.c_int, [_P, C.POINTER(hp_bvh), C.POINTER(hp_mesh), _P]),
    "hp_trace": (C.c_int, [_P, C.POINTER(hp_bvh), _P, C.c_int64, _P, _P, C.c_uint32, _P]),
    "hp_trace_adjoint": (C.c_int, [_P, C.POINTER(hp_mesh), _P, _P, _P, C.c_int64, _P, _P]),
    "hp_batch_create": (C.c_int, [_P, C.POINTER(hp_mesh), C.c_int32, C.POINTER(C.c_int64),
                                  C.POINTER(hp_build_params), C.POINTER(C.c_void_p)]),
    "hp_batch_destroy": (C.c_int, [_P]),
    "hp_batch_info": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "hp_batch_ray_offset": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int64)]),
    "hp_batch_build": (C.c_int, [_P, _P, C.c_uint32, _P]),
    "hp_batch_trace": (C.c_int, [_P, _P, _P, _P, _P, C.c_uint32, _P]),
    "hp_batch_build_trace": (C.c_int, [_P, _P, _P, _P, _P, C.c_uint32, _P]),
    "hp_batch_bvh": (C.c_int, [_P, C.c_int32, C.POINTER(hp_bvh)]),
    "hp_trace_sorted": (C.c_int, [_P, C.POINTER(hp_bvh), _P, C.c_int64, _P, _P, C.c_uint32, C.c_int32, _P, _P]),
    "hp_trace_host": (C.c_int, [_P, C.POINTER(hp_bvh), _P, C.c_int64, _P, _P, C.c_uint32, C.c_int64, _P]),
    "hp_pixel_table": (C.c_int, [C.c_int32, C.c_int32, _P]),
    "hp_scene_read_bin": (C.c_int, [C.c_char_p, C.POINTER(hp_host_scene)]),
    "hp_scene_write_bin": (C.c_int, [C.c_char_p, C.POINTER(hp_host_scene)]),
    "hp_scene_read_obj": (C.c_int, [C.c_char_p, C.POINTER(hp_host_scene)]),
    "hp_scene_normalize": (C.c_int, [C.POINTER(hp_host_scene)]),
    "hp_scene_load": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(hp_host_scene)]),
    "hp_scene_free": (None, [C.POINTER(hp_host_scene)]),
    "hp_camera_screen_to_world": (C.c_int, [_P, _P, C.c_float, C.c_int32, C.c_int32, C.c_float, C.c_float, _P]),
    "hp_gen_primary_rays": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, C.c_float, C.c_int32, _P, _P, _P]),
    "hp_ray_keys": (C.c_int, [_P, _P, C.c_int64, _P, C.c_int32, _P, _P]),
    "hp_ctx_set_ray_keys": (C.c_int, [_P, C.c_int32, C.c_float]),
    "hp_ray_keys_method": (C.c_int32, [C.c_char_p]),
    "hp_tune_default": (None, [C.POINTER(hp_tune)]),
    "hp_ctx_set_tune": (C.c_int, [_P, C.POINTER(hp_tune)]),
    "hp_ctx_get_tune": (C.c_int, [_P, C.POINTER(hp_tune)]),
    "hp_autotune": (C.c_int, [_P, C.POINTER(hp_mesh), C.POINTER(hp_build_params), _P, C.c_int64, C.c_uint32,
                              C.POINTER(hp_tune), _P]),
    "hp_radix_sort": (C.c_int, [_P, _P, _P, _P, _P, C.c_int64, C.c_int32, C.c_int32, _P]),
    "hp_radix_sort_noalloc": (C.c_int, [_P, _P, _P, _P, C.c_int64, C.c_int32, C.c_int32, _P, _P]),
    "hp_ctx_set_sort_spin_limit": (C.c_int, [_P, C.c_uint32]),
    "hp_ctx_set_arithmetic": (C.c_int, [_P, C.c_int32]),
    "hp_ctx_set_checked": (C.c_int, [_P, C.c_int32]),
    "hp_ctx_get_checked": (C.c_int32, [_P]),
    "hp_bvh_reserve": (C.c_int, [_P, C.POINTER(hp_bvh), C.c_int64, C.c_int32]),
    "hp_bvh_set_info": (C.c_int, [_P, C.POINTER(hp_bvh), C.c_int32, C.c_int32, _P, _P, _P]),
    "hp_env_create": (C.c_int, [C.POINTER(C.c_void_p)]),
    "hp_env_destroy": (C.c_int, [_P]),
    "hp_env_read_file": (C.c_int, [_P, C.c_char_p]),
    "hp_env_read_string": (C.c_int, [_P, C.c_char_p]),
    "hp_env_get_int": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int32)]),
    "hp_env_get_float": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_float)]),
    "hp_env_get_bool": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int32)]),
    "hp_env_get_string": (C.c_int, [_P, C.c_char_p, C.c_char_p, C.c_int64]),
    "hp_env_build_params": (C.c_int, [_P, C.POINTER(hp_build_params)]),
    "hp_gen_uniform_mesh": (C.c_int, [C.c_uint64, C.c_int64, C.c_float, _P, _P]),
    "hp_gen_clustered_mesh": (C.c_int, [C.c_uint64, C.c_int64, C.c_int32, C.c_float, C.c_float, _P, _P]),
    "hp_gen_heightfield": (C.c_int, [C.c_uint64, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_int32,
                                     _P, _P]),
    "hp_gen_rays_targeted": (C.c_int, [C.c_uint64, C.c_int64, C.c_float, C.c_float, _P]),
    "hp_gen_rays_sphere": (C.c_int, [C.c_uint64, C.c_int64, _P, _P]),
    "hp_gen_rays_grid_down": (C.c_int, [C.c_uint64, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float,
                                        _P]),
}

_lib = None


def load():
    """Load libhippie_b200.so (building it first if sources are present and it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        if os.environ.get("HP_NO_AUTOBUILD"):
            raise RuntimeError(f"{LIB_PATH} is missing; run `python -m hippie_b200.build`")
        from . import build as _build
        _build.build()
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    """Names declared in the C header that the library must export."""
    return sorted(_SIGS)


class HPError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status: int):
    if status != HP_OK:
        raise HPError(status, load().hp_last_error().decode(errors="replace"))
