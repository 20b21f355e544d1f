"""ctypes declarations for libsurface_rt.so (include/surface_rt.h).

The library is the product: there is no CPU fallback.  ``load()`` raises if
the shared object is missing and cannot be built, and ``Context`` raises if no
CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import build as _build

SRT_OK, SRT_ERR_INVALID, SRT_ERR_CUDA, SRT_ERR_NO_MEMORY, SRT_ERR_LIMIT, SRT_ERR_UNSUPPORTED = range(6)
SRT_TRIANGLES, SRT_TETRAHEDRA, SRT_SPHERES = 0, 1, 2
MISS = 0xFFFFFFFF
SRT_TRACE_SINGLE_PASS = 1
SRT_TRACE_SORT_RAYS = 2
SRT_TRACE_GRID = 4


class Camera(C.Structure):
    """srt_camera (include/surface_rt.h)."""
    _fields_ = [("eye", C.c_float * 3), ("lookat", C.c_float * 3), ("up", C.c_float * 3),
                ("fov", C.c_float), ("ortho", C.c_int32), ("width", C.c_int32),
                ("height", C.c_int32), ("viewport", C.c_int32 * 4),
                ("region", C.c_int32 * 4), ("step", C.c_int32)]


class CameraSamples(C.Structure):
    """srt_camera_samples (include/surface_rt.h)."""
    _fields_ = [("subsamples", C.c_int32), ("stereo_env", C.c_int32),
                ("zero_parallax", C.c_float), ("eye_separation", C.c_float),
                ("jitter_seed", C.c_uint64), ("jitter_offset", C.c_uint64)]


class VolumeSampling(C.Structure):
    """srt_volume_sampling (include/surface_rt.h)."""
    _fields_ = [("remap", C.c_void_p * 3), ("remap_n", C.c_uint32 * 3),
                ("clamp", C.c_int32 * 3)]


class CacheKey(C.Structure):
    """srt_cache_key (include/surface_rt.h)."""
    _fields_ = [("elem_buffer", C.c_uint64), ("array_buffer", C.c_uint64),
                ("position_offset", C.c_uint64), ("count", C.c_uint32), ("offset", C.c_uint32)]


class CacheInfo(C.Structure):
    """srt_cache_info (include/surface_rt.h)."""
    _fields_ = [("bytes_used", C.c_uint64), ("bytes_max", C.c_uint64),
                ("static_entries", C.c_uint64), ("dynamic_entries", C.c_uint64),
                ("hits", C.c_uint64), ("builds", C.c_uint64)]


RAY_DTYPE = np.dtype([("org", "<f4", 3), ("prev_prim", "<u4"), ("dir", "<f4", 3),
                      ("prev_t", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("prim", "<u4")])
# srt_isect: BuildIntersection's shading record of a hit (80 bytes)
ISECT_DTYPE = np.dtype([("position", "<f4", 3), ("f0", "<u4"), ("normal", "<f4", 3),
                        ("f1", "<u4"), ("tangent", "<f4", 3), ("f2", "<u4"),
                        ("binormal", "<f4", 3), ("f3", "<u4"), ("d", "<f4", 4)])
VOL_DTYPE = np.dtype([("width", "<i4"), ("height", "<i4"), ("max_steps", "<i4"),
                      ("reserved", "<i4"), ("eye", "<f4", 3), ("corner", "<f4", 3),
                      ("du", "<f4", 3), ("dv", "<f4", 3), ("step", "<f4"),
                      ("sigma_scale", "<f4"), ("alpha_max", "<f4")])


class SurfaceError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"surface_rt error {status}: {msg}")
        self.status = status


class TraceOpts(C.Structure):
    _fields_ = [("prev_normals", C.c_void_p), ("subface", C.c_void_p),
                ("vertex_scalar", C.c_void_p), ("scalar_out", C.c_void_p),
                ("normal_out", C.c_void_p), ("stats", C.c_void_p),
                ("flags", C.c_uint32), ("max_iter", C.c_uint32), ("isect", C.c_void_p)]


class AccelInfo(C.Structure):
    _fields_ = [("kind", C.c_int32), ("node_bytes", C.c_int32), ("num_prims", C.c_uint64),
                ("num_nodes", C.c_uint64), ("num_branches", C.c_uint64),
                ("num_leaves", C.c_uint64), ("scene_min", C.c_float * 3),
                ("scene_max", C.c_float * 3), ("eps_scale", C.c_double)]


_P = C.c_void_p
_SZ = C.c_size_t
_S = C.c_int

# name -> argtypes (all return srt_status unless listed in _RESTYPES)
_SIGS = {
    "srt_ctx_create": [C.c_int, C.POINTER(_P)],
    "srt_ctx_destroy": [_P],
    "srt_ctx_set_stream": [_P, _P],
    "srt_ctx_get_stream": [_P],
    "srt_ctx_synchronize": [_P],
    "srt_last_error": [],
    "srt_ctx_launch_count": [_P],
    "srt_accel_create": [_P, C.c_int, C.POINTER(_P)],
    "srt_accel_destroy": [_P],
    "srt_accel_build_triangles": [_P, _P, _SZ, _P, _SZ],
    "srt_accel_build_tetrahedra": [_P, _P, _SZ, _P, _SZ],
    "srt_accel_build_tetrahedra_double": [_P, _P, _SZ, _P, _SZ],
    "srt_accel_build_spheres": [_P, _P, _P, C.c_float, _SZ],
    "srt_build_triangles": [_P, _P, _SZ, _P, _SZ, C.POINTER(_P)],
    "srt_build_tetrahedra": [_P, _P, _SZ, _P, _SZ, C.POINTER(_P)],
    "srt_build_spheres": [_P, _P, _P, C.c_float, _SZ, C.POINTER(_P)],
    "srt_accel_bbox": [_P, _P, _P],
    "srt_accel_info_get": [_P, C.POINTER(AccelInfo)],
    "srt_accel_export": [_P, _P, _P, _P],
    "srt_accel_dump": [_P, C.c_char_p],
    "srt_trace_closest": [_P, _P, _SZ, _P, C.POINTER(TraceOpts)],
    "srt_trace_closest_noalloc": [_P, _P, _SZ, _P],
    "srt_stage_morton": [_P, C.c_int, _P, _SZ, _P, _P, C.c_float, _SZ, _P, _P],
    "srt_stage_sort_pairs": [_P, _P, _P, _SZ],
    "srt_stage_karras": [_P, _P, _SZ, _P, _P, _P],
    "srt_volume_camera": [C.c_int32, C.c_int32, _P, _P, _P, C.c_float, _P],
    "srt_volume_march_fwd": [_P, _P, _P, _P, _P, C.c_int32, _P, _P],
    "srt_volume_march_bwd": [_P, _P, _P, _P, _P, C.c_int32, _P, _P, _P, _P, _P],
    "srt_volume_march_fwd_ex": [_P, _P, _P, _P, _P, _P, C.c_int32, _P, _P],
    "srt_volume_march_bwd_ex": [_P, _P, _P, _P, _P, _P, C.c_int32, _P, _P, _P, _P, _P],
    "srt_spawn_secondary": [_P, _P, _P, _P, _SZ, C.c_uint64, _P, _P, _P],
    "srt_camera_rays": [_P, _P, _P, _P, _P],
    "srt_scene_create": [_P, C.POINTER(_P)],
    "srt_scene_destroy": [_P],
    "srt_scene_add": [_P, _P, _P, _P, _P, _P, _P, _P],
    "srt_scene_add_element": [_P, _P, _P, _P],
    "srt_scene_add_lines": [_P, _P, _P, _P],
    "srt_scene_add_solids": [_P, _P, _P, _P],
    "srt_matrix_inverse": [_P],
    "srt_scene_build": [_P],
    "srt_scene_trace": [_P, _P, _SZ, _P, _P, _P, _P, _P],
    "srt_scene_top_nodes": [_P, _P, _P, _SZ],
    "srt_framebuffer_write": [_P, _P, _P, _P, _P, C.c_uint32, C.c_int32, _P, _P],
    "srt_camera_rays_ex": [_P, _P, _P, _P, _P, _P, _P],
    "srt_framebuffer_write_ex": [_P, _P, _P, _P, _P, _P, C.c_uint32, C.c_int32, _P, _P],
    "srt_accel_load_triangles": [_P, C.c_char_p, _P, _SZ, _P, _SZ],
    "srt_accel_load_tetrahedra": [_P, C.c_char_p, _P, _SZ, _P, _SZ],
    "srt_accel_load_spheres": [_P, C.c_char_p, _P, _P, C.c_float, _SZ],
    "srt_cache_create": [_P, C.c_uint64, C.POINTER(_P)],
    "srt_cache_destroy": [_P],
    "srt_cache_build_triangles": [_P, _P, C.c_int, _P, _SZ, _P, _SZ, C.POINTER(_P)],
    "srt_cache_build_tetrahedra": [_P, _P, C.c_int, _P, _SZ, _P, _SZ, C.POINTER(_P)],
    "srt_cache_build_spheres": [_P, _P, C.c_int, _P, _P, C.c_float, _SZ, C.POINTER(_P)],
    "srt_cache_invalidate": [_P, C.c_uint64],
    "srt_cache_end_frame": [_P],
    "srt_cache_info_get": [_P, _P],
    "srt_texture3d_create": [_P, C.POINTER(_P)],
    "srt_texture3d_destroy": [_P],
    "srt_texture3d_set_dense": [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "srt_texture3d_set_wrap": [_P, C.c_int, C.c_int, C.c_int],
    "srt_texture3d_set_remap": [_P, C.c_int, _P, _SZ],
    "srt_texture3d_set_sparse": [_P, C.c_int, C.c_int, _P, _P, _SZ, _P, _SZ],
    "srt_texture3d_fetch": [_P, _P, _SZ, _P],
    "srt_line_create": [_P, C.POINTER(_P)],
    "srt_line_destroy": [_P],
    "srt_line_build": [_P, _P, _SZ, _P, C.c_float, _P, _SZ, C.c_int32, C.c_int32, C.c_int32],
    "srt_line_trace": [_P, _P, _SZ, _P, _P, _P],
    "srt_line_bbox": [_P, _P, _P],
    "srt_line_info": [_P, _P, _P, _P],
    "srt_line_export": [_P, _P, _P],
    "srt_line_dump": [_P, C.c_char_p],
    "srt_cache_build_lines": [_P, _P, C.c_int, _P, _SZ, _P, C.c_float, _P, _SZ, C.c_int32,
                              C.POINTER(_P)],
    "srt_cache_build_solids": [_P, _P, C.c_int, C.c_int32, _P, _SZ, _P, _SZ, C.POINTER(_P)],
    "srt_solid_create": [_P, C.POINTER(_P)],
    "srt_solid_destroy": [_P],
    "srt_solid_build": [_P, C.c_int32, _P, _SZ, _P, _SZ],
    "srt_solid_build_sah": [_P, C.c_int32, _P, _SZ, _P, _SZ],
    "srt_solid_build_sah_double": [_P, C.c_int32, _P, _SZ, _P, _SZ],
    "srt_solid_build_double": [_P, C.c_int32, _P, _SZ, _P, _SZ],
    "srt_solid_trace": [_P, _P, _SZ, _P, _P, _P],
    "srt_solid_bbox": [_P, _P, _P],
    "srt_solid_info": [_P, _P, _P],
    "srt_solid_export": [_P, _P, _P],
    "srt_solid_dump": [_P, C.c_char_p],
    "srt_batch_create": [_P, C.POINTER(_P)],
    "srt_batch_destroy": [_P],
    "srt_batch_build_trace": [_P, C.c_int32, _P, _P, _P, _P, _P, _P],
    "srt_batch_config": [_P, _P, _P, _P, _P],
    "srt_batch_tuning": [_P, _P, _P, _P, _P],
    "srt_batch_set_tuning": [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32],
}
_RESTYPES = {"srt_last_error": C.c_char_p, "srt_ctx_get_stream": _P,
             "srt_scene_top_nodes": _SZ, "srt_matrix_inverse": None,
             "srt_ctx_launch_count": C.c_uint64}

_lib = None
_lock = threading.Lock()


def library_path():
    return _build.LIB


def load():
    """Load libsurface_rt.so, building it first if it is absent or stale."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(_build.LIB):
            try:
                _build.build()
            except Exception as e:  # noqa: BLE001
                raise ImportError(f"libsurface_rt.so is missing and could not be built: {e}")
        L = C.CDLL(_build.LIB)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, _S)
        _lib = L
        return L


def check(status):
    if status != SRT_OK:
        raise SurfaceError(status, load().srt_last_error().decode(errors="replace"))
    return status


def exported_symbols():
    return list(_SIGS)
