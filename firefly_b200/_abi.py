"""ctypes declarations of include/firefly_b200.h.

Loads firefly_b200/lib/libfirefly_b200.so.  There is no fallback: if the
library is missing or a CUDA device is absent, calls fail with an error.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# FIREFLY_B200_LIB overrides the library location (e.g. an alternative build).
LIB_PATH = Path(os.environ.get("FIREFLY_B200_LIB", Path(__file__).resolve().parent / "lib" / "libfirefly_b200.so"))

FF_OK = 0
FF_ERR_INVALID_ARG = 1
FF_ERR_OOM = 2
FF_ERR_CUDA = 3
FF_ERR_TIMEOUT = 4
FF_ERR_UNSUPPORTED = 5
FF_ERR_INTERNAL = 6
STATUS_NAMES = {0: "FF_OK", 1: "FF_ERR_INVALID_ARG", 2: "FF_ERR_OOM", 3: "FF_ERR_CUDA",
                4: "FF_ERR_TIMEOUT", 5: "FF_ERR_UNSUPPORTED", 6: "FF_ERR_INTERNAL"}

FF_NOALLOC_MAX_RAYS = 65536
FF_MEM_HOST = 0
FF_MEM_DEVICE = 1
FF_TRACE_CLOSEST = 0
FF_TRACE_ANY = 2
FF_TRACE_TWO_SIDED = 4
FF_RENDER_PROFILE = 1
FF_LIGHT_ALL = -2
FF_ADJOINT_STORE_ALL = 4
FF_ADJOINT_MEGAKERNEL = 16
FF_ENV_KEEP_TABLES = 8
FF_CACHE_GRADIENTS_ONLY = 16
FF_CACHE_LEVELS = 16
FF_CACHE_MLP_PARAMS = 5 * 64 * 64
FF_MODE_PARITY = 0
FF_MODE_CORRECTED = 1
FF_DEBUG_WAIT_DEFAULT = 0xFFFFFFFF

FF_MAT_MIX = 0
FF_MAT_DIFFUSE = 1
FF_MAT_CONDUCTOR = 2
FF_MAT_DIELECTRIC = 3
FF_MAT_COAT = 4


class ff_device_opts(C.Structure):
    _fields_ = [("device", C.c_int32), ("stream", C.c_void_p), ("flags", C.c_uint32)]


class ff_material(C.Structure):
    _fields_ = [("base_color", C.c_float * 3), ("emissive", C.c_float * 3), ("fresnel", C.c_float * 3),
                ("roughness", C.c_float), ("metallic", C.c_float), ("radiance", C.c_float), ("ior", C.c_float),
                ("kind", C.c_int32), ("base_color_tex", C.c_int32), ("roughness_tex", C.c_int32),
                ("metallic_tex", C.c_int32), ("metallic_roughness_tex", C.c_int32), ("normal_tex", C.c_int32)]


class ff_texture_desc(C.Structure):
    _fields_ = [("rgb", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32)]


class ff_area_light(C.Structure):
    _fields_ = [("p0", C.c_float * 3), ("a", C.c_float * 3), ("b", C.c_float * 3), ("normal", C.c_float * 3),
                ("emissive", C.c_float * 3), ("radiance", C.c_float)]


class ff_directional_light(C.Structure):
    _fields_ = [("direction", C.c_float * 3), ("emissive", C.c_float * 3), ("radiance", C.c_float),
                ("pad", C.c_float)]


class ff_camera(C.Structure):
    _fields_ = [("inv_view_proj", C.c_float * 16), ("lens_radius", C.c_float), ("focal_distance", C.c_float),
                ("exposure", C.c_float), ("pixel_jitter", C.c_float)]


class ff_scene_desc(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("num_vertices", C.c_uint32),
                ("indices", C.c_void_p), ("num_triangles", C.c_uint32),
                ("normals", C.c_void_p), ("texcoords", C.c_void_p), ("material_ids", C.c_void_p),
                ("materials", C.c_void_p), ("num_materials", C.c_uint32),
                ("textures", C.c_void_p), ("num_textures", C.c_uint32),
                ("env_rgb", C.c_void_p), ("env_width", C.c_uint32), ("env_height", C.c_uint32),
                ("env_color", C.c_float * 3),
                ("area_lights", C.c_void_p), ("num_area_lights", C.c_uint32),
                ("camera", ff_camera), ("flags", C.c_uint32),
                ("directional_lights", C.c_void_p), ("num_directional_lights", C.c_uint32),
                ("tangents", C.c_void_p), ("bitangents", C.c_void_p)]


class ff_scene_stats(C.Structure):
    _fields_ = [("num_triangles", C.c_uint32), ("num_nodes", C.c_uint32), ("num_leaf_refs", C.c_uint32),
                ("bvh_depth", C.c_uint32), ("device_bytes", C.c_uint64), ("build_ms", C.c_float),
                ("scene_lo", C.c_float * 3), ("scene_hi", C.c_float * 3)]


class ff_render_settings(C.Structure):
    _fields_ = [("spp", C.c_uint32), ("max_depth", C.c_uint32), ("rr_depth", C.c_uint32), ("seed", C.c_uint32),
                ("mode", C.c_uint32), ("light", C.c_int32), ("max_paths", C.c_uint32),
                ("sample_offset", C.c_uint32), ("flags", C.c_uint32), ("shadow_offset", C.c_float)]


class ff_render_stats(C.Structure):
    _fields_ = [("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("samples", C.c_uint64),
                ("frames", C.c_uint32), ("ms_total", C.c_float), ("ms_trace_extension", C.c_float),
                ("ms_trace_shadow", C.c_float), ("ms_logic", C.c_float), ("ms_shade", C.c_float),
                ("kernel_launches", C.c_uint32), ("ms_cache_paths", C.c_float), ("ms_cache_train", C.c_float),
                ("ms_cache_query", C.c_float), ("cache_queries", C.c_uint64), ("cache_records", C.c_uint64),
                ("grad_atomics", C.c_uint64), ("grad_atomics_roughness", C.c_uint64), ("ext_nodes", C.c_uint64),
                ("ext_tris", C.c_uint64), ("shadow_nodes", C.c_uint64), ("shadow_tris", C.c_uint64)]


class ff_adjoint_desc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("d_image", C.c_void_p), ("texture", C.c_int32),
                ("grad_texture", C.c_void_p), ("grad_env", C.c_void_p), ("flags", C.c_uint32),
                ("roughness_texture", C.c_int32), ("grad_roughness", C.c_void_p)]


class ff_adam_params(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("lo", C.c_float),
                ("hi", C.c_float), ("step", C.c_uint32)]


class ff_cache_params(C.Structure):
    _fields_ = [("log2_table_size", C.c_uint32), ("base_resolution", C.c_uint32), ("max_resolution", C.c_uint32),
                ("seed", C.c_uint32), ("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("eps", C.c_float), ("rough_threshold", C.c_float), ("train_paths", C.c_uint32),
                ("train_batch", C.c_uint32), ("flags", C.c_uint32)]


# ff_cache_record as a numpy structured dtype (64 bytes)
import numpy as _np  # noqa: E402
CACHE_RECORD_DTYPE = _np.dtype([("pos", _np.float32, 3), ("roughness", _np.float32), ("wo", _np.float32, 3),
                                ("value_r", _np.float32), ("normal", _np.float32, 3), ("value_g", _np.float32),
                                ("pixel", _np.uint32), ("value_b", _np.float32), ("pad", _np.float32, 2)])
assert CACHE_RECORD_DTYPE.itemsize == 64


# Every symbol include/firefly_b200.h declares, with its ctypes signature.
P = C.c_void_p
PP = C.POINTER(C.c_void_p)
SIGNATURES = {
    "ff_context_create": (C.c_int, [C.POINTER(ff_device_opts), PP]),
    "ff_context_destroy": (C.c_int, [P]),
    "ff_last_error_message": (C.c_char_p, [P]),
    "ff_context_sync": (C.c_int, [P]),
    "ff_context_stream": (P, [P]),
    "ff_scene_create": (C.c_int, [P, C.POINTER(ff_scene_desc), PP]),
    "ff_scene_destroy": (C.c_int, [P]),
    "ff_scene_update_camera": (C.c_int, [P, C.POINTER(ff_camera)]),
    "ff_scene_get_stats": (C.c_int, [P, C.POINTER(ff_scene_stats)]),
    "ff_trace": (C.c_int, [P, P, P, C.c_uint64, P, C.c_uint32]),
    "ff_trace_host_noalloc": (C.c_int, [P, P, P, C.c_uint64, P, C.c_uint32]),
    "ff_trace_count": (C.c_int, [P, P, P, C.c_uint64, C.c_uint32, P]),
    "ff_film_create": (C.c_int, [P, C.c_uint32, C.c_uint32, PP]),
    "ff_film_destroy": (C.c_int, [P]),
    "ff_film_clear": (C.c_int, [P]),
    "ff_film_read": (C.c_int, [P, P, P, C.c_uint32]),
    "ff_film_tonemap": (C.c_int, [P, C.c_float, P, C.c_uint32]),
    "ff_render": (C.c_int, [P, P, C.POINTER(ff_render_settings), P, C.POINTER(ff_render_stats)]),
    "ff_scene_read_env_tables": (C.c_int, [P, P, P, P, P]),
    "ff_scene_read_bvh": (C.c_int, [P, P, C.c_uint64, P, C.c_uint64, P, P]),
    "ff_render_adjoint": (C.c_int, [P, P, C.POINTER(ff_render_settings), C.POINTER(ff_adjoint_desc),
                                    C.POINTER(ff_render_stats)]),
    "ff_scene_set_texture": (C.c_int, [P, C.c_uint32, P, C.c_uint32]),
    "ff_scene_set_environment": (C.c_int, [P, P, C.c_uint32]),
    "ff_optimizer_adam_step": (C.c_int, [P, P, P, P, P, C.c_uint64, C.POINTER(ff_adam_params)]),
    "ff_cache_create": (C.c_int, [P, P, C.POINTER(ff_cache_params), PP]),
    "ff_cache_destroy": (C.c_int, [P]),
    "ff_cache_reset": (C.c_int, [P]),
    "ff_cache_query": (C.c_int, [P, P, C.c_uint32, P, C.c_uint32]),
    "ff_cache_train": (C.c_int, [P, P, C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]),
    "ff_cache_read_params": (C.c_int, [P, P, P, P, P]),
    "ff_cache_write_params": (C.c_int, [P, P, P]),
    "ff_render_cached": (C.c_int, [P, P, P, C.POINTER(ff_render_settings), P, C.POINTER(ff_render_stats)]),
    "ff_debug_alloc_stats": (C.c_int, [C.POINTER(C.c_uint64), C.POINTER(C.c_int64)]),
    "ff_debug_fail_alloc_after": (C.c_int, [C.c_int64]),
    "ff_debug_cache_wait_limit": (C.c_int, [P, C.c_uint32]),
    "ff_debug_env_pick": (C.c_int, [P, P, C.c_uint64, P]),
}

_lib = None


def load() -> C.CDLL:
    """Load the shared library (build it first with firefly_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m firefly_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
