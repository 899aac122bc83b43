"""ctypes loader of oracle/_ref/libffref.so: the reference's own routines
compiled for the host (recipe: oracle/Makefile, target `ref`).  TEST
INFRASTRUCTURE and CPU BASELINE ONLY: used by tests/golden/make_golden.py,
the tests, and bench.py's CPU-baseline / reference arm.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libffref.so"
P = C.c_void_p


class RenderDesc(C.Structure):
    _fields_ = [("tris", P), ("normals", P), ("material_ids", P), ("num_tris", C.c_int), ("mats", P),
                ("num_mats", C.c_int), ("env_rgb", P), ("env_w", C.c_int), ("env_h", C.c_int), ("rect", P),
                ("cam_inv", P), ("lens_radius", C.c_float), ("focal", C.c_float), ("width", C.c_int),
                ("height", C.c_int), ("spp", C.c_int), ("max_depth", C.c_int), ("rr_depth", C.c_int),
                ("light_env", C.c_int), ("threads", C.c_int), ("pixel_stride", C.c_int)]


_lib = None


def available() -> bool:
    return LIB.exists()


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        lib = C.CDLL(str(LIB))
        lib.ffref_render.restype = None
        lib.ffref_render.argtypes = [C.POINTER(RenderDesc), P, P, P]
        lib.ffref_bvh_build.restype = P
        lib.ffref_bvh_build.argtypes = [P, C.c_int, C.POINTER(C.c_double)]
        lib.ffref_bvh_trace.restype = None
        lib.ffref_bvh_trace.argtypes = [P, P, C.c_long, P, C.c_int, C.c_int]
        lib.ffref_bvh_free.restype = None
        lib.ffref_bvh_free.argtypes = [P]
        lib.ffref_bvh_num_nodes.restype = C.c_int
        lib.ffref_bvh_num_nodes.argtypes = [P]
        lib.ffref_bvh_data.restype = None
        lib.ffref_bvh_data.argtypes = [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(C.c_int)]
        lib.ffref_sizes.restype = None
        lib.ffref_sizes.argtypes = [C.POINTER(C.c_int)] * 3
        _lib = lib
    return _lib


def render(scene, width, height, spp, max_depth=3, rr_depth=3, light=-1, threads=None, pixel_stride=1,
           want_image=False):
    """The reference's path tracer on the host.  Returns (image sums or None,
    (extension rays, visibility rays, samples), (render ms, setup ms))."""
    lib = load()
    tris = scene.triangle_soup()
    nrm = np.ascontiguousarray(scene.normals[scene.indices].reshape(-1, 9), np.float32)
    mids = None if scene.material_ids is None else np.ascontiguousarray(scene.material_ids, np.uint32)
    mats = np.zeros((max(1, len(scene.materials)), 8), np.float32)
    for i, m in enumerate(scene.materials):
        mats[i, 0:3] = list(m.base_color)
        mats[i, 3:6] = list(m.fresnel)
        mats[i, 6], mats[i, 7] = m.roughness, m.metallic
    env = None if scene.env_rgb is None else np.ascontiguousarray(scene.env_rgb, np.float32)
    rect = None
    if light >= 0:
        L = scene.area_lights[light]
        rect = np.array([*L.p0, *L.a, *L.b, *L.normal, L.radiance, *L.emissive], np.float32)
    inv = np.array(scene.camera.inv_view_proj, np.float32)
    d = RenderDesc()
    d.tris, d.normals = tris.ctypes.data, nrm.ctypes.data
    d.material_ids = None if mids is None else mids.ctypes.data
    d.num_tris = len(tris)
    d.mats, d.num_mats = mats.ctypes.data, len(mats)
    d.env_rgb = None if env is None else env.ctypes.data
    d.env_w = 0 if env is None else env.shape[1]
    d.env_h = 0 if env is None else env.shape[0]
    d.rect = None if rect is None else rect.ctypes.data
    d.cam_inv = inv.ctypes.data
    d.lens_radius, d.focal = scene.camera.lens_radius, scene.camera.focal_distance
    d.width, d.height, d.spp, d.max_depth, d.rr_depth = width, height, spp, max_depth, rr_depth
    d.light_env = 1 if light < 0 else 0
    d.threads = threads or os.cpu_count() or 1
    d.pixel_stride = pixel_stride
    out = np.zeros((height, width, 3), np.float32) if want_image else None
    stats = np.zeros(3, np.uint64)
    ms = np.zeros(2, np.float64)
    lib.ffref_render(C.byref(d), None if out is None else out.ctypes.data, stats.ctypes.data, ms.ctypes.data)
    return out, tuple(int(x) for x in stats), (float(ms[0]), float(ms[1]))
