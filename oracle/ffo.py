"""ctypes loader of the CPU oracle (oracle/libffo.so).  TEST INFRASTRUCTURE ONLY.

Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libffo.so"
REF_LIB = HERE / "_ref" / "libffref.so"

_lib = None


def build() -> Path:
    srcs = list(HERE.glob("ffo_*.c")) + [HERE / "ffo.h"]
    if not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        P = C.c_void_p
        lib.ffo_intersect_cull.restype = C.c_int
        lib.ffo_intersect_cull.argtypes = [P] * 8
        lib.ffo_shadow_hit.restype = C.c_int
        lib.ffo_shadow_hit.argtypes = [P] * 6
        lib.ffo_trace_brute.restype = None
        lib.ffo_trace_brute.argtypes = [P, C.c_int64, P, C.c_int64, P, C.c_int, C.c_int]
        lib.ffo_trace_brute2.restype = None
        lib.ffo_trace_brute2.argtypes = [P, C.c_int64, P, C.c_int64, P, C.c_int, C.c_int, C.c_int]
        lib.ffo_bvh_build.restype = P
        lib.ffo_bvh_build.argtypes = [P, C.c_int64]
        lib.ffo_bvh_free.restype = None
        lib.ffo_bvh_free.argtypes = [P]
        lib.ffo_bvh_trace.restype = None
        lib.ffo_bvh_trace.argtypes = [P, P, C.c_int64, P, C.c_int, C.c_int, C.c_int]
        lib.ffo_bvh8_trace.restype = C.c_int64
        lib.ffo_bvh8_trace.argtypes = [P, C.c_uint32, P, C.c_uint32, P, C.c_int64, P, C.c_int, C.c_int, P, C.c_int]
        lib.ffo_intersect_two_sided.restype = C.c_int
        lib.ffo_intersect_two_sided.argtypes = [P] * 9
        lib.ffo_probe_dielectric.restype = None
        lib.ffo_probe_dielectric.argtypes = [P, C.c_int, P, P, P, P]
        lib.ffo_probe_dielectric_sample.restype = C.c_int
        lib.ffo_probe_dielectric_sample.argtypes = [P, C.c_int, P, P, C.c_float, C.c_float, C.c_float, P]
        lib.ffo_probe_fresnel_dielectric.restype = C.c_float
        lib.ffo_probe_fresnel_dielectric.argtypes = [C.c_float, C.c_float]
        lib.ffo_probe_coat.restype = None
        lib.ffo_probe_coat.argtypes = [P, P, P, P, P]
        lib.ffo_wang_hash.restype = C.c_uint32
        lib.ffo_wang_hash.argtypes = [C.c_uint32]
        lib.ffo_rand.restype = C.c_float
        lib.ffo_rand.argtypes = [C.c_uint32, C.c_uint32]
        lib.ffo_path_key.restype = C.c_uint32
        lib.ffo_path_key.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


HIT_DTYPE = np.dtype([("t", np.float32), ("u", np.float32), ("v", np.float32), ("prim", np.int32)])


def trace_brute(tris: np.ndarray, rays: np.ndarray, any_hit: bool = False, threads: int | None = None,
                two_sided: bool = False) -> np.ndarray:
    """Brute-force reference query over a triangle soup (T x 9) for rays (n x 8).
    two_sided: closest hits that also take back faces (prim = -2 - id there)."""
    lib = load()
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = np.empty(rays.shape[0], HIT_DTYPE)
    lib.ffo_trace_brute2(_p(tris), tris.shape[0], _p(rays), rays.shape[0], _p(out), int(any_hit), int(two_sided),
                         threads or os.cpu_count() or 1)
    return out


class BVH:
    """The oracle's ray queries over a CPU hierarchy (ffo_bvh.c): the same
    closest hits as trace_brute (ties to the lowest index), for ray sets and
    meshes too large for brute force.  Any-hit reports some occluder."""

    def __init__(self, tris: np.ndarray):
        self._tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
        self._h = load().ffo_bvh_build(_p(self._tris), self._tris.shape[0])
        if not self._h:
            raise MemoryError("ffo_bvh_build failed")

    def trace(self, rays: np.ndarray, any_hit: bool = False, two_sided: bool = False,
              threads: int | None = None) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.empty(rays.shape[0], HIT_DTYPE)
        load().ffo_bvh_trace(self._h, _p(rays), rays.shape[0], _p(out), int(any_hit), int(two_sided),
                             threads or os.cpu_count() or 1)
        return out

    def close(self):
        if getattr(self, "_h", None):
            load().ffo_bvh_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bvh8_trace(nodes: np.ndarray, tris: np.ndarray, rays: np.ndarray, any_hit: bool = False,
               two_sided: bool = False, threads: int | None = None):
    """The device traversal restated (ffo_bvh8.c) over a BVH read back with
    ff_scene_read_bvh: (hits as HIT_DTYPE, node records fetched, triangles
    tested, rays whose traversal overflowed)."""
    nodes = np.ascontiguousarray(nodes, np.uint8)
    tris = np.ascontiguousarray(tris, np.uint8)
    assert nodes.size % 80 == 0 and tris.size % 48 == 0
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = np.empty(rays.shape[0], HIT_DTYPE)
    counts = np.zeros(2, np.uint64)
    errors = load().ffo_bvh8_trace(_p(nodes), nodes.size // 80, _p(tris), tris.size // 48, _p(rays), rays.shape[0],
                                   _p(out), int(any_hit), int(two_sided), _p(counts), threads or os.cpu_count() or 1)
    return out, int(counts[0]), int(counts[1]), int(errors)


def intersect_two_sided(v0, v1, v2, o, d):
    lib = load()
    arrs = [np.ascontiguousarray(x, np.float32) for x in (v0, v1, v2, o, d)]
    t, u, v, back = C.c_float(0), C.c_float(0), C.c_float(0), C.c_int(0)
    ok = lib.ffo_intersect_two_sided(*[_p(a) for a in arrs], C.byref(t), C.byref(u), C.byref(v), C.byref(back))
    return ok, t.value, u.value, v.value, back.value


def _mat5(tint, roughness, ior):
    return np.array([tint[0], tint[1], tint[2], roughness, ior], np.float32)


def dielectric_eval(tint, roughness, ior, back, n, wo, wi):
    """The restated rough dielectric: (f rgb, pdf) of wi given wo."""
    lib = load()
    out = np.zeros(4, np.float32)
    m = _mat5(tint, roughness, ior)
    arrs = [np.ascontiguousarray(x, np.float32) for x in (n, wo, wi)]
    lib.ffo_probe_dielectric(_p(m), int(back), *[_p(a) for a in arrs], _p(out))
    return out[:3].copy(), float(out[3])


def dielectric_sample(tint, roughness, ior, back, n, wo, e0, e1, e2):
    """The restated sampling step: (ok, wi)."""
    lib = load()
    out = np.zeros(3, np.float32)
    m = _mat5(tint, roughness, ior)
    nn, ww = np.ascontiguousarray(n, np.float32), np.ascontiguousarray(wo, np.float32)
    ok = lib.ffo_probe_dielectric_sample(_p(m), int(back), _p(nn), _p(ww), e0, e1, e2, _p(out))
    return bool(ok), out


def fresnel_dielectric(c, n):
    return float(load().ffo_probe_fresnel_dielectric(c, n))


def coat_eval(albedo, roughness, ior, n, wi, wo):
    """The restated coat: (f rgb, pdf of the 50/50 continuation) of wi given wo."""
    lib = load()
    out = np.zeros(4, np.float32)
    m = _mat5(albedo, roughness, ior)
    arrs = [np.ascontiguousarray(x, np.float32) for x in (n, wi, wo)]
    lib.ffo_probe_coat(_p(m), *[_p(a) for a in arrs], _p(out))
    return out[:3].copy(), float(out[3])


def intersect_cull(v0, v1, v2, o, d):
    lib = load()
    arrs = [np.ascontiguousarray(x, np.float32) for x in (v0, v1, v2, o, d)]
    t, u, v = C.c_float(0), C.c_float(0), C.c_float(0)
    ok = lib.ffo_intersect_cull(*[_p(a) for a in arrs], C.byref(t), C.byref(u), C.byref(v))
    return ok, t.value, u.value, v.value


def shadow_hit(v0, v1, v2, o, d):
    lib = load()
    arrs = [np.ascontiguousarray(x, np.float32) for x in (v0, v1, v2, o, d)]
    t = C.c_float(0)
    ok = lib.ffo_shadow_hit(*[_p(a) for a in arrs], C.byref(t))
    return ok, t.value


# ------------------------------------------------------------------ render
class ffo_material(C.Structure):
    _fields_ = [("base_color", C.c_float * 3), ("fresnel", C.c_float * 3), ("roughness", C.c_float),
                ("metallic", C.c_float), ("kind", C.c_int32), ("base_color_tex", C.c_int32),
                ("roughness_tex", C.c_int32), ("metallic_tex", C.c_int32), ("metallic_roughness_tex", C.c_int32),
                ("normal_tex", C.c_int32), ("ior", C.c_float)]


class ffo_texture(C.Structure):
    _fields_ = [("rgb", C.c_void_p), ("width", C.c_int32), ("height", C.c_int32)]


class ffo_area_light(C.Structure):
    _fields_ = [("p0", C.c_float * 3), ("a", C.c_float * 3), ("b", C.c_float * 3), ("normal", C.c_float * 3),
                ("emissive", C.c_float * 3), ("radiance", C.c_float)]


class ffo_render_desc(C.Structure):
    _fields_ = [("tris", C.c_void_p), ("normals", C.c_void_p), ("material_ids", C.c_void_p),
                ("num_tris", C.c_int32), ("texcoords", C.c_void_p), ("textures", C.c_void_p),
                ("num_textures", C.c_int32), ("materials", C.c_void_p), ("num_materials", C.c_int32),
                ("area_lights", C.c_void_p), ("num_area_lights", C.c_int32),
                ("env_rgb", C.c_void_p), ("env_w", C.c_int32), ("env_h", C.c_int32), ("env_color", C.c_float * 3),
                ("cam_inv", C.c_float * 16), ("cam_lens_radius", C.c_float), ("cam_focal", C.c_float),
                ("cam_jitter", C.c_float), ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("sample_offset", C.c_int32), ("max_depth", C.c_int32), ("rr_depth", C.c_int32),
                ("seed", C.c_uint32), ("mode", C.c_int32), ("light", C.c_int32), ("shadow_offset", C.c_float),
                ("threads", C.c_int32), ("dir_lights", C.c_void_p), ("num_dir_lights", C.c_int32),
                ("tangents", C.c_void_p), ("bitangents", C.c_void_p)]


class ffo_dir_light(C.Structure):
    _fields_ = [("direction", C.c_float * 3), ("emissive", C.c_float * 3), ("radiance", C.c_float),
                ("pad", C.c_float)]


def render(scene, width, height, spp, max_depth=3, rr_depth=3, seed=0, mode=0, light=-1, sample_offset=0,
           shadow_offset=0.001, threads=None):
    """Oracle render: per-pixel radiance SUMS (height x width x 3, float64) and
    (extension rays, shadow rays)."""
    lib = load()
    lib.ffo_render.restype = C.c_int
    lib.ffo_render.argtypes = [C.POINTER(ffo_render_desc), C.c_void_p, C.c_void_p]
    tris = scene.triangle_soup()
    if scene.normals is None:
        raise ValueError("oracle render needs per-vertex normals")
    nrm = np.ascontiguousarray(scene.normals[scene.indices].reshape(-1, 9), np.float32)
    mids = None if scene.material_ids is None else np.ascontiguousarray(scene.material_ids, np.uint32)
    mats = (ffo_material * max(1, len(scene.materials)))()
    for i, m in enumerate(scene.materials):
        for k in range(3):
            mats[i].base_color[k] = m.base_color[k]
            mats[i].fresnel[k] = m.fresnel[k]
        mats[i].roughness, mats[i].metallic, mats[i].kind = m.roughness, m.metallic, m.kind
        mats[i].base_color_tex, mats[i].roughness_tex = m.base_color_tex, m.roughness_tex
        mats[i].metallic_tex, mats[i].metallic_roughness_tex = m.metallic_tex, m.metallic_roughness_tex
        mats[i].normal_tex = m.normal_tex
        mats[i].ior = m.ior
    texs = [np.ascontiguousarray(t, np.float32) for t in getattr(scene, "textures", [])]
    tdesc = (ffo_texture * max(1, len(texs)))()
    for i, t in enumerate(texs):
        tdesc[i].rgb, tdesc[i].width, tdesc[i].height = t.ctypes.data, t.shape[1], t.shape[0]
    tc = None
    if scene.texcoords is not None:
        tc = np.ascontiguousarray(scene.texcoords[scene.indices].reshape(-1, 6), np.float32)
    lights = (ffo_area_light * max(1, len(scene.area_lights)))()
    for i, L in enumerate(scene.area_lights):
        for f in ("p0", "a", "b", "normal", "emissive"):
            for k in range(3):
                getattr(lights[i], f)[k] = getattr(L, f)[k]
        lights[i].radiance = L.radiance
    env = None if scene.env_rgb is None else np.ascontiguousarray(scene.env_rgb, np.float32)
    d = ffo_render_desc()
    d.tris, d.normals = tris.ctypes.data, nrm.ctypes.data
    d.material_ids = None if mids is None else mids.ctypes.data
    d.num_tris = len(tris)
    d.texcoords = None if tc is None else tc.ctypes.data
    d.textures, d.num_textures = C.cast(tdesc, C.c_void_p), len(texs)
    d.materials, d.num_materials = C.cast(mats, C.c_void_p), len(scene.materials)
    d.area_lights, d.num_area_lights = C.cast(lights, C.c_void_p), len(scene.area_lights)
    dls = list(getattr(scene, "directional_lights", []) or [])
    dirs = (ffo_dir_light * max(1, len(dls)))()
    for i, L in enumerate(dls):
        for k in range(3):
            dirs[i].direction[k] = L.direction[k]
            dirs[i].emissive[k] = L.emissive[k]
        dirs[i].radiance = L.radiance
    d.dir_lights, d.num_dir_lights = C.cast(dirs, C.c_void_p), len(dls)
    tg = btg = None
    if getattr(scene, "tangents", None) is not None:
        tg = np.ascontiguousarray(np.asarray(scene.tangents, np.float32)[scene.indices].reshape(-1, 9))
        btg = np.ascontiguousarray(np.asarray(scene.bitangents, np.float32)[scene.indices].reshape(-1, 9))
    d.tangents = None if tg is None else tg.ctypes.data
    d.bitangents = None if btg is None else btg.ctypes.data
    d.env_rgb = None if env is None else env.ctypes.data
    d.env_w = 0 if env is None else env.shape[1]
    d.env_h = 0 if env is None else env.shape[0]
    for k in range(3):
        d.env_color[k] = scene.env_color[k]
    cam = scene.camera
    for k in range(16):
        d.cam_inv[k] = cam.inv_view_proj[k]
    d.cam_lens_radius, d.cam_focal, d.cam_jitter = cam.lens_radius, cam.focal_distance, cam.pixel_jitter
    d.width, d.height, d.spp, d.sample_offset = width, height, spp, sample_offset
    d.max_depth, d.rr_depth, d.seed, d.mode, d.light = max_depth, rr_depth, seed, mode, light
    d.shadow_offset = shadow_offset
    d.threads = threads or os.cpu_count() or 1
    out = np.zeros((height, width, 3), np.float64)
    stats = np.zeros(2, np.uint64)
    rc = lib.ffo_render(C.byref(d), out.ctypes.data, stats.ctypes.data)
    if rc == 2:
        raise ValueError("oracle render: a material kind the oracle does not restate")
    if rc != 0:
        raise ValueError("oracle render: invalid light selection")
    return out, (int(stats[0]), int(stats[1]))


def env_build(rgb: np.ndarray):
    """Environment tables of the reference (marginal, conditional, pdf, denom)."""
    lib = load()
    lib.ffo_env_build.restype = None
    lib.ffo_env_build.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    marginal = np.zeros(h, np.float64)
    cond = np.zeros((h, w), np.float64)
    pdf = np.zeros((h, w), np.float32)
    denom = np.zeros(1, np.float64)
    lib.ffo_env_build(rgb.ctypes.data, w, h, marginal.ctypes.data, cond.ctypes.data, pdf.ctypes.data, denom.ctypes.data)
    return marginal, cond, pdf, float(denom[0])
