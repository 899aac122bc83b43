"""firefly_b200 — B200 (sm_100a) wavefront path tracer behind a C ABI.

Python mirror of the reference's host-side interface (JakeKurtz/Firefly,
CUDA-RayTracer/):

* :class:`dScene` — the device scene (dScene.h:13-65): built from triangle
  arrays, materials, lights and a camera; ``update()`` replaces the camera
  (dScene::update, dScene.cpp:55-58).  The BVH is built on the device.
* :class:`PathTracer` — the tracer (PathTracer.h:11-62): ``PathTracer(w, h)``,
  ``draw(scene)`` and ``clear_buffer()``, with a headless film instead of the
  GL surface.
* :meth:`dScene.trace` — closest-hit / any-hit ray queries (wf_extend /
  wf_shadow, kernel.cu:488-543).

Everything runs in libfirefly_b200.so; this module only marshals arguments.
Errors are raised as :class:`FireflyError` carrying the ABI status code.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _abi as A
from ._abi import (FF_LIGHT_ALL, FF_MAT_COAT, FF_MAT_CONDUCTOR, FF_MAT_DIELECTRIC, FF_MAT_DIFFUSE, FF_MAT_MIX,
                   FF_MODE_CORRECTED, FF_MODE_PARITY, FF_TRACE_ANY, FF_TRACE_CLOSEST)

__all__ = ["Context", "dScene", "PathTracer", "FireflyError", "lib", "FF_LIGHT_ALL", "FF_MAT_MIX", "FF_MAT_DIFFUSE",
           "FF_MAT_CONDUCTOR", "FF_MAT_DIELECTRIC", "FF_MAT_COAT", "FF_MODE_PARITY", "FF_MODE_CORRECTED",
           "FF_TRACE_ANY", "FF_TRACE_CLOSEST", "HIT_DTYPE", "RAY_DTYPE"]

RAY_DTYPE = np.dtype([("o", np.float32, 3), ("tmin", np.float32), ("d", np.float32, 3), ("tmax", np.float32)])
HIT_DTYPE = np.dtype([("t", np.float32), ("u", np.float32), ("v", np.float32), ("prim", np.int32)])


class FireflyError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{A.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    return A.load()


def _check(status: int, ctx_ptr=None):
    if status != A.FF_OK:
        msg = lib().ff_last_error_message(ctx_ptr)
        raise FireflyError(status, (msg or b"").decode(errors="replace"))


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    """One CUDA device and one stream (ff_context)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        opts = A.ff_device_opts(device=device, stream=stream, flags=0)
        h = C.c_void_p()
        _check(lib().ff_context_create(C.byref(opts), C.byref(h)))
        self.handle = h
        self.device = device
        self._children = weakref.WeakSet()   # scenes and tracers, closed before the context

    @property
    def stream(self) -> int:
        return lib().ff_context_stream(self.handle)

    def sync(self):
        _check(lib().ff_context_sync(self.handle), self.handle)

    def close(self):
        if getattr(self, "handle", None):
            for child in list(self._children):
                child.close()
            lib().ff_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class dScene:
    """Device scene (ff_scene).  Arrays are copied at construction."""

    def __init__(self, ctx: Context, scene):
        self.ctx = ctx
        s = scene
        self._keep = []
        P = np.ascontiguousarray(s.positions, np.float32)
        I = np.ascontiguousarray(s.indices, np.uint32)
        N = None if s.normals is None else np.ascontiguousarray(s.normals, np.float32)
        T = None if s.texcoords is None else np.ascontiguousarray(s.texcoords, np.float32)
        M = None if s.material_ids is None else np.ascontiguousarray(s.material_ids, np.uint32)
        E = None if s.env_rgb is None else np.ascontiguousarray(s.env_rgb, np.float32)
        mats = (A.ff_material * max(1, len(s.materials)))(*s.materials)
        lights = (A.ff_area_light * max(1, len(s.area_lights)))(*s.area_lights)
        d = A.ff_scene_desc()
        d.positions, d.num_vertices = _ptr(P), P.shape[0]
        d.indices, d.num_triangles = _ptr(I), I.shape[0]
        d.normals, d.texcoords, d.material_ids = _ptr(N), _ptr(T), _ptr(M)
        d.materials = C.cast(mats, C.c_void_p)
        d.num_materials = len(s.materials)
        texs = [np.ascontiguousarray(t, np.float32) for t in getattr(s, "textures", [])]
        self._keep.append(texs)
        tdesc = (A.ff_texture_desc * max(1, len(texs)))()
        for i, t in enumerate(texs):
            tdesc[i].rgb, tdesc[i].width, tdesc[i].height = t.ctypes.data, t.shape[1], t.shape[0]
        self._keep.append(tdesc)
        d.textures = C.cast(tdesc, C.c_void_p) if texs else None
        d.num_textures = len(texs)
        d.env_rgb = _ptr(E)
        d.env_width = 0 if E is None else E.shape[1]
        d.env_height = 0 if E is None else E.shape[0]
        for k in range(3):
            d.env_color[k] = float(s.env_color[k])
        d.area_lights = C.cast(lights, C.c_void_p)
        d.num_area_lights = len(s.area_lights)
        dls = list(getattr(s, "directional_lights", []) or [])
        dirs = (A.ff_directional_light * max(1, len(dls)))(*dls)
        d.directional_lights = C.cast(dirs, C.c_void_p)
        d.num_directional_lights = len(dls)
        tg, btg = getattr(s, "tangents", None), getattr(s, "bitangents", None)
        if (tg is None) != (btg is None):
            raise ValueError("tangents and bitangents come together")
        if tg is not None:
            tg = np.ascontiguousarray(tg, np.float32)
            btg = np.ascontiguousarray(btg, np.float32)
            if tg.shape != P.shape or btg.shape != P.shape:
                raise ValueError("tangents / bitangents: one float3 per vertex")
            self._keep += [tg, btg]
        d.tangents, d.bitangents = _ptr(tg), _ptr(btg)
        if s.camera is not None:
            d.camera = s.camera
        h = C.c_void_p()
        _check(lib().ff_scene_create(ctx.handle, C.byref(d), C.byref(h)), ctx.handle)
        self.handle = h
        self.source = scene
        ctx._children.add(self)

    def update(self, camera: A.ff_camera):
        """dScene::update: replace the camera."""
        _check(lib().ff_scene_update_camera(self.handle, C.byref(camera)), self.ctx.handle)

    def set_texture(self, index: int, rgb: np.ndarray):
        """Replace the texels of texture `index` (same size)."""
        t = np.ascontiguousarray(rgb, np.float32)
        _check(lib().ff_scene_set_texture(self.handle, index, _ptr(t), A.FF_MEM_HOST), self.ctx.handle)

    def set_environment(self, rgb: np.ndarray, keep_tables: bool = False):
        """Replace the environment map's texels (same size); rebuilds the
        importance tables unless keep_tables."""
        e = np.ascontiguousarray(rgb, np.float32)
        flags = A.FF_ENV_KEEP_TABLES if keep_tables else 0
        _check(lib().ff_scene_set_environment(self.handle, _ptr(e), flags), self.ctx.handle)

    def render_adjoint(self, width: int, height: int, d_image: np.ndarray, texture: int = 0, grad_texture=None,
                       grad_env=None, spp: int = 1, max_depth: int = 3, rr_depth: int = 3, seed: int = 0,
                       light: int = -1, sample_offset: int = 0, shadow_offset: float = 0.001,
                       store_all: bool = False, roughness_texture: int = -1, grad_roughness=None,
                       megakernel: bool = False, profile: bool = False) -> dict:
        """Path-replay adjoint of PathTracer.draw(mode=FF_MODE_CORRECTED) with
        the same settings: adds dL/d(texture texels) to grad_texture,
        dL/d(env texels) to grad_env and dL/d(roughness texels) to
        grad_roughness (float32 host arrays shaped like their textures;
        channel 0 where a material reads the texture as its roughness_tex,
        channel 1 where it is the packed metallic_roughness_tex), given
        d_image = dL/dI of the mean-radiance image (height, width, 3).
        The replay runs on the wavefront stages; megakernel=True runs the
        one-thread-per-sample replay instead, store_all=True the store-all
        reference variant.  profile=True times the wavefront stages
        (ms_logic, ms_shade, ms_trace_extension, ms_trace_shadow)."""
        dimg = np.ascontiguousarray(d_image, np.float32)
        s = A.ff_render_settings(spp=spp, max_depth=max_depth, rr_depth=rr_depth, seed=seed,
                                 mode=A.FF_MODE_CORRECTED, light=light, max_paths=0, sample_offset=sample_offset,
                                 flags=A.FF_RENDER_PROFILE if profile else 0, shadow_offset=shadow_offset)
        d = A.ff_adjoint_desc(width=width, height=height, d_image=dimg.ctypes.data, texture=texture,
                              grad_texture=None if grad_texture is None else grad_texture.ctypes.data,
                              grad_env=None if grad_env is None else grad_env.ctypes.data,
                              flags=(A.FF_ADJOINT_STORE_ALL if store_all else 0)
                              | (A.FF_ADJOINT_MEGAKERNEL if megakernel else 0),
                              roughness_texture=roughness_texture,
                              grad_roughness=None if grad_roughness is None else grad_roughness.ctypes.data)
        for g in (grad_texture, grad_env, grad_roughness):
            if g is not None and (g.dtype != np.float32 or not g.flags.c_contiguous):
                raise ValueError("gradient buffers must be contiguous float32")
        st = A.ff_render_stats()
        _check(lib().ff_render_adjoint(self.ctx.handle, self.handle, C.byref(s), C.byref(d), C.byref(st)),
               self.ctx.handle)
        return {k: getattr(st, k) for k, _ in st._fields_}

    def stats(self) -> dict:
        st = A.ff_scene_stats()
        _check(lib().ff_scene_get_stats(self.handle, C.byref(st)), self.ctx.handle)
        return {k: (list(getattr(st, k)) if k.startswith("scene_") else getattr(st, k)) for k, _ in st._fields_}

    def read_bvh(self) -> tuple[np.ndarray, np.ndarray]:
        """The 8-wide BVH as ff_trace walks it (ff_scene_read_bvh): node records
        (num_nodes x 80 bytes, uint8) and triangle records in leaf order
        (num_tris x 48 bytes, uint8)."""
        nn, nt = C.c_uint32(), C.c_uint32()
        _check(lib().ff_scene_read_bvh(self.handle, None, 0, None, 0, C.byref(nn), C.byref(nt)), self.ctx.handle)
        nodes = np.empty((nn.value, 80), np.uint8)
        tris = np.empty((nt.value, 48), np.uint8)
        _check(lib().ff_scene_read_bvh(self.handle, C.c_void_p(nodes.ctypes.data), nodes.nbytes,
                                       C.c_void_p(tris.ctypes.data), tris.nbytes, C.byref(nn), C.byref(nt)),
               self.ctx.handle)
        return nodes, tris

    def trace(self, rays: np.ndarray, any_hit: bool = False, out: np.ndarray | None = None,
              two_sided: bool = False) -> np.ndarray:
        """Host rays (n x 8 float32 or RAY_DTYPE) -> host hits (HIT_DTYPE).

        Synchronous: copies the rays in, traces, copies the hits out.  Pass
        pinned buffers (rays and ``out``) for full copy bandwidth.
        two_sided: closest hits that also take back faces (FF_TRACE_TWO_SIDED;
        a back face reports prim = -2 - index)."""
        if rays.dtype == RAY_DTYPE:
            rays = rays.view(np.float32)
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        if out is None:
            out = np.empty(r.shape[0], HIT_DTYPE)
        elif out.dtype != HIT_DTYPE or out.shape != (r.shape[0],) or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous HIT_DTYPE array with one entry per ray")
        flags = (A.FF_TRACE_ANY if any_hit else A.FF_TRACE_CLOSEST) | (A.FF_TRACE_TWO_SIDED if two_sided else 0)
        _check(lib().ff_trace(self.ctx.handle, self.handle, _ptr(r), r.shape[0], _ptr(out), flags),
               self.ctx.handle)
        return out

    def trace_device(self, rays_ptr: int, n: int, hits_ptr: int, any_hit: bool = False, two_sided: bool = False):
        """Device pointers (e.g. torch tensors' data_ptr()), asynchronous on the context stream."""
        flags = (A.FF_TRACE_ANY if any_hit else A.FF_TRACE_CLOSEST) | A.FF_MEM_DEVICE
        flags |= A.FF_TRACE_TWO_SIDED if two_sided else 0
        _check(lib().ff_trace(self.ctx.handle, self.handle, C.c_void_p(rays_ptr), n, C.c_void_p(hits_ptr), flags),
               self.ctx.handle)

    def trace_count(self, rays, n: int | None = None, any_hit: bool = False, two_sided: bool = False) -> dict:
        """Traversal work of the rays (host array, or a device pointer with
        n): node records fetched, triangles tested, and the fetched bytes per
        ray (records times their sizes), for the same traversal ff_trace runs."""
        flags = (A.FF_TRACE_ANY if any_hit else A.FF_TRACE_CLOSEST) | (A.FF_TRACE_TWO_SIDED if two_sided else 0)
        if isinstance(rays, int):
            ptr, count = C.c_void_p(rays), int(n)
            flags |= A.FF_MEM_DEVICE
        else:
            r = np.ascontiguousarray(rays.view(np.float32) if rays.dtype == RAY_DTYPE else rays,
                                     np.float32).reshape(-1, 8)
            ptr, count = _ptr(r), r.shape[0]
        out = (C.c_uint64 * 4)()
        _check(lib().ff_trace_count(self.ctx.handle, self.handle, ptr, count, flags, out), self.ctx.handle)
        nodes, tris, node_b, tri_b = (int(v) for v in out)
        return {"rays": count, "nodes": nodes, "tris": tris, "node_bytes": node_b, "tri_bytes": tri_b,
                "fetch_bytes_per_ray": (nodes * node_b + tris * tri_b) / max(1, count)}

    def close(self):
        if getattr(self, "handle", None):
            if getattr(self.ctx, "handle", None):
                lib().ff_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PathTracer:
    """The wavefront tracer with its film (PathTracer(w, h), draw, clear_buffer)."""

    def __init__(self, ctx: Context, w: int, h: int):
        self.ctx = ctx
        self.width, self.height = w, h
        f = C.c_void_p()
        _check(lib().ff_film_create(ctx.handle, w, h, C.byref(f)), ctx.handle)
        self.film = f
        self.last_stats = None
        ctx._children.add(self)

    def draw(self, scene: dScene, spp: int = 1, max_depth: int = 3, rr_depth: int = 3, seed: int = 0,
             mode: int = A.FF_MODE_PARITY, light: int = -1, max_paths: int = 0, sample_offset: int = 0,
             shadow_offset: float = 0.001, profile: bool = False) -> dict:
        """PathTracer::draw: render `spp` more samples per pixel into the film."""
        s = A.ff_render_settings(spp=spp, max_depth=max_depth, rr_depth=rr_depth, seed=seed, mode=mode,
                                 light=light, max_paths=max_paths, sample_offset=sample_offset,
                                 flags=A.FF_RENDER_PROFILE if profile else 0, shadow_offset=shadow_offset)
        st = A.ff_render_stats()
        _check(lib().ff_render(self.ctx.handle, scene.handle, C.byref(s), self.film, C.byref(st)), self.ctx.handle)
        self.last_stats = {k: getattr(st, k) for k, _ in st._fields_}
        return self.last_stats

    def clear_buffer(self):
        _check(lib().ff_film_clear(self.film), self.ctx.handle)

    def read(self):
        """(rgba float32 [h, w, 4], n_samples uint32 [h, w])"""
        rgba = np.empty((self.height, self.width, 4), np.float32)
        n = np.empty((self.height, self.width), np.uint32)
        _check(lib().ff_film_read(self.film, _ptr(rgba), _ptr(n), A.FF_MEM_HOST), self.ctx.handle)
        return rgba, n

    def image(self):
        """Mean radiance per pixel (accum / n), float32 [h, w, 3]."""
        rgba, n = self.read()
        return rgba[..., :3] / np.maximum(n, 1)[..., None]

    def save(self, path, exposure: float = 1.0):
        """Tonemapped 8-bit PNG (ff_film_tonemap), or the float mean radiance
        as PFM when the path ends in .pfm."""
        from . import image
        if str(path).lower().endswith(".pfm"):
            image.write_pfm(path, self.image())
        else:
            image.write_png(path, self.tonemap(exposure))

    def tonemap(self, exposure: float = 1.0) -> np.ndarray:
        out = np.empty((self.height, self.width, 4), np.uint8)
        _check(lib().ff_film_tonemap(self.film, exposure, _ptr(out), A.FF_MEM_HOST), self.ctx.handle)
        return out

    def close(self):
        if getattr(self, "film", None):
            if getattr(self.ctx, "handle", None):
                lib().ff_film_destroy(self.film)
            self.film = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
