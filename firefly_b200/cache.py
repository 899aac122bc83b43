"""Learned radiance cache (ff_cache_* of the C ABI).

A multiresolution hash grid over the scene box and a 64-wide MLP (4 hidden
ReLU layers, 3 outputs) trained online on the tracer's own paths and queried
at the first rough vertex after the camera hit, where the path then ends.
Forward and backward passes run on the tensor cores (bf16 operands, FP32
accumulation in tensor memory).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A
from . import _check, _ptr, lib

RECORD_DTYPE = A.CACHE_RECORD_DTYPE


def records(pos, wo, normal, roughness, value=None, pixel=None) -> np.ndarray:
    """Structured ff_cache_record array from per-record arrays."""
    pos = np.asarray(pos, np.float32).reshape(-1, 3)
    n = len(pos)
    r = np.zeros(n, RECORD_DTYPE)
    r["pos"] = pos
    r["wo"] = np.asarray(wo, np.float32).reshape(n, 3)
    r["normal"] = np.asarray(normal, np.float32).reshape(n, 3)
    r["roughness"] = np.broadcast_to(np.asarray(roughness, np.float32), (n,))
    if value is not None:
        v = np.asarray(value, np.float32).reshape(n, 3)
        r["value_r"], r["value_g"], r["value_b"] = v[:, 0], v[:, 1], v[:, 2]
    if pixel is not None:
        r["pixel"] = np.asarray(pixel, np.uint32)
    return r


class RadianceCache:
    """ff_cache over the box of `scene` (a firefly_b200.dScene)."""

    def __init__(self, scene, log2_table_size: int = 19, base_resolution: int = 16, max_resolution: int = 2048,
                 seed: int = 0, lr: float = 1e-2, beta1: float = 0.9, beta2: float = 0.99, eps: float = 1e-8,
                 rough_threshold: float = 0.25, train_paths: int = 65536, train_batch: int = 16384):
        self.ctx = scene.ctx
        self.log2_table_size = log2_table_size
        self.params = A.ff_cache_params(log2_table_size=log2_table_size, base_resolution=base_resolution,
                                        max_resolution=max_resolution, seed=seed, lr=lr, beta1=beta1, beta2=beta2,
                                        eps=eps, rough_threshold=rough_threshold, train_paths=train_paths,
                                        train_batch=train_batch, flags=0)
        h = C.c_void_p()
        _check(lib().ff_cache_create(self.ctx.handle, scene.handle, C.byref(self.params), C.byref(h)),
               self.ctx.handle)
        self.handle = h
        self.ctx._children.add(self)

    @property
    def grid_floats(self) -> int:
        return A.FF_CACHE_LEVELS * (1 << self.log2_table_size) * 2

    def close(self):
        if getattr(self, "handle", None) and self.ctx.handle:
            lib().ff_cache_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        _check(lib().ff_cache_reset(self.handle), self.ctx.handle)

    def query(self, recs: np.ndarray) -> np.ndarray:
        recs = np.ascontiguousarray(recs, RECORD_DTYPE)
        out = np.empty((len(recs), 3), np.float32)
        _check(lib().ff_cache_query(self.handle, _ptr(recs), len(recs), _ptr(out), A.FF_MEM_HOST), self.ctx.handle)
        return out

    def train(self, recs: np.ndarray, gradients_only: bool = False) -> float:
        """One optimiser step on the records (value = target radiance); the
        batch's mean relative L2 loss."""
        recs = np.ascontiguousarray(recs, RECORD_DTYPE)
        loss = C.c_float(0.0)
        flags = A.FF_CACHE_GRADIENTS_ONLY if gradients_only else 0
        _check(lib().ff_cache_train(self.handle, _ptr(recs), len(recs), flags, C.byref(loss)), self.ctx.handle)
        return float(loss.value)

    def read_params(self) -> dict:
        mlp = np.empty(A.FF_CACHE_MLP_PARAMS, np.float32)
        gm = np.empty_like(mlp)
        grid = np.empty(self.grid_floats, np.float32)
        gg = np.empty_like(grid)
        _check(lib().ff_cache_read_params(self.handle, _ptr(mlp), _ptr(grid), _ptr(gm), _ptr(gg)), self.ctx.handle)
        L, T = A.FF_CACHE_LEVELS, 1 << self.log2_table_size
        return {"mlp": mlp.reshape(5, 64, 64), "grad_mlp": gm.reshape(5, 64, 64), "grid": grid.reshape(L, T, 2),
                "grad_grid": gg.reshape(L, T, 2)}

    def write_params(self, mlp: np.ndarray | None = None, grid: np.ndarray | None = None):
        m = None if mlp is None else np.ascontiguousarray(mlp, np.float32)
        g = None if grid is None else np.ascontiguousarray(grid, np.float32)
        _check(lib().ff_cache_write_params(self.handle, _ptr(m), _ptr(g)), self.ctx.handle)

    def render(self, scene, tracer, frames: int = 1, max_depth: int = 5, rr_depth: int = 3, seed: int = 0,
               light: int = -1, sample_offset: int = 0, shadow_offset: float = 0.001) -> dict:
        """ff_render_cached: `frames` frames of one cached path per pixel into
        the tracer's film, training the cache as it goes."""
        s = A.ff_render_settings(spp=frames, max_depth=max_depth, rr_depth=rr_depth, seed=seed,
                                 mode=A.FF_MODE_CORRECTED, light=light, max_paths=0, sample_offset=sample_offset,
                                 flags=0, shadow_offset=shadow_offset)
        st = A.ff_render_stats()
        _check(lib().ff_render_cached(self.ctx.handle, scene.handle, self.handle, C.byref(s), tracer.film,
                                      C.byref(st)), self.ctx.handle)
        return {k: getattr(st, k) for k, _ in st._fields_}
