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


def trace_brute(tris: np.ndarray, rays: np.ndarray, any_hit: bool = False, threads: int | None = None) -> np.ndarray:
    """Brute-force reference query over a triangle soup (T x 9) for rays (n x 8)."""
    lib = load()
    tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = np.empty(rays.shape[0], HIT_DTYPE)
    lib.ffo_trace_brute(_p(tris), tris.shape[0], _p(rays), rays.shape[0], _p(out), int(any_hit),
                        threads or os.cpu_count() or 1)
    return out


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
