"""The reference's own GPU traversal (oracle/_ref/libffrefcuda.so, built by
`make -C oracle refcuda` from CUDA-RayTracer/dRay.cu + dTriangle.cu) over the
reference's own host-built BVH (oracle/_ref/libffref.so).  TEST
INFRASTRUCTURE ONLY: the "reference CUDA" baseline of the trace benchmark,
and a cross-check of hit ids.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import ffref

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libffrefcuda.so"
P = C.c_void_p
_lib = None


def available() -> bool:
    return LIB.exists() and ffref.available()


def load():
    global _lib
    if _lib is None:
        lib = C.CDLL(str(LIB))
        lib.ffrefcuda_sizes.argtypes = [C.POINTER(C.c_int)] * 3
        lib.ffrefcuda_trace.restype = C.c_int
        lib.ffrefcuda_trace.argtypes = [P, C.c_int, P, C.c_int, P, C.c_long, P, P, C.c_int, C.c_int,
                                        C.POINTER(C.c_float)]
        _lib = lib
    return _lib


class RefGpuBVH:
    """The reference's BVH (host build) ready for its GPU traversal."""

    def __init__(self, tris9: np.ndarray):
        r = ffref.load()
        tris9 = np.ascontiguousarray(tris9, np.float32)
        ms = C.c_double()
        self.h = r.ffref_bvh_build(tris9.ctypes.data, len(tris9), C.byref(ms))
        self.build_ms = ms.value
        self.num_nodes = r.ffref_bvh_num_nodes(self.h)
        nodes, tris, ordered, nt = P(), P(), P(), C.c_int()
        r.ffref_bvh_data(self.h, C.byref(nodes), C.byref(tris), C.byref(ordered), C.byref(nt))
        self.nodes, self.tris, self.num_tris = nodes, tris, nt.value
        self.ordered = np.ctypeslib.as_array(C.cast(ordered, C.POINTER(C.c_int)), shape=(nt.value,)).copy()
        hs = [C.c_int() for _ in range(3)]
        r.ffref_sizes(*[C.byref(x) for x in hs])
        ds = [C.c_int() for _ in range(3)]
        load().ffrefcuda_sizes(*[C.byref(x) for x in ds])
        if [x.value for x in hs] != [x.value for x in ds]:
            raise RuntimeError(f"host and device struct sizes differ: {[x.value for x in hs]} vs {[x.value for x in ds]}")

    def trace(self, rays: np.ndarray, any_hit: bool = False, reps: int = 1):
        """(t float32, original prim int32 or -1 | occluded 1/-1, ms per launch)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = len(rays)
        t = np.empty(n, np.float32)
        prim = np.empty(n, np.int32)
        ms = C.c_float()
        rc = load().ffrefcuda_trace(self.nodes, self.num_nodes, self.tris, self.num_tris, rays.ctypes.data, n,
                                    t.ctypes.data, prim.ctypes.data, int(any_hit), reps, C.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference CUDA trace failed: cudaError {rc}")
        if not any_hit:
            hit = prim >= 0
            prim[hit] = self.ordered[prim[hit]]
        return t, prim, ms.value

    def close(self):
        if self.h:
            ffref.load().ffref_bvh_free(self.h)
            self.h = None
