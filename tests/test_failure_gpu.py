"""Error paths that replace the reference's process exits (checkCudaErrors ->
exit(99), CUDA-RayTracer/CudaHelpers.cpp:3-11; m_assert -> abort(),
massert.cpp:3-12), driven without faulting or hanging the GPU:

* a tensor-core wait of the radiance cache that gives up (its poll bound set
  to zero through ff_debug_cache_wait_limit; the MMA itself completes
  normally and the kernel drains it before freeing its tensor memory) must
  return FF_ERR_TIMEOUT, and the cache must work normally afterwards;
* device allocations refused on the host (ff_debug_fail_alloc_after: the
  refusal happens before cudaMalloc is called) must return FF_ERR_OOM from
  whichever call needed the memory, and destroying what was created must
  give every allocation back.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _alloc_stats(lib):
    total, live = C.c_uint64(), C.c_int64()
    assert lib.ff_debug_alloc_stats(C.byref(total), C.byref(live)) == 0
    return total.value, live.value


def _records(scn, n, seed):
    from firefly_b200 import cache as fc
    rng = np.random.default_rng(seed)
    P = np.asarray(scn.positions, np.float64)
    lo, hi = P.min(0), P.max(0)
    pos = lo + (hi - lo) * rng.random((n, 3))
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    return fc.records(pos, wo, nrm, rng.uniform(0.2, 1.0, n), value=rng.uniform(0.0, 2.0, (n, 3)))


def test_cache_wait_that_gives_up_returns_timeout_and_recovers(ctx):
    import firefly_b200 as ff
    from firefly_b200 import _abi as A
    from firefly_b200 import scenes
    from firefly_b200.cache import RadianceCache

    lib = ff.lib()
    scn = scenes.small_room(seed=0)
    ds = ff.dScene(ctx, scn)
    cache = RadianceCache(ds, log2_table_size=14)
    try:
        recs = _records(scn, 1000, seed=3)
        ref = cache.query(recs)
        out = np.empty((len(recs), 3), np.float32)
        assert lib.ff_debug_cache_wait_limit(cache.handle, 0) == A.FF_OK
        st = lib.ff_cache_query(cache.handle, recs.ctypes.data_as(C.c_void_p), len(recs),
                                out.ctypes.data_as(C.c_void_p), A.FF_MEM_HOST)
        assert st == A.FF_ERR_TIMEOUT
        assert b"tensor-core wait" in lib.ff_last_error_message(ctx.handle)
        loss = C.c_float()
        st = lib.ff_cache_train(cache.handle, recs.ctypes.data_as(C.c_void_p), len(recs), 0, C.byref(loss))
        assert st == A.FF_ERR_TIMEOUT
        # back to the built-in bound: the same answers as before the failures
        assert lib.ff_debug_cache_wait_limit(cache.handle, A.FF_DEBUG_WAIT_DEFAULT) == A.FF_OK
        ctx.sync()
        again = cache.query(recs)
        assert np.array_equal(again, ref), "a timed-out call changed the cache"
        # and training works: the loss falls on a fixed batch
        l0 = cache.train(recs)
        for _ in range(20):
            l1 = cache.train(recs)
        assert np.isfinite(l0) and np.isfinite(l1) and l1 < l0
    finally:
        lib.ff_debug_cache_wait_limit(cache.handle, A.FF_DEBUG_WAIT_DEFAULT)
        cache.close()
        ds.close()


def _render_cycle(lib, scn, w, h):
    """Context, scene, film and one render; returns the status of the first
    failing call (0 when all succeed).  Everything created is destroyed."""
    import firefly_b200 as ff
    from firefly_b200 import _abi as A
    ctx = None
    objs = []
    try:
        try:
            ctx = ff.Context(0)
        except ff.FireflyError as e:
            return e.status
        try:
            ds = ff.dScene(ctx, scn)
            objs.append(ds)
            pt = ff.PathTracer(ctx, w, h)
            objs.append(pt)
            pt.draw(ds, spp=2, max_depth=4, rr_depth=3, seed=0, mode=A.FF_MODE_CORRECTED, light=0)
            pt.read()
        except ff.FireflyError as e:
            return e.status
        return A.FF_OK
    finally:
        for o in reversed(objs):
            o.close()
        if ctx is not None:
            ctx.close()


def test_refused_allocations_return_oom_and_leak_nothing():
    import firefly_b200 as ff
    from firefly_b200 import _abi as A
    from firefly_b200 import scenes

    lib = ff.lib()
    w = h = 16
    scn = scenes.small_room(seed=0, width=w, height=h)
    t0, live0 = _alloc_stats(lib)
    assert _render_cycle(lib, scn, w, h) == A.FF_OK
    t1, live1 = _alloc_stats(lib)
    needed = t1 - t0
    assert live1 == live0, "a full cycle leaked device allocations"
    assert needed > 5
    try:
        for k in range(needed):
            lib.ff_debug_fail_alloc_after(k)
            st = _render_cycle(lib, scn, w, h)
            lib.ff_debug_fail_alloc_after(-1)
            assert st == A.FF_ERR_OOM, (k, A.STATUS_NAMES.get(st, st))
            _, live = _alloc_stats(lib)
            assert live == live0, f"refusing allocation {k} leaked {live - live0} allocations"
        # with enough allocations allowed the cycle completes
        lib.ff_debug_fail_alloc_after(needed)
        assert _render_cycle(lib, scn, w, h) == A.FF_OK
    finally:
        lib.ff_debug_fail_alloc_after(-1)
    assert _alloc_stats(lib)[1] == live0
