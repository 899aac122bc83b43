"""ff_trace_host_noalloc: the host-pointer ray query that allocates no device
memory, for callers that cannot allocate (an application whose device memory
is owned by its own pool allocator, or a loop that cannot take the implicit
synchronisation of cudaMalloc / cudaFree).

The entry point is called through the C ABI and its hits must equal those of
ff_trace (the existing entry point) bit for bit, the tolerance of every trace
test here, on two calls in a row: the scratch array it stages through keeps
the previous call's contents, so the second call checks that nothing stale
leaks into it.  Across both calls the library's own count of device
allocations (ff_debug_alloc_stats, every cudaMalloc it makes goes through
one wrapper) must not move, and neither may the device's free memory as the
driver reports it (cudaMemGetInfo through torch.cuda.mem_get_info): the
point of the entry point is that it allocates nothing.  A warm-up call of
each kind comes first, so that loading the kernels' code and resolving the
scratch array's address (one-time costs of the first call on a device, not
allocations of the call) fall outside the measured calls.  The file is named
to be collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, ctx, ds, rays, any_hit):
    import firefly_b200 as ff
    from firefly_b200 import _abi as A
    r = np.ascontiguousarray(rays, np.float32)
    out = np.empty(len(r), ff.HIT_DTYPE)
    flags = A.FF_TRACE_ANY if any_hit else A.FF_TRACE_CLOSEST
    st = lib.ff_trace_host_noalloc(ctx.handle, ds.handle, r.ctypes.data_as(C.c_void_p), len(r),
                                   out.ctypes.data_as(C.c_void_p), flags)
    return st, out


def _alloc_stats(lib):
    total, live = C.c_uint64(), C.c_int64()
    assert lib.ff_debug_alloc_stats(C.byref(total), C.byref(live)) == 0
    return total.value, live.value


def _free_bytes():
    import torch
    return torch.cuda.mem_get_info(0)[0]


def test_noalloc_matches_ff_trace_on_two_calls():
    import firefly_b200 as ff
    from firefly_b200 import _abi as A
    from firefly_b200 import scenes

    lib = ff.lib()
    ctx = ff.Context(0)
    try:
        scn = scenes.small_room(seed=0)
        ds = ff.dScene(ctx, scn)
        warm = scenes.incoherent_rays(scn, 64, seed=100)
        for any_hit in (False, True):
            st, _ = _noalloc(lib, ctx, ds, warm, any_hit=any_hit)
            assert st == A.FF_OK, lib.ff_last_error_message(ctx.handle)
        # call 1: the maximum size, closest-hit
        rays1 = scenes.incoherent_rays(scn, A.FF_NOALLOC_MAX_RAYS, seed=101)
        before, free0 = _alloc_stats(lib), _free_bytes()
        st, got1 = _noalloc(lib, ctx, ds, rays1, any_hit=False)
        assert st == A.FF_OK, lib.ff_last_error_message(ctx.handle)
        assert _alloc_stats(lib) == before, "the first call allocated device memory"
        assert _free_bytes() == free0, "the device's free memory changed across the first call"
        ref1 = ds.trace(rays1)
        assert np.array_equal(got1.view(np.uint32), ref1.view(np.uint32))
        # call 2: fewer rays, any-hit, into the same scratch
        rays2 = scenes.with_random_tmax(scenes.incoherent_rays(scn, 40_000, seed=102), scn, seed=103)
        before, free0 = _alloc_stats(lib), _free_bytes()
        st, got2 = _noalloc(lib, ctx, ds, rays2, any_hit=True)
        assert st == A.FF_OK, lib.ff_last_error_message(ctx.handle)
        assert _alloc_stats(lib) == before, "the second call allocated device memory"
        assert _free_bytes() == free0, "the device's free memory changed across the second call"
        ref2 = ds.trace(rays2, any_hit=True)
        assert np.array_equal(got2.view(np.uint32), ref2.view(np.uint32))
        assert 0 < (got2["prim"] >= 0).sum() < len(rays2)
        # beyond the maximum: rejected with a message naming the limit
        big = np.zeros((A.FF_NOALLOC_MAX_RAYS + 1, 8), np.float32)
        st, _ = _noalloc(lib, ctx, ds, big, any_hit=False)
        assert st == A.FF_ERR_INVALID_ARG
        assert b"FF_NOALLOC_MAX_RAYS" in lib.ff_last_error_message(ctx.handle)
        # device pointers are rejected (this entry point stages host memory)
        st = lib.ff_trace_host_noalloc(ctx.handle, ds.handle, rays1.ctypes.data_as(C.c_void_p), 1,
                                       got1.ctypes.data_as(C.c_void_p), A.FF_MEM_DEVICE)
        assert st == A.FF_ERR_INVALID_ARG
        ds.close()
    finally:
        ctx.close()
