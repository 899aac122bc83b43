"""Sample-parallel rendering over several GPUs (one process per GPU).

Paths are independent given the scene, so N ranks render one frame by
splitting its samples: rank r renders samples [spp * (r + N * step),
spp * (r + N * step) + spp) of every pixel into its own film, then the films
are summed with one all-reduce per step (the per-frame film reduce; 16 B of
radiance + 4 B of count per pixel, 41 MB at 1920 x 1080).  Every rank holds
the whole scene; nothing else crosses the interconnect.  The reference has
no multi-GPU path (its Interop(multi_gpu) flag only picks a GL blit path).
"""
from __future__ import annotations


def sample_offset(rank: int, world: int, spp: int, step: int) -> int:
    """First sample index rank `rank` renders at `step` (disjoint across ranks and steps)."""
    return spp * (rank + world * step)


def allreduce_film(rgba, counts, group=None):
    """Sum the films (radiance float tensor, sample-count int tensor) of all ranks in place."""
    import torch.distributed as dist
    dist.all_reduce(rgba, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    return rgba, counts


def read_film_device(tracer, rgba, counts):
    """Copy a PathTracer's film into device tensors (float32 [h, w, 4], int32 [h, w])."""
    import ctypes as C
    from . import _abi as A
    from . import lib
    rc = lib().ff_film_read(tracer.film, C.c_void_p(rgba.data_ptr()), C.c_void_p(counts.data_ptr()), A.FF_MEM_DEVICE)
    if rc != 0:
        raise RuntimeError(lib().ff_last_error_message(tracer.ctx.handle).decode())
