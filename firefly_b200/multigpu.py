"""Sample-parallel rendering over several GPUs (one process per GPU).

Paths are independent given the scene, so N ranks render one frame by
splitting its samples: rank r renders samples [spp * (r + N * step),
spp * (r + N * step) + spp) of every pixel into its own film, then the films
are summed with one all-reduce per step (the per-frame film reduce; 16 B of
radiance + 4 B of count per pixel, 41 MB at 1920 x 1080).  Every rank holds
the whole scene; nothing else crosses the interconnect.  The reference has
no multi-GPU path (its Interop(multi_gpu) flag only picks a GL blit path).

Inverse rendering shards the same way: every rank renders and replays its
own sample range of each step (inverse_sample_offset), the films are summed
and the texture and environment gradients averaged (allreduce_mean: 3.5 MB
per step at a 512x512 texture and a 256x128 map), and every rank applies the
same optimiser step to its replica of the parameters.
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


def inverse_sample_offset(rank: int, spp: int) -> int:
    """First sample index rank `rank` renders and replays in an inverse-rendering
    step.  Every step draws a fresh seed, so ranks only need disjoint ranges
    within a step: rank r takes samples [r * spp, (r + 1) * spp)."""
    return rank * spp


def allreduce_mean(tensors, group=None):
    """Average tensors over the ranks in place.  Each rank's adjoint weighs its
    samples by 1/spp, so every rank's gradient estimates the whole gradient
    and the mean of N of them is the estimate from all N * spp samples."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        if world > 1:
            t.div_(world)
    return tensors
