"""Sample-parallel film reduction across ranks, on CPU with the gloo backend
(world size 2).  Each rank "renders" a deterministic stand-in film for its
sample range; the reduced film must equal one rank rendering every sample,
and the sample ranges must be disjoint and cover everything."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from firefly_b200 import multigpu

W, H, SPP, STEPS = 16, 8, 4, 3


def fake_render(offset, spp):
    """Film of samples [offset, offset + spp): radiance of a sample is a fixed hash of (pixel, sample)."""
    pix = np.arange(W * H)[:, None]
    smp = offset + np.arange(spp)[None, :]
    val = ((pix * 2654435761 + smp * 40503) % 1000 / 1000.0).astype(np.float64)
    rgba = np.zeros((H * W, 4), np.float64)
    rgba[:, 0] = val.sum(1)
    rgba[:, 1] = (val * val).sum(1)
    counts = np.full(H * W, spp, np.int64)
    return rgba.reshape(H, W, 4), counts.reshape(H, W)


def worker(rank, world, port, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    acc = torch.zeros((H, W, 4), dtype=torch.float64)
    cnt = torch.zeros((H, W), dtype=torch.int64)
    seen = []
    for step in range(STEPS):
        off = multigpu.sample_offset(rank, world, SPP, step)
        seen.extend(range(off, off + SPP))
        rgba, counts = fake_render(off, SPP)
        r, c = torch.from_numpy(rgba), torch.from_numpy(counts)
        multigpu.allreduce_film(r, c)
        acc += r
        cnt += c
    gathered = [None] * world
    dist.all_gather_object(gathered, seen)
    if rank == 0:
        out_q.put((acc.numpy(), cnt.numpy(), gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_sample_parallel_film_reduce_world2():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 300
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    acc, cnt, gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    samples = sorted(s for g in gathered for s in g)
    assert samples == list(range(world * SPP * STEPS)), "sample ranges must be disjoint and complete"
    ref, ref_cnt = fake_render(0, world * SPP * STEPS)
    assert np.array_equal(cnt, ref_cnt)
    assert np.allclose(acc, ref, rtol=1e-12)


TEX = 32   # texels of the stand-in gradient


def fake_adjoint(offset, spp):
    """Gradient estimate from samples [offset, offset + spp): the mean over
    the samples of a fixed hash of (texel, sample), as the adjoint weighs each
    sample by 1/spp."""
    tex = np.arange(TEX)[:, None]
    smp = offset + np.arange(spp)[None, :]
    return (((tex * 2246822519 + smp * 3266489917) % 997) / 997.0 - 0.5).mean(1)


def grad_worker(rank, world, port, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    off = multigpu.inverse_sample_offset(rank, SPP)
    g_tex = torch.from_numpy(fake_adjoint(off, SPP))
    g_env = torch.from_numpy(2.0 * fake_adjoint(off, SPP))
    multigpu.allreduce_mean([g_tex, g_env])
    offs = [None] * world
    dist.all_gather_object(offs, off)
    if rank == 0:
        out_q.put((g_tex.numpy(), g_env.numpy(), offs))
    dist.barrier()
    dist.destroy_process_group()


def test_inverse_gradient_average_world2():
    """Each rank adjoints its own samples of a step; the averaged gradient
    equals one process adjointing all of them, and the ranges are disjoint."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() + 150) % 300
    procs = [ctx.Process(target=grad_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    g_tex, g_env, offs = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(offs) == [r * SPP for r in range(world)]
    ref = fake_adjoint(0, world * SPP)
    assert np.allclose(g_tex, ref, rtol=1e-12, atol=1e-15)
    assert np.allclose(g_env, 2.0 * ref, rtol=1e-12, atol=1e-15)
