"""Inverse rendering with the path-replay adjoint: recover an albedo texture
and an environment map from a target image.

Every iteration renders the current parameters (ff_render, corrected mode),
forms dL/dI of L = 0.5 * mean((I - target)^2), runs ff_render_adjoint with
the same settings but an independent seed, and applies one Adam step per
parameter.  The two passes must not share samples: with the same samples
E[dL/dI * dI/dtheta] picks up the covariance of the estimate and the descent
minimises the image's variance (darkening it) instead of its error
(ff_optimizer_adam_step); the environment's importance tables are rebuilt
from the updated map.  Parameters, gradients, moments and images stay on the
device (torch tensors are used only as device buffers).
"""
from __future__ import annotations

import ctypes as C
import time

from . import _abi as A
from . import lib
from . import multigpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def optimize(ds, tracer, target, albedo, env, steps: int = 200, spp: int = 16, lr: float = 1e-2,
             max_depth: int = 3, rr_depth: int = 3, seed: int = 0, light: int = -1, texture: int = 0,
             lr_env: float | None = None, lr_decay: float = 1.0, callback=None, rank: int = 0, world: int = 1,
             group=None) -> dict:
    """target: device float32 [h, w, 3]; albedo [th, tw, 3] and env [eh, ew, 3]:
    device float32 tensors updated in place (env only when its learning rate,
    lr_env, defaulting to lr, is non-zero).  Both rates fall geometrically by
    the factor lr_decay over the run (1: constant): Adam's steps have the
    size of the rate whatever the gradient's signal-to-noise ratio, so with a
    constant rate the texels that few samples see keep drifting by about the
    rate per step once their mean gradient is lost in the Monte Carlo noise.
    With world > 1 (torch.distributed initialised, one process per GPU), rank
    `rank` renders and replays samples [rank * spp, (rank + 1) * spp) of every
    step; the films are summed and the gradients averaged across the ranks
    (firefly_b200.multigpu), so every rank takes the same optimiser step.
    Returns timings and the loss history."""
    lr_env = lr if lr_env is None else lr_env
    import torch
    L = lib()
    ctx = ds.ctx
    dev = albedo.device
    h, w = target.shape[:2]
    g_tex, g_env = torch.zeros_like(albedo), torch.zeros_like(env)
    m_tex, v_tex, m_env, v_env = (torch.zeros_like(x) for x in (albedo, albedo, env, env))
    rgba = torch.empty((h, w, 4), dtype=torch.float32, device=dev)
    cnt = torch.empty((h, w), dtype=torch.int32, device=dev)
    losses, t_primal, t_adjoint, adj_samples, atomics, launches = [], 0.0, 0.0, 0, 0, 0
    # The library runs on the context's stream, torch on its current stream:
    # every hand-over between the two waits for the producer (torch side:
    # torch.cuda.synchronize; library side: ctx.sync).
    for it in range(steps):
        torch.cuda.synchronize(dev)
        rc = L.ff_scene_set_texture(ds.handle, texture, _p(albedo), A.FF_MEM_DEVICE)
        rc |= L.ff_scene_set_environment(ds.handle, _p(env), A.FF_MEM_DEVICE)
        if rc:
            raise RuntimeError(L.ff_last_error_message(ctx.handle).decode())
        tracer.clear_buffer()
        off = multigpu.inverse_sample_offset(rank, spp)
        st = tracer.draw(ds, spp=spp, max_depth=max_depth, rr_depth=rr_depth, seed=seed + it, light=light,
                         mode=A.FF_MODE_CORRECTED, sample_offset=off)
        t_primal += st["ms_total"]
        launches += st["kernel_launches"]
        rc = L.ff_film_read(tracer.film, _p(rgba), _p(cnt), A.FF_MEM_DEVICE)
        if rc:
            raise RuntimeError(L.ff_last_error_message(ctx.handle).decode())
        ctx.sync()
        if world > 1:
            multigpu.allreduce_film(rgba, cnt, group=group)
        img = rgba[..., :3] / cnt.clamp(min=1)[..., None].float()
        diff = img - target
        losses.append(float(0.5 * (diff * diff).mean()))
        d_image = (diff / diff.numel()).contiguous()
        g_tex.zero_()
        g_env.zero_()
        torch.cuda.synchronize(dev)
        s = A.ff_render_settings(spp=spp, max_depth=max_depth, rr_depth=rr_depth, seed=seed + it + 0x40000000,
                                 mode=A.FF_MODE_CORRECTED, light=light, max_paths=0, sample_offset=off, flags=0,
                                 shadow_offset=0.001)
        d = A.ff_adjoint_desc(width=w, height=h, d_image=d_image.data_ptr(), texture=texture,
                              grad_texture=g_tex.data_ptr(), grad_env=g_env.data_ptr(), flags=A.FF_MEM_DEVICE)
        ast = A.ff_render_stats()
        rc = L.ff_render_adjoint(ctx.handle, ds.handle, C.byref(s), C.byref(d), C.byref(ast))
        if rc:
            raise RuntimeError(L.ff_last_error_message(ctx.handle).decode())
        t_adjoint += ast.ms_total
        adj_samples += ast.samples
        atomics += ast.grad_atomics
        launches += ast.kernel_launches + 2
        if world > 1:
            ctx.sync()
            multigpu.allreduce_mean([g_tex, g_env], group=group)
            torch.cuda.synchronize(dev)
        fall = lr_decay ** (it / max(1, steps - 1))
        for prm, g, m, v, hi, rate in ((albedo, g_tex, m_tex, v_tex, 1.0, lr), (env, g_env, m_env, v_env, 1e6, lr_env)):
            if rate == 0:
                continue
            hp = A.ff_adam_params(lr=rate * fall, beta1=0.9, beta2=0.999, eps=1e-8, lo=1e-3, hi=hi, step=it + 1)
            rc = L.ff_optimizer_adam_step(ctx.handle, _p(prm), _p(g), _p(m), _p(v), prm.numel(), C.byref(hp))
            if rc:
                raise RuntimeError(L.ff_last_error_message(ctx.handle).decode())
        ctx.sync()
        if callback:
            callback(it, losses[-1])
    torch.cuda.synchronize(dev)
    return {"losses": losses, "ms_primal": t_primal, "ms_adjoint": t_adjoint, "adjoint_samples": adj_samples,
            "grad_atomics": atomics, "kernel_launches": launches,
            "adjoint_spp_per_s": adj_samples / (t_adjoint / 1e3) if t_adjoint > 0 else 0.0}
