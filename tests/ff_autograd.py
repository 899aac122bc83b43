"""torch.autograd.Function over ff_render / ff_render_adjoint (test
infrastructure: used by the gradient tests only)."""
from __future__ import annotations

import numpy as np
import torch


class RenderFn(torch.autograd.Function):
    """image = render(albedo_texture, env_map[, roughness_texture]); backward by
    path replay.  The albedo is texture 0; a roughness tensor, when given, is
    texture 1 (channel 0 is read).  settings: ff_render settings, plus
    keep_tables (keep the environment's importance tables) and decorrelate
    (the adjoint draws its own samples: with the primal's samples the descent
    would also minimise the image's variance)."""

    @staticmethod
    def forward(ctx, albedo, env, ds, tracer, settings, rough=None):
        ds.set_texture(0, albedo.detach().cpu().numpy())
        if rough is not None:
            ds.set_texture(1, rough.detach().cpu().numpy())
        ds.set_environment(env.detach().cpu().numpy(), keep_tables=settings.get("keep_tables", False))
        tracer.clear_buffer()
        kw = {k: v for k, v in settings.items() if k not in ("keep_tables", "decorrelate")}
        tracer.draw(ds, mode=1, **kw)
        img = tracer.image()
        ctx.save_for_backward(albedo, env)
        ctx.rough_shape = None if rough is None else tuple(rough.shape)
        ctx.ds, ctx.tracer, ctx.settings = ds, tracer, kw
        ctx.decorrelate = bool(settings.get("decorrelate", False))
        return torch.from_numpy(img.astype(np.float32))

    @staticmethod
    def backward(ctx, grad_img):
        albedo, env = ctx.saved_tensors
        g_tex = np.zeros(albedo.shape, np.float32)
        g_env = np.zeros(env.shape, np.float32)
        h, w = grad_img.shape[:2]
        kw = {k: v for k, v in ctx.settings.items() if k not in ("max_paths",)}
        if ctx.decorrelate:
            kw["seed"] = kw.get("seed", 0) + 0x40000000
        extra = {}
        g_rough = None
        if ctx.rough_shape is not None:
            g_rough = np.zeros(ctx.rough_shape, np.float32)
            extra = dict(roughness_texture=1, grad_roughness=g_rough)
        ctx.ds.render_adjoint(w, h, grad_img.detach().cpu().numpy(), texture=0, grad_texture=g_tex, grad_env=g_env,
                              **extra, **kw)
        return (torch.from_numpy(g_tex), torch.from_numpy(g_env), None, None, None,
                None if g_rough is None else torch.from_numpy(g_rough))
