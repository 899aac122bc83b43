"""torch.autograd.Function over ff_render / ff_render_adjoint (test
infrastructure: used by the gradient tests only)."""
from __future__ import annotations

import numpy as np
import torch


class RenderFn(torch.autograd.Function):
    """image = render(albedo_texture, env_map); backward by path replay."""

    @staticmethod
    def forward(ctx, albedo, env, ds, tracer, settings):
        ds.set_texture(0, albedo.detach().cpu().numpy())
        ds.set_environment(env.detach().cpu().numpy(), keep_tables=settings.get("keep_tables", False))
        tracer.clear_buffer()
        kw = {k: v for k, v in settings.items() if k != "keep_tables"}
        tracer.draw(ds, mode=1, **kw)
        img = tracer.image()
        ctx.save_for_backward(albedo, env)
        ctx.ds, ctx.tracer, ctx.settings = ds, tracer, kw
        return torch.from_numpy(img.astype(np.float32))

    @staticmethod
    def backward(ctx, grad_img):
        albedo, env = ctx.saved_tensors
        g_tex = np.zeros(albedo.shape, np.float32)
        g_env = np.zeros(env.shape, np.float32)
        h, w = grad_img.shape[:2]
        kw = {k: v for k, v in ctx.settings.items() if k not in ("max_paths",)}
        ctx.ds.render_adjoint(w, h, grad_img.detach().cpu().numpy(), texture=0, grad_texture=g_tex, grad_env=g_env, **kw)
        return torch.from_numpy(g_tex), torch.from_numpy(g_env), None, None, None
