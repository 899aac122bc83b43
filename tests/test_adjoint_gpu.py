"""Path-replay adjoint (wavefront stages by default, one-thread-per-sample
megakernel as a cross-check): against the store-all-vertices adjoint, against FP64
central finite differences with common random numbers (same seeds, so every
path not touching the perturbed texel is bit-identical between the two
renders), and through torch.autograd."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from firefly_b200 import scenes

pytestmark = pytest.mark.gpu

W = H = 48
SET = dict(spp=8, max_depth=3, rr_depth=3, seed=3, light=-1)   # rr_depth = max_depth: no roulette


@pytest.fixture(scope="module")
def setup(ctx):
    import firefly_b200 as ff
    target = scenes.textured_room(seed=0, width=W, height=H, tex_res=32, env_w=32, env_h=16)
    start = scenes.textured_room(seed=0, width=W, height=H, tex_res=32, env_w=32, env_h=16,
                                 albedo=np.full((32, 32, 3), 0.5, np.float32))
    ds = ff.dScene(ctx, start)
    pt = ff.PathTracer(ctx, W, H)
    # reference image from the hidden parameters
    ds.set_texture(0, target.textures[0])
    pt.draw(ds, mode=ff.FF_MODE_CORRECTED, **SET)
    ref = pt.image().astype(np.float64)
    ds.set_texture(0, start.textures[0])
    yield ds, pt, start, target, ref
    pt.close()
    ds.close()


def loss_and_grad_image(pt, ds, ref, **kw):
    import firefly_b200 as ff
    pt.clear_buffer()
    pt.draw(ds, mode=ff.FF_MODE_CORRECTED, **{**SET, **kw})
    img = pt.image().astype(np.float64)
    diff = img - ref
    return 0.5 * float((diff * diff).sum()) / diff.size, (diff / diff.size).astype(np.float32)


def test_replay_matches_store_all(setup):
    ds, pt, start, target, ref = setup
    _, dimg = loss_and_grad_image(pt, ds, ref)
    g1, e1 = np.zeros_like(start.textures[0]), np.zeros_like(start.env_rgb)
    g2, e2 = np.zeros_like(start.textures[0]), np.zeros_like(start.env_rgb)
    st = ds.render_adjoint(W, H, dimg, grad_texture=g1, grad_env=e1, **SET)
    ds.render_adjoint(W, H, dimg, grad_texture=g2, grad_env=e2, store_all=True, **SET)
    assert st["samples"] == W * H * SET["spp"] and st["extension_rays"] > 0
    assert np.abs(g1).max() > 0 and np.abs(e1).max() > 0
    assert np.allclose(g1, g2, rtol=1e-4, atol=1e-7 * np.abs(g1).max())
    assert np.allclose(e1, e2, rtol=1e-4, atol=1e-5 * np.abs(e1).max())   # float-atomic order, as below


def test_wavefront_replay_matches_megakernel_replay(setup):
    """The default replay runs on the wavefront stages; the one-thread-per-
    sample megakernel replays the same paths (both compiled without FMA
    contraction, so path for path)."""
    ds, pt, start, target, ref = setup
    _, dimg = loss_and_grad_image(pt, ds, ref)
    g1, e1 = np.zeros_like(start.textures[0]), np.zeros_like(start.env_rgb)
    g2, e2 = np.zeros_like(start.textures[0]), np.zeros_like(start.env_rgb)
    s1 = ds.render_adjoint(W, H, dimg, grad_texture=g1, grad_env=e1, **SET)
    s2 = ds.render_adjoint(W, H, dimg, grad_texture=g2, grad_env=e2, megakernel=True, **SET)
    assert s1["shadow_rays"] > 0 and s1["frames"] > 0
    # the megakernel counts every traced ray in extension_rays
    assert s1["extension_rays"] + s1["shadow_rays"] == s2["extension_rays"]
    assert np.allclose(g1, g2, rtol=1e-4, atol=1e-7 * np.abs(g1).max())
    # the env texels sum many float atomics in no fixed order: the same call
    # repeated differs by up to about 1e-6 of the largest texel (measured
    # 5.8e-11 and 8.7e-11 at a largest texel of 2.5e-4), so the absolute
    # floor covers that and a relative bound does the rest
    assert np.allclose(e1, e2, rtol=1e-4, atol=1e-5 * np.abs(e1).max())


def test_wavefront_adjoint_takes_deep_paths(setup):
    """The wavefront replay keeps nothing per vertex, so any depth the
    renderer takes works; the megakernel variants stop at 15."""
    import firefly_b200 as ff
    ds, pt, start, target, ref = setup
    _, dimg = loss_and_grad_image(pt, ds, ref)
    g = np.zeros_like(start.textures[0])
    st = dict(SET, max_depth=24, rr_depth=3)
    ds.render_adjoint(W, H, dimg, grad_texture=g, **st)
    assert np.isfinite(g).all() and np.abs(g).max() > 0
    g2 = np.zeros_like(g)
    ds.render_adjoint(W, H, dimg, grad_texture=g2, **dict(st, max_depth=3))
    assert not np.allclose(g, g2), "deeper paths add gradient"
    with pytest.raises(ff.FireflyError):
        ds.render_adjoint(W, H, dimg, grad_texture=g, megakernel=True, **st)


def test_albedo_gradient_vs_central_differences(setup):
    ds, pt, start, target, ref = setup
    _, dimg = loss_and_grad_image(pt, ds, ref)
    g = np.zeros_like(start.textures[0])
    ds.render_adjoint(W, H, dimg, grad_texture=g, **SET)
    rng = np.random.default_rng(1)
    flat = np.abs(g).reshape(-1)
    # 64 texel channels among those the camera's paths reach
    cand = np.nonzero(flat > 1e-3 * flat.max())[0]
    picks = rng.choice(cand, size=min(64, len(cand)), replace=False)
    eps = 1e-3
    tex = start.textures[0].copy()
    fd = []
    for k in picks:
        t = tex.copy().reshape(-1)
        t[k] += eps
        ds.set_texture(0, t.reshape(tex.shape))
        lp, _ = loss_and_grad_image(pt, ds, ref)
        t[k] -= 2 * eps
        ds.set_texture(0, t.reshape(tex.shape))
        lm, _ = loss_and_grad_image(pt, ds, ref)
        fd.append((lp - lm) / (2 * eps))
    ds.set_texture(0, tex)
    fd = np.array(fd)
    ad = g.reshape(-1)[picks].astype(np.float64)
    rel = np.abs(ad - fd) / np.maximum(np.abs(fd), 1e-12)
    print(f"[adjoint] albedo FD: median rel err {np.median(rel):.2e}, max {rel.max():.2e}, n={len(picks)}")
    assert np.median(rel) < 1e-2
    assert np.mean(rel < 5e-2) > 0.9
    assert np.corrcoef(ad, fd)[0, 1] > 0.999


def test_env_gradient_vs_central_differences(setup):
    ds, pt, start, target, ref = setup
    _, dimg = loss_and_grad_image(pt, ds, ref)
    e = np.zeros_like(start.env_rgb)
    ds.render_adjoint(W, H, dimg, grad_env=e, texture=-1, **SET)
    flat = np.abs(e).reshape(-1)
    # 64 random texel channels among those the paths reach (the importance
    # tables are kept, so the image is linear in every texel)
    cand = np.nonzero(flat > 1e-3 * flat.max())[0]
    picks = np.random.default_rng(3).choice(cand, size=min(64, len(cand)), replace=False)
    assert len(picks) == 64
    env = start.env_rgb.copy()
    fd = []
    for k in picks:
        eps = 1e-3 * max(1.0, abs(env.reshape(-1)[k]))
        x = env.copy().reshape(-1)
        x[k] += eps
        ds.set_environment(x.reshape(env.shape), keep_tables=True)
        lp, _ = loss_and_grad_image(pt, ds, ref)
        x[k] -= 2 * eps
        ds.set_environment(x.reshape(env.shape), keep_tables=True)
        lm, _ = loss_and_grad_image(pt, ds, ref)
        fd.append((lp - lm) / (2 * eps))
    ds.set_environment(env, keep_tables=True)
    fd = np.array(fd)
    ad = e.reshape(-1)[picks].astype(np.float64)
    rel = np.abs(ad - fd) / np.maximum(np.abs(fd), 1e-12)
    print(f"[adjoint] env FD: median rel err {np.median(rel):.2e}, max {rel.max():.2e}, n={len(picks)}")
    assert np.median(rel) < 1e-2
    assert np.mean(rel < 5e-2) > 0.9
    assert np.corrcoef(ad, fd)[0, 1] > 0.999


def test_autograd_descent_reduces_loss(setup):
    from tests.ff_autograd import RenderFn
    ds, pt, start, target, ref = setup
    albedo = torch.from_numpy(start.textures[0].copy()).requires_grad_(True)
    env = torch.from_numpy(start.env_rgb.copy()).requires_grad_(True)
    opt = torch.optim.Adam([albedo], lr=2e-2)
    reft = torch.from_numpy(ref.astype(np.float32))
    losses = []
    for it in range(15):
        opt.zero_grad()
        img = RenderFn.apply(albedo, env, ds, pt, {**SET, "seed": 100 + it, "keep_tables": True})
        loss = 0.5 * ((img - reft) ** 2).mean()
        loss.backward()
        opt.step()
        with torch.no_grad():
            albedo.clamp_(0.01, 1.0)
        losses.append(float(loss))
    print(f"[adjoint] autograd loss {losses[0]:.4e} -> {losses[-1]:.4e}")
    assert losses[-1] < 0.7 * losses[0]
    ds.set_texture(0, start.textures[0])


def test_inverse_driver_on_device(ctx):
    """firefly_b200.inverse.optimize: device-resident parameters, native Adam
    steps; under known lighting the albedo moves to the hidden one and the
    held-out image error falls to the floor that the noise sets.  (The
    training loss is no measure here: it holds the 8-spp image's variance,
    which grows with the albedo.)"""
    import firefly_b200 as ff
    from firefly_b200 import inverse
    # a soft sky (no hard sun): low variance, so 40 noisy steps can show the fit
    sky = scenes.sky_env(32, 16, seed=0, sun_radiance=8.0, sun_diameter_deg=20.0)
    hidden = scenes.textured_room(seed=0, width=40, height=40, tex_res=32, env=sky)
    start = scenes.textured_room(seed=0, width=40, height=40, env=sky,
                                 albedo=np.full((32, 32, 3), 0.2, np.float32))
    ds = ff.dScene(ctx, hidden)
    pt = ff.PathTracer(ctx, 40, 40)
    pt.draw(ds, spp=64, max_depth=3, seed=77, light=-1, mode=ff.FF_MODE_CORRECTED)
    target = torch.from_numpy(pt.image().astype(np.float32)).cuda()
    albedo = torch.from_numpy(start.textures[0].copy()).cuda()
    env = torch.from_numpy(hidden.env_rgb.copy()).cuda()      # known lighting: recover the albedo alone
    r = inverse.optimize(ds, pt, target, albedo, env, steps=40, spp=8, lr=2e-2, lr_env=0.0, lr_decay=0.1)
    assert len(r["losses"]) == 40 and np.all(np.isfinite(r["losses"]))
    assert r["adjoint_spp_per_s"] > 0
    rmse = lambda a: float(np.sqrt(((a - hidden.textures[0]) ** 2).mean()))
    r0, r1 = rmse(start.textures[0]), rmse(albedo.cpu().numpy())

    def heldout(tex):
        # fresh seed, more samples: the image error, not the noisy training loss
        ds.set_texture(0, tex)
        pt.clear_buffer()
        pt.draw(ds, spp=64, max_depth=3, seed=991, light=-1, mode=ff.FF_MODE_CORRECTED)
        return float(((pt.image() - target.cpu().numpy()) ** 2).mean())
    e0, e1, ef = heldout(start.textures[0]), heldout(albedo.cpu().numpy()), heldout(hidden.textures[0])
    print(f"[adjoint] driver albedo rmse {r0:.4f} -> {r1:.4f}; held-out image error {e0:.4e} -> {e1:.4e} "
          f"(hidden albedo {ef:.4e}); {r['adjoint_spp_per_s']:.3e} spp/s")
    assert r1 < 0.5 * r0
    assert e1 - ef < 0.25 * (e0 - ef)
    pt.close()
    ds.close()


# ----------------------------------------------------------------- roughness
# The sphere carries a GGX material whose roughness reads texture 1 (channel
# 0, Perlin in [0.1, 0.6]); the walls keep the albedo texture.  Lights: the
# environment (light -1) and one directional light (light 0).

RW = RH = 48
DIR_LIGHT = 0


@pytest.fixture(scope="module", params=["MIX", "CONDUCTOR", "DIELECTRIC", "COAT"])
def rough_setup(ctx, request):
    import firefly_b200 as ff
    kind = getattr(ff, f"FF_MAT_{request.param}")
    # a soft sky (no small bright sun): glossy reflections of a hard sun would
    # make the finite differences of the full-depth test too noisy to compare
    sky = scenes.sky_env(32, 16, seed=0, sun_radiance=8.0, sun_diameter_deg=20.0)
    scn = scenes.textured_room(seed=0, width=RW, height=RH, tex_res=32, env=sky, sphere_kind=kind,
                               sphere_metallic=1.0 if request.param == "CONDUCTOR" else 0.3)
    scn.directional_lights = [scenes.directional_light((0.3, 1.0, 0.2), (1.0, 0.95, 0.8), 2.5)]
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, RW, RH)
    yield request.param, ds, pt, scn
    pt.close()
    ds.close()


def _linear_weights(seed=11):
    # a fixed dL/dI: the loss sum(w * I) is linear in the image, so the FD of
    # one seed's image and the adjoint of the same seed estimate the same
    # derivative of E[loss]
    return np.random.default_rng(seed).uniform(0.0, 1.0, (RH, RW, 3)).astype(np.float32) / (RW * RH)


def _render_loss(pt, ds, w, **kw):
    import firefly_b200 as ff
    pt.clear_buffer()
    pt.draw(ds, mode=ff.FF_MODE_CORRECTED, **kw)
    return float((pt.image().astype(np.float64) * w).sum())


@pytest.mark.parametrize("light", [-1, DIR_LIGHT])
def test_roughness_replay_matches_store_all(rough_setup, light):
    kind, ds, pt, scn = rough_setup
    w = _linear_weights()
    g1, g2 = np.zeros_like(scn.textures[1]), np.zeros_like(scn.textures[1])
    st = dict(SET, light=light)
    s1 = ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=g1, **st)
    ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=g2, store_all=True, **st)
    assert s1["grad_atomics_roughness"] > 0 and s1["grad_atomics"] == 0
    assert np.isfinite(g1).all()
    assert np.abs(g1[..., 0]).max() > 0
    assert not g1[..., 1:].any(), "only channel 0 carries the roughness"
    assert np.allclose(g1, g2, rtol=1e-4, atol=1e-6 * np.abs(g1).max()), kind


@pytest.mark.parametrize("light", [-1, DIR_LIGHT])
def test_roughness_gradient_nee_vs_central_differences(rough_setup, light):
    """Depth 1 (camera vertex + NEE): the light-sampled directions do not
    depend on the roughness, so common random numbers make the central
    difference of one seed's render the derivative the adjoint computes.
    The mixed material and the dielectric under the environment also add a
    BSDF-sampled light term whose direction moves with r (and MIS weights
    that depend on r); under the directional light (a delta light: no
    BSDF-sampled term, weight 1) they are checked like the others."""
    kind, ds, pt, scn = rough_setup
    if kind in ("MIX", "DIELECTRIC") and light == -1:
        pytest.skip("the BSDF-sampled light term's direction moves with r (checked in expectation below)")
    st = dict(SET, max_depth=1, spp=4, light=light)
    w = _linear_weights()
    g = np.zeros_like(scn.textures[1])
    ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=g, **st)
    flat = np.abs(g[..., 0]).reshape(-1)
    assert np.isfinite(flat).all() and flat.max() > 0
    cand = np.nonzero(flat > 1e-3 * flat.max())[0]
    picks = np.random.default_rng(2).choice(cand, size=min(64, len(cand)), replace=False)
    eps = 1e-3
    rough = scn.textures[1].copy()
    fd = []
    for k in picks:
        t = rough.copy()
        t.reshape(-1, 3)[k, 0] += eps
        ds.set_texture(1, t)
        lp = _render_loss(pt, ds, w, **st)
        t.reshape(-1, 3)[k, 0] -= 2 * eps
        ds.set_texture(1, t)
        lm = _render_loss(pt, ds, w, **st)
        fd.append((lp - lm) / (2 * eps))
    ds.set_texture(1, rough)
    fd = np.array(fd)
    ad = g[..., 0].reshape(-1)[picks].astype(np.float64)
    rel = np.abs(ad - fd) / np.maximum(np.abs(fd), 1e-12)
    print(f"[adjoint] roughness ({kind}, light {light}) NEE FD: median rel err {np.median(rel):.2e}, "
          f"max {rel.max():.2e}, n={len(picks)}")
    assert np.median(rel) < 1e-2
    assert np.corrcoef(ad, fd)[0, 1] > 0.999


@pytest.mark.parametrize("light", [-1, DIR_LIGHT])
def test_roughness_gradient_full_depth_in_expectation(rough_setup, light):
    """Depth 3: a BSDF-sampled direction moves with the roughness, so one
    seed's central difference (directions re-sampled) and the detached
    adjoint (directions held) differ sample by sample but estimate the same
    derivative of the expected loss.  Directional derivative along the sign
    of a pilot adjoint gradient (an independent seed, so the direction does
    not correlate with the noise of the compared runs), 256 spp per seed,
    16 seeds under the directional light and 64 under the environment (its
    glossy reflections of the sun are noisier); the means must agree within
    4 standard errors, and the standard error must be small against the
    derivative."""
    kind, ds, pt, scn = rough_setup
    w = _linear_weights()
    rough = scn.textures[1].copy()
    pilot = np.zeros_like(rough)
    ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=pilot,
                      **dict(SET, spp=2048, seed=77, light=light))
    delta = np.zeros_like(rough)
    delta[..., 0] = np.sign(pilot[..., 0])
    assert np.abs(delta).sum() > 0
    eps = 1e-2
    ad, fd = [], []
    for s in range(16 if light == DIR_LIGHT else 64):
        st = dict(SET, spp=256, seed=1000 + s, light=light)
        g = np.zeros_like(rough)
        ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=g, **st)
        ad.append(float((g.astype(np.float64) * delta).sum()))
        ds.set_texture(1, rough + eps * delta)
        lp = _render_loss(pt, ds, w, **st)
        ds.set_texture(1, rough - eps * delta)
        lm = _render_loss(pt, ds, w, **st)
        ds.set_texture(1, rough)
        fd.append((lp - lm) / (2 * eps))
    ad, fd = np.array(ad), np.array(fd)
    se = np.sqrt(ad.var(ddof=1) / len(ad) + fd.var(ddof=1) / len(fd))
    print(f"[adjoint] roughness ({kind}, light {light}) full depth: adjoint {ad.mean():.4e} "
          f"+- {ad.std(ddof=1):.1e}, FD {fd.mean():.4e} +- {fd.std(ddof=1):.1e} (per seed), "
          f"z = {(ad.mean() - fd.mean()) / se:.2f}")
    assert abs(ad.mean() - fd.mean()) < 4 * se + 0.02 * abs(fd.mean())
    # under the environment the coat's roughness derivative is small against
    # the noise of its re-sampled finite differences (se ~ 0.25 of the mean)
    assert se < (0.1 if light == DIR_LIGHT else 0.35) * abs(ad.mean()), "too noisy to tell"


def test_autograd_roughness_descent(ctx):
    """torch.autograd over the roughness texture of a conductor sphere lit by
    a directional light (the roughness sets the size of its highlight): Adam
    on a one-texel roughness texture (every hit on the sphere reads it) from
    0.5 moves it to the hidden 0.2 and lowers the image error measured with a
    held-out seed.  (Under an environment light alone, a smooth conductor's
    highlight reaches the image only through light-sampled NEE, whose
    roughness derivative is heavy-tailed: Adam, which follows the typical
    sample, drifts there.)"""
    import firefly_b200 as ff
    from tests.ff_autograd import RenderFn
    res = 64
    sky = scenes.sky_env(32, 16, seed=0, sun_radiance=8.0, sun_diameter_deg=20.0)
    r_hidden, r_start = 0.2, 0.5
    hidden = scenes.textured_room(seed=0, width=res, height=res, tex_res=32, env=sky, sphere_kind=ff.FF_MAT_CONDUCTOR,
                                  roughness=np.full((1, 1, 3), r_hidden, np.float32))
    hidden.directional_lights = [scenes.directional_light((0.3, 1.0, 0.2), (1.0, 0.95, 0.8), 2.5)]
    ds = ff.dScene(ctx, hidden)
    pt = ff.PathTracer(ctx, res, res)
    st = dict(SET, spp=16, light=DIR_LIGHT)
    pt.draw(ds, mode=ff.FF_MODE_CORRECTED, **dict(st, spp=1024, seed=4242))
    target = torch.from_numpy(pt.image().astype(np.float32))

    def heldout(r):
        ds.set_texture(1, r)
        pt.clear_buffer()
        pt.draw(ds, mode=ff.FF_MODE_CORRECTED, **dict(st, spp=256, seed=777))
        return float(((torch.from_numpy(pt.image()) - target) ** 2).mean())

    start = np.full((1, 1, 3), r_start, np.float32)
    floor, e0 = heldout(np.full((1, 1, 3), r_hidden, np.float32)), heldout(start)
    albedo = torch.from_numpy(hidden.textures[0].copy())
    env = torch.from_numpy(hidden.env_rgb.copy())
    rough = torch.from_numpy(start.copy()).requires_grad_(True)
    opt = torch.optim.Adam([rough], lr=3e-2)
    for it in range(40):
        opt.zero_grad()
        img = RenderFn.apply(albedo, env, ds, pt, {**st, "seed": 100 + it, "keep_tables": True, "decorrelate": True},
                             rough)
        loss = 0.5 * ((img - target) ** 2).mean()
        loss.backward()
        assert rough.grad is not None and torch.isfinite(rough.grad).all()
        opt.step()
        with torch.no_grad():
            rough.clamp_(0.02, 1.0)
    r_end = float(rough.detach()[..., 0].mean())
    e1 = heldout(rough.detach().numpy())
    print(f"[adjoint] autograd roughness {r_start} -> {r_end:.3f} (hidden {r_hidden}); held-out error "
          f"{e0:.4e} -> {e1:.4e} (hidden roughness {floor:.4e})")
    assert abs(r_end - r_hidden) < 0.2 * abs(r_start - r_hidden)
    assert e1 - floor < 0.3 * (e0 - floor)
    pt.close()
    ds.close()


def test_roughness_texture_index_is_checked(rough_setup):
    import firefly_b200 as ff
    kind, ds, pt, scn = rough_setup
    g = np.zeros_like(scn.textures[1])
    with pytest.raises(ff.FireflyError):
        ds.render_adjoint(RW, RH, _linear_weights(), texture=-1, roughness_texture=7, grad_roughness=g, **SET)


@pytest.mark.parametrize("kind_name", ["MIX", "CONDUCTOR"])
def test_roughness_gradient_packed_metallic_roughness(ctx, kind_name):
    """A glTF-style material reads its roughness from channel y of the packed
    metallic-roughness texture: the gradient lands in channel y only (x is
    unused, z is the metallic), the wavefront replay agrees with the
    store-all and megakernel variants, and at depth 1 under the directional
    light it matches central differences of channel y."""
    import firefly_b200 as ff
    kind = getattr(ff, f"FF_MAT_{kind_name}")
    sky = scenes.sky_env(32, 16, seed=0, sun_radiance=8.0, sun_diameter_deg=20.0)
    scn = scenes.textured_room(seed=0, width=RW, height=RH, tex_res=32, env=sky, sphere_kind=kind, packed=True,
                               sphere_metallic=1.0 if kind_name == "CONDUCTOR" else 0.3)
    scn.directional_lights = [scenes.directional_light((0.3, 1.0, 0.2), (1.0, 0.95, 0.8), 2.5)]
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, RW, RH)
    try:
        w = _linear_weights()
        gs = [np.zeros_like(scn.textures[1]) for _ in range(3)]
        s1 = ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=gs[0], **SET)
        ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=gs[1], store_all=True, **SET)
        ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=gs[2], megakernel=True, **SET)
        assert s1["grad_atomics_roughness"] > 0
        for g in gs:
            assert np.isfinite(g).all()
            assert np.abs(g[..., 1]).max() > 0
            assert not g[..., 0].any() and not g[..., 2].any(), "only channel y carries the roughness"
        tol = 1e-6 * np.abs(gs[0]).max()
        assert np.allclose(gs[0], gs[1], rtol=1e-4, atol=tol), kind_name
        assert np.allclose(gs[0], gs[2], rtol=1e-4, atol=tol), kind_name

        st = dict(SET, max_depth=1, spp=4, light=DIR_LIGHT)
        g = np.zeros_like(scn.textures[1])
        ds.render_adjoint(RW, RH, w, texture=-1, roughness_texture=1, grad_roughness=g, **st)
        flat = np.abs(g[..., 1]).reshape(-1)
        cand = np.nonzero(flat > 1e-3 * flat.max())[0]
        picks = np.random.default_rng(2).choice(cand, size=min(32, len(cand)), replace=False)
        eps = 1e-3
        base = scn.textures[1].copy()
        fd = []
        for k in picks:
            t = base.copy()
            t.reshape(-1, 3)[k, 1] += eps
            ds.set_texture(1, t)
            lp = _render_loss(pt, ds, w, **st)
            t.reshape(-1, 3)[k, 1] -= 2 * eps
            ds.set_texture(1, t)
            lm = _render_loss(pt, ds, w, **st)
            fd.append((lp - lm) / (2 * eps))
        ds.set_texture(1, base)
        fd = np.array(fd)
        ad = g[..., 1].reshape(-1)[picks].astype(np.float64)
        rel = np.abs(ad - fd) / np.maximum(np.abs(fd), 1e-12)
        print(f"[adjoint] packed roughness ({kind_name}) NEE FD: median rel err {np.median(rel):.2e}, n={len(picks)}")
        assert np.median(rel) < 1e-2
        assert np.corrcoef(ad, fd)[0, 1] > 0.999
    finally:
        pt.close()
        ds.close()
