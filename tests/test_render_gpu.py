"""Image parity of ff_render against the oracle's restatement of the
reference's wavefront stages, with the same per-pixel sampler seeds.

Tolerance: mean relative error <= 1e-4 (the bar for floating-point parity), measured as
    mre = sum |gpu - oracle| / sum |oracle|
over all pixels and channels of the per-pixel mean radiance.  Both sides
follow the reference's arithmetic operation by operation; what remains are
last-bit differences of the device and host sinf/cosf/atan2f/asinf/acosf/atanf
and FP64 sin/cos, which occasionally send a path across a triangle edge.
"""
from __future__ import annotations

import numpy as np
import pytest

from firefly_b200 import scenes
from tests.conftest import cpu_threads

pytestmark = pytest.mark.gpu

MRE_TOL = 1e-4


def _gpu_render(ctx, scn, w, h, spp, **kw):
    import firefly_b200 as ff
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, w, h)
    stats = pt.draw(ds, spp=spp, **kw)
    rgba, n = pt.read()
    pt.close()
    ds.close()
    return rgba[..., :3].astype(np.float64), n, stats


def _mre(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-30))


def _parity(ctx, oracle, scn, w, h, spp, light=0, max_depth=5, rr_depth=3, seed=0, mode=0, **kw):
    got, n, stats = _gpu_render(ctx, scn, w, h, spp, light=light, max_depth=max_depth, rr_depth=rr_depth,
                                seed=seed, mode=mode, **kw)
    ref, (ref_ext, ref_sh) = oracle.render(scn, w, h, spp, max_depth=max_depth, rr_depth=rr_depth, seed=seed,
                                           mode=mode, light=light, threads=cpu_threads())
    assert np.all(n == spp)
    mre = _mre(got / spp, ref / spp)
    print(f"[parity] {w}x{h} spp={spp} depth={max_depth} mode={mode}: mre={mre:.3e} "
          f"ext={stats['extension_rays']}/{ref_ext} shadow={stats['shadow_rays']}/{ref_sh} "
          f"gpu_ms={stats['ms_total']:.2f} frames={stats['frames']}")
    assert mre <= MRE_TOL, f"mean relative error {mre:.3e} > {MRE_TOL}"
    # the same paths were traced
    assert abs(stats["extension_rays"] - ref_ext) <= max(2, 1e-3 * ref_ext), (stats["extension_rays"], ref_ext)
    assert abs(stats["shadow_rays"] - ref_sh) <= max(2, 1e-3 * ref_sh), (stats["shadow_rays"], ref_sh)
    return got, ref, stats, mre


def test_small_room_parity_64(ctx, oracle):
    scn = scenes.small_room(seed=0, width=64, height=64)
    got, ref, stats, mre = _parity(ctx, oracle, scn, 64, 64, 4)
    assert (ref.sum(-1) > 0).mean() > 0.8   # the light reaches most pixels


def test_small_room_parity_full_config(ctx, oracle):
    """The plain-tracer workload itself: 256 x 256, 16 spp, depth 5, RR from depth 3, seed 0."""
    scn = scenes.small_room(seed=0)
    _parity(ctx, oracle, scn, 256, 256, 16)


def test_parity_with_lens_and_depth3(ctx, oracle):
    scn = scenes.small_room(seed=1, width=48, height=40, lens_radius=0.05)
    _parity(ctx, oracle, scn, 48, 40, 3, max_depth=3, rr_depth=2, seed=7)


def test_parity_single_lobe_materials(ctx, oracle):
    import firefly_b200 as ff
    for kind in (ff.FF_MAT_DIFFUSE, ff.FF_MAT_CONDUCTOR):
        scn = scenes.small_room(seed=2, width=40, height=40, kind=kind)
        for m in scn.materials:
            m.roughness = 0.4
        # parity: the reference's diff_L / spec_L return 0, so only corrected mode carries light
        _parity(ctx, oracle, scn, 40, 40, 2, mode=ff.FF_MODE_CORRECTED)


def test_corrected_mode_parity(ctx, oracle):
    import firefly_b200 as ff
    scn = scenes.small_room(seed=3, width=48, height=48)
    _parity(ctx, oracle, scn, 48, 48, 4, mode=ff.FF_MODE_CORRECTED)


def test_progressive_and_pool_size_invariance(ctx):
    import firefly_b200 as ff
    scn = scenes.small_room(seed=0, width=64, height=48)
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, 64, 48)
    pt.draw(ds, spp=8, max_depth=5, seed=5, light=0)
    one, n1 = pt.read()
    pt.clear_buffer()
    z, nz = pt.read()
    assert np.all(nz == 0) and np.all(z == 0)
    # two progressive calls, small pool (one slot per pixel)
    pt.draw(ds, spp=3, max_depth=5, seed=5, sample_offset=0, max_paths=64 * 48, light=0)
    pt.draw(ds, spp=5, max_depth=5, seed=5, sample_offset=3, max_paths=64 * 48, light=0)
    two, n2 = pt.read()
    assert np.array_equal(n1, n2)
    assert np.allclose(one, two, rtol=1e-5, atol=1e-6)
    # determinism
    pt.clear_buffer()
    pt.draw(ds, spp=8, max_depth=5, seed=5, light=0)
    again, _ = pt.read()
    assert np.array_equal(one, again)
    img8 = pt.tonemap(1.0)
    assert img8.shape == (48, 64, 4) and img8[..., 3].min() == 255
    pt.close()
    ds.close()


def test_stream_concurrency_is_invisible(ctx):
    """ff_render runs the any-hit trace beside the closest-hit trace and the
    material kinds' shade launches side by side; under stage timing
    (profile) everything runs on one stream.  Both schedules give the same
    image bit for bit (hits by slot, shadow answers by tag, disjoint slots)."""
    import firefly_b200 as ff
    sky = scenes.sky_env(64, 32, seed=0, sun_radiance=50.0, sun_diameter_deg=4.0)
    scn = scenes.textured_room(seed=1, width=96, height=72, tex_res=32, env=sky, sphere_kind=ff.FF_MAT_CONDUCTOR)
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, 96, 72)
    out = []
    for profile in (False, True, False):
        pt.clear_buffer()
        st = pt.draw(ds, spp=8, max_depth=6, rr_depth=3, seed=7, light=-1, mode=ff.FF_MODE_CORRECTED,
                     profile=profile)
        out.append((pt.read(), st["extension_rays"], st["shadow_rays"]))
    (a, na), ea, sa = out[0]
    for (b, nb), eb, sb in out[1:]:
        assert np.array_equal(na, nb) and ea == eb and sa == sb
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert a[..., :3].sum() > 0
    pt.close()
    ds.close()


def test_render_argument_errors(ctx):
    import firefly_b200 as ff
    scn = scenes.small_room(seed=0, width=16, height=16)
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, 16, 16)
    with pytest.raises(ff.FireflyError):
        pt.draw(ds, spp=1, light=-1)     # no environment map in this scene
    with pytest.raises(ff.FireflyError):
        pt.draw(ds, spp=1, light=3)      # no such area light
    with pytest.raises(ff.FireflyError):
        pt.draw(ds, spp=0, light=0)
    pt.close()
    ds.close()


def test_textured_env_scene_parity(ctx, oracle):
    """Albedo texture (bilinear, wrap, 8-bit weights as the reference's texture
    units filter) on room and sphere, lit by the environment map."""
    import firefly_b200 as ff
    scn = scenes.textured_room(seed=4, width=48, height=48, tex_res=64, env_w=64, env_h=32)
    for mode in (ff.FF_MODE_PARITY, ff.FF_MODE_CORRECTED):
        got, n, stats = _gpu_render(ctx, scn, 48, 48, 4, light=-1, max_depth=4, rr_depth=3, seed=9, mode=mode)
        ref, _ = oracle.render(scn, 48, 48, 4, max_depth=4, rr_depth=3, seed=9, mode=mode, light=-1,
                               threads=cpu_threads())
        fin = np.isfinite(got) & np.isfinite(ref)
        assert np.array_equal(np.isfinite(got), np.isfinite(ref))
        mre = _mre(got[fin], ref[fin])
        print(f"[parity] textured env mode={mode}: mre={mre:.3e}")
        assert mre <= MRE_TOL


def test_material_textures_and_normal_map_parity(ctx, oracle):
    """Every material texture kind against the oracle, in both modes: a
    base-colour texture, a packed metallic-roughness texture (roughness y,
    metallic z) and a normal texture on the walls (mixed material); roughness
    and metallic textures and the normal texture on a conductor sphere.  The
    tangent frame comes per vertex with the scene (dMaterial.cu:10-88)."""
    import firefly_b200 as ff
    scn = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=64)
    for mode in (ff.FF_MODE_PARITY, ff.FF_MODE_CORRECTED):
        got, n, stats = _gpu_render(ctx, scn, 48, 48, 4, light=-1, max_depth=4, rr_depth=3, seed=5, mode=mode)
        ref, (ref_ext, ref_sh) = oracle.render(scn, 48, 48, 4, max_depth=4, rr_depth=3, seed=5, mode=mode, light=-1,
                                               threads=cpu_threads())
        fin = np.isfinite(got) & np.isfinite(ref)
        assert np.array_equal(np.isfinite(got), np.isfinite(ref))
        mre = _mre(got[fin], ref[fin])
        print(f"[parity] material textures + normal map mode={mode}: mre={mre:.3e} "
              f"ext={stats['extension_rays']}/{ref_ext} shadow={stats['shadow_rays']}/{ref_sh}")
        assert mre <= MRE_TOL
        assert abs(stats["extension_rays"] - ref_ext) <= max(2, 1e-3 * ref_ext)


def test_normal_map_and_packed_textures_change_the_image(ctx):
    """The normal texture, the packed metallic-roughness texture and derived
    tangents (no per-vertex frame given) all reach the image."""
    import firefly_b200 as ff
    scn = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=64)
    kw = dict(light=-1, max_depth=4, rr_depth=3, seed=5, mode=ff.FF_MODE_CORRECTED)
    img, _, _ = _gpu_render(ctx, scn, 48, 48, 16, **kw)
    flat = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=64)
    for m in flat.materials:
        m.normal_tex = -1
    img_flat, _, _ = _gpu_render(ctx, flat, 48, 48, 16, **kw)
    packed = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=64)
    packed.materials[0].metallic_roughness_tex = -1
    img_factors, _, _ = _gpu_render(ctx, packed, 48, 48, 16, **kw)
    derived = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=64, derive_tangents=True)
    img_derived, _, _ = _gpu_render(ctx, derived, 48, 48, 16, **kw)
    for a in (img, img_flat, img_factors, img_derived):
        assert np.isfinite(a).all() and a.mean() > 0
    assert _mre(img, img_flat) > 1e-2, "the normal texture changes the shading"
    assert _mre(img, img_factors) > 1e-2, "the packed texture replaces the factors"
    # derived frames differ from the given ones only by the orientation within the tangent plane
    assert _mre(img_derived, img) < 0.5


def test_gltf_textured_round_trip_renders_the_same(ctx, tmp_path):
    """A scene with base-colour, metallic-roughness and normal textures and a
    tangent frame, written to .glb and read back, renders the same image."""
    import firefly_b200 as ff
    from firefly_b200 import gltf
    scn = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=32)
    scn.textures = [(np.round(np.clip(t, 0.0, 1.0) * 255.0) / 255.0).astype(np.float32) for t in scn.textures]
    for m in scn.materials:
        m.roughness_tex = -1
        m.metallic_tex = -1
    gltf.save(tmp_path / "pbr.glb", scn)
    got = gltf.load(tmp_path / "pbr.glb", 48, 48)
    for a, b in zip(scn.materials, got.materials):
        b.kind = a.kind
    got.env_rgb, got.camera = scn.env_rgb, scn.camera
    kw = dict(light=-1, max_depth=4, rr_depth=3, seed=5, mode=ff.FF_MODE_CORRECTED)
    a, _, _ = _gpu_render(ctx, scn, 48, 48, 8, **kw)
    b, _, _ = _gpu_render(ctx, got, 48, 48, 8, **kw)
    mre = _mre(b, a)
    print(f"[gltf] textured round trip: mre={mre:.3e}")
    assert mre < 1e-4


def test_directional_light_and_light_selection_parity(ctx, oracle):
    """dDirectionalLight (delta: MIS weights 1, no BSDF-sampled visibility
    rays) as light 0 of the room open to the sky, in both modes; and
    FF_LIGHT_ALL (one of env + area + directional chosen per vertex, scaled
    by the light count) in corrected mode."""
    import firefly_b200 as ff
    scn = scenes.textured_room(seed=5, width=40, height=40, tex_res=32, env_w=64, env_h=32, kind=ff.FF_MAT_MIX)
    scn.directional_lights = [scenes.directional_light((0.3, 1.0, 0.2), (1.0, 0.95, 0.8), 2.5)]
    scn.area_lights = [scenes.area_light((-1.0, 9.0, -1.0), (2.0, 0.0, 0.0), (0.0, 0.0, 2.0), (0.0, -1.0, 0.0),
                                        radiance=8.0)]
    for light, mode in ((1, ff.FF_MODE_PARITY), (1, ff.FF_MODE_CORRECTED), (ff.FF_LIGHT_ALL, ff.FF_MODE_CORRECTED)):
        got, n, stats = _gpu_render(ctx, scn, 40, 40, 4, light=light, max_depth=4, rr_depth=3, seed=13, mode=mode)
        ref, (re, rs) = oracle.render(scn, 40, 40, 4, max_depth=4, rr_depth=3, seed=13, mode=mode, light=light,
                                      threads=cpu_threads())
        fin = np.isfinite(got) & np.isfinite(ref)
        assert np.array_equal(np.isfinite(got), np.isfinite(ref))
        mre = _mre(got[fin], ref[fin])
        print(f"[parity] light={light} mode={mode}: mre={mre:.3e} ext={stats['extension_rays']}/{re} "
              f"shadow={stats['shadow_rays']}/{rs} mean={ref[fin].mean():.4f}")
        assert ref[fin].mean() > 0
        assert mre <= MRE_TOL
        assert abs(stats["shadow_rays"] - rs) <= max(2, 1e-3 * rs)
    import firefly_b200 as ff2
    ds = ff2.dScene(ctx, scn)
    pt = ff2.PathTracer(ctx, 8, 8)
    with pytest.raises(ff2.FireflyError):
        pt.draw(ds, spp=1, light=ff2.FF_LIGHT_ALL, mode=ff2.FF_MODE_PARITY)   # selection needs the corrected mode
    with pytest.raises(ff2.FireflyError):
        pt.draw(ds, spp=1, light=2)                                           # 1 area + 1 directional light
    pt.close()
    ds.close()


def test_gltf_round_trip_renders_the_same(ctx, tmp_path):
    """A scene written to .glb and imported again (triangles regrouped by
    material, so the BVH differs) renders the same image with the same seeds."""
    import firefly_b200 as ff
    from firefly_b200 import gltf
    scn = scenes.small_room(seed=1, width=48, height=48)
    p = tmp_path / "room.glb"
    gltf.save(p, scn)
    imp = gltf.load(p, 48, 48)
    imp.camera, imp.area_lights = scn.camera, scn.area_lights
    a, _, _ = _gpu_render(ctx, scn, 48, 48, 4, light=0, max_depth=5, rr_depth=3, seed=3, mode=ff.FF_MODE_CORRECTED)
    b, _, _ = _gpu_render(ctx, imp, 48, 48, 4, light=0, max_depth=5, rr_depth=3, seed=3, mode=ff.FF_MODE_CORRECTED)
    mre = _mre(b, a)
    print(f"[gltf] round-trip render mre={mre:.3e}")
    assert mre < 1e-4


def test_render_edge_cases(ctx, oracle):
    """One-pixel film, depth 1 (camera hits only), an empty scene lit by the
    environment, and a film larger than the path pool (max_paths)."""
    import firefly_b200 as ff
    scn = scenes.small_room(seed=2, width=16, height=16)
    _parity(ctx, oracle, scn, 1, 1, 8, max_depth=5)
    _parity(ctx, oracle, scn, 16, 16, 2, max_depth=1)
    sky = scenes.sphere_under_sky(seed=3, width=16, height=16, env_w=64, env_h=32)
    empty = scenes.Scene(positions=np.zeros((0, 3), np.float32), indices=np.zeros((0, 3), np.uint32),
                         normals=np.zeros((0, 3), np.float32), env_rgb=sky.env_rgb, camera=sky.camera)
    got, n, _ = _gpu_render(ctx, empty, 16, 16, 2, light=-1, mode=ff.FF_MODE_CORRECTED)
    assert np.all(n == 2) and np.all(np.isfinite(got)) and got.min() > 0      # every camera ray sees the sky
    got_small_pool, n2, st = _gpu_render(ctx, scn, 16, 16, 3, light=0, max_depth=5, rr_depth=3, seed=4,
                                         mode=ff.FF_MODE_CORRECTED, max_paths=100)
    ref, _ = oracle.render(scn, 16, 16, 3, max_depth=5, rr_depth=3, seed=4, mode=1, light=0, threads=cpu_threads())
    assert np.all(n2 == 3)
    assert _mre(got_small_pool / 3, ref / 3) <= MRE_TOL


def tonemap_restated(rgba: np.ndarray, n: np.ndarray, exposure: float) -> np.ndarray:
    """wf_logic's display write (CUDA-RayTracer/kernel.cu:446-454) in float32:
    final_col = accum / (float)n, *= exposure, /= (final_col + 1), then
    (int)255 * c per channel and alpha 255; pixels without samples stay
    black.  The reference stores into a signed char4 (values above 127
    wrap); the headless film saturates to 0..255 instead."""
    f32 = np.float32
    acc = rgba[..., :3].astype(f32)
    nn = n.astype(f32)[..., None]
    col = (acc / np.where(nn >= 1, nn, f32(1))).astype(f32)
    col = (col * f32(exposure)).astype(f32)
    col = (col / (col + f32(1))).astype(f32)
    byte = np.clip(np.trunc((f32(255) * col).astype(f32)), 0, 255).astype(np.uint8)
    out = np.zeros(rgba.shape[:2] + (4,), np.uint8)
    out[..., :3] = np.where(n[..., None] >= 1, byte, 0)
    out[..., 3] = 255
    return out


def test_tonemap_matches_the_reference_display_formula(ctx):
    """ff_film_tonemap byte for byte against the restated kernel.cu:446-454,
    on dark and bright pixels (exposure 16 pushes many channels past the 0.5
    point of x / (1 + x), where the reference's signed char4 would wrap) and
    on an empty film."""
    import firefly_b200 as ff
    w, h = 64, 48
    scn = scenes.small_room(seed=1, width=w, height=h)
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, w, h)
    try:
        pt.draw(ds, spp=6, max_depth=5, seed=11, light=0)
        for exposure in (1.0, 16.0, 0.25):
            rgba, n = pt.read()
            got = pt.tonemap(exposure)
            want = tonemap_restated(rgba, n, exposure)
            assert np.array_equal(got, want), (exposure, int((got != want).sum()))
            if exposure > 8.0:
                assert (got[..., :3] > 128).mean() > 0.1
        # an empty film maps to opaque black
        pt.clear_buffer()
        got = pt.tonemap(1.0)
        assert np.all(got[..., :3] == 0) and np.all(got[..., 3] == 255)
    finally:
        pt.close()
        ds.close()


def test_committed_gltf_renders_like_the_oracle(ctx, oracle):
    """The committed .glb fixture (tests/golden/room_pbr.glb: base-colour,
    metallic-roughness and normal textures with known texels, a tangent
    frame) imported through firefly_b200.gltf and rendered on the GPU agrees
    with the oracle rendering the same imported scene: MRE <= 1e-4 and the
    same ray counts, in both modes."""
    import firefly_b200 as ff
    from firefly_b200 import gltf
    from tests.conftest import ROOT
    scn = gltf.load(ROOT / "tests" / "golden" / "room_pbr.glb", 48, 48)
    scn.env_rgb = scenes.sky_env(64, 32, seed=2, sun_radiance=20.0, sun_diameter_deg=8.0)
    # the camera of the scene the fixture was made from
    scn.camera = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=16).camera
    for mode in (ff.FF_MODE_PARITY, ff.FF_MODE_CORRECTED):
        got, n, stats = _gpu_render(ctx, scn, 48, 48, 4, light=-1, max_depth=4, rr_depth=3, seed=21, mode=mode)
        ref, (re, rs) = oracle.render(scn, 48, 48, 4, max_depth=4, rr_depth=3, seed=21, mode=mode, light=-1,
                                      threads=cpu_threads())
        fin = np.isfinite(got) & np.isfinite(ref)
        assert np.array_equal(np.isfinite(got), np.isfinite(ref))
        mre = _mre(got[fin], ref[fin])
        print(f"[gltf] fixture mode={mode}: mre={mre:.3e} ext={stats['extension_rays']}/{re} "
              f"shadow={stats['shadow_rays']}/{rs}")
        assert ref[fin].mean() > 0 and mre <= MRE_TOL
        assert abs(stats["extension_rays"] - re) <= max(2, 1e-3 * re)
        assert abs(stats["shadow_rays"] - rs) <= max(2, 1e-3 * rs)
