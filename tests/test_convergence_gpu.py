"""Convergence against float64-accumulated references: the renderer's error
falls as 1/spp against a reference of the same estimator (unbiased in the
corrected mode, the reference's own estimator in the parity mode), and a tile
reference agrees with the full-frame one on its pixels."""
import numpy as np
import pytest

from firefly_b200 import convergence, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1])
def test_relmse_falls_as_one_over_spp(ctx, mode):
    import firefly_b200 as ff
    scn = scenes.small_room(seed=0, width=128, height=128)
    ds = ff.dScene(ctx, scn)
    kw = dict(max_depth=5, rr_depth=3, light=0, mode=mode)
    ref, info = convergence.reference_image(ctx, ds, scn.camera, 128, 128, spp=8192, **kw)
    pt = ff.PathTracer(ctx, 128, 128)
    errs = {}
    for spp in (4, 16, 64):
        pt.clear_buffer()
        pt.draw(ds, spp=spp, seed=3, **kw)
        errs[spp] = convergence.relmse(pt.image(), ref)
    print(f"[convergence] mode={mode} relMSE {errs} (reference {info['seconds']:.1f} s, "
          f"{convergence.nonfinite_pixels(ref)} non-finite reference pixels)")
    assert convergence.nonfinite_pixels(ref) <= (128 * 128 // 1000 if mode == 0 else 0)
    for a, b in ((4, 16), (16, 64)):
        assert 0.15 < errs[b] / errs[a] < 0.4
    pt.close()
    ds.close()


def test_tile_reference_matches_full_frame(ctx):
    import firefly_b200 as ff
    scn = scenes.small_room(seed=0, width=64, height=48)
    ds = ff.dScene(ctx, scn)
    kw = dict(max_depth=5, rr_depth=3, light=0, mode=1)
    full, _ = convergence.reference_image(ctx, ds, scn.camera, 64, 48, spp=4096, **kw)
    tile = (20, 10, 24, 16)
    part, _ = convergence.reference_image(ctx, ds, scn.camera, 64, 48, tile=tile, spp=4096, **kw)
    sub = full[10:26, 20:44]
    # two independent 4096-spp estimates of the same pixels
    err = convergence.relmse(part, sub)
    print(f"[convergence] tile vs full frame, two 4096-spp estimates: relMSE {err:.2e}")
    assert err < 1e-2
    assert abs(part.mean() - sub.mean()) < 0.01 * sub.mean()
    ds.close()
