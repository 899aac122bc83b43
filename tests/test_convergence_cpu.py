"""Host-side pieces of the convergence measurement: the tile camera sees the
same pixel centres as the full frame, and relMSE's definition."""
import numpy as np

from firefly_b200 import convergence, scenes


def test_tile_camera_rays_match_full_frame():
    scn = scenes.small_room(seed=0, width=96, height=64)
    W, H = 96, 64
    full = scenes.camera_rays(scn, W, H).reshape(H, W, 8)
    for (x0, y0, tw, th) in [(10, 7, 32, 20), (0, 0, 96, 64), convergence.centre_tile(W, H)]:
        cam = convergence.tile_camera(scn.camera, W, H, x0, y0, tw, th)
        tile = scenes.camera_rays(scenes.Scene(**{**scn.__dict__, "camera": cam}), tw, th).reshape(th, tw, 8)
        ref = full[y0:y0 + th, x0:x0 + tw]
        assert np.allclose(tile[..., :3], ref[..., :3], atol=1e-4)
        assert np.allclose(tile[..., 4:7], ref[..., 4:7], atol=1e-5)


def test_relmse():
    ref = np.full((4, 4, 3), 2.0)
    img = ref * 1.1
    assert abs(convergence.relmse(img, ref) - 0.04 / (4 + 1e-2)) < 1e-12
    assert convergence.relmse(ref, ref) == 0.0


def test_relmse_skips_nonfinite_and_trims():
    ref = np.ones((100, 100, 3))
    img = ref.copy()
    img[0, 0] = np.nan
    img[1, 1] = 1000.0
    assert convergence.nonfinite_pixels(img) == 1
    full = convergence.relmse(img, ref)
    assert np.isfinite(full) and full > 10
    assert convergence.relmse_trimmed(img, ref) == 0.0
