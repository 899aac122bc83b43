"""Converged reference images and the relative MSE of a render against them.

A reference is the same scene, camera and settings rendered with many more
samples (16,384 per pixel by default), drawn in chunks with disjoint sample
indices (ff_render_settings.sample_offset) under its own seed and summed in
float64 on the host, so that its own noise and rounding sit far below the
error of the render it judges.  Where a full frame at that count would take
minutes, a tile of the frame is rendered through a camera whose projection
covers exactly that tile's pixels (the same pixel centres as the full frame),
and the render is judged on the same tile.

relMSE follows the usual definition for Monte Carlo renders: the mean over
pixels and channels of (I - R)^2 / (R^2 + eps), eps = 1e-2, over the pixels
finite in both images (the parity mode keeps the reference renderer's rare
non-finite samples, which a 16k-spp sum collects).  Under a small, very
bright light a handful of paths that reach it through specular chains carry
most of the squared error; relmse_trimmed drops the largest 0.01 % of the
per-pixel terms as well, as rendering papers often do.
"""
from __future__ import annotations

import time

import numpy as np

from . import _abi as A

REFERENCE_SPP = 16384


def pixel_terms(img: np.ndarray, ref: np.ndarray, eps: float = 1e-2) -> np.ndarray:
    """Per-pixel relative squared error (mean over channels), finite pixels only."""
    img = np.asarray(img, np.float64)
    ref = np.asarray(ref, np.float64)
    ok = np.isfinite(img).all(-1) & np.isfinite(ref).all(-1)
    return ((img[ok] - ref[ok]) ** 2 / (ref[ok] * ref[ok] + eps)).mean(-1)


def relmse(img: np.ndarray, ref: np.ndarray, eps: float = 1e-2) -> float:
    return float(np.mean(pixel_terms(img, ref, eps)))


def relmse_trimmed(img: np.ndarray, ref: np.ndarray, eps: float = 1e-2, drop: float = 1e-4) -> float:
    t = np.sort(pixel_terms(img, ref, eps))
    return float(np.mean(t[:len(t) - int(np.ceil(len(t) * drop))]))


def nonfinite_pixels(img: np.ndarray) -> int:
    return int((~np.isfinite(np.asarray(img)).all(-1)).sum())


def tile_camera(cam: A.ff_camera, width: int, height: int, x0: int, y0: int, tw: int, th: int) -> A.ff_camera:
    """A camera whose tw x th film sees pixels [x0, x0+tw) x [y0, y0+th) of
    the width x height film of `cam`: the tile's NDC maps affinely onto the
    full frame's (x right, y down in pixels, up in NDC), composed into the
    inverse view-projection."""
    inv = np.asarray(cam.inv_view_proj, np.float64).reshape(4, 4).T      # math matrix, column vectors
    m = np.eye(4)
    m[0, 0], m[0, 3] = tw / width, (2.0 * x0 + tw) / width - 1.0
    m[1, 1], m[1, 3] = th / height, 1.0 - (2.0 * y0 + th) / height
    out = A.ff_camera()
    flat = (inv @ m).T.astype(np.float32).ravel()
    for k in range(16):
        out.inv_view_proj[k] = float(flat[k])
    out.lens_radius, out.focal_distance = cam.lens_radius, cam.focal_distance
    out.exposure, out.pixel_jitter = cam.exposure, cam.pixel_jitter
    return out


def centre_tile(width: int, height: int, frac: int = 4) -> tuple[int, int, int, int]:
    """The centred tile of 1/frac of each side (1/frac^2 of the pixels)."""
    tw, th = width // frac, height // frac
    return (width - tw) // 2, (height - th) // 2, tw, th


def reference_image(ctx, ds, cam: A.ff_camera, width: int, height: int, tile=None, spp: int = REFERENCE_SPP,
                    chunk: int = 256, seed: int = 0x5EED5EED, **settings) -> tuple[np.ndarray, dict]:
    """float64 [h, w, 3] mean radiance at `spp` samples per pixel of the
    width x height frame (or of its tile (x0, y0, tw, th)) rendered with
    PathTracer.draw `settings` (max_depth, rr_depth, mode, light, ...).
    The scene's camera is restored to `cam` afterwards."""
    from . import PathTracer
    x0, y0, tw, th = tile if tile is not None else (0, 0, width, height)
    ds.update(tile_camera(cam, width, height, x0, y0, tw, th) if tile is not None else cam)
    pt = PathTracer(ctx, tw, th)
    acc = np.zeros((th, tw, 3), np.float64)
    done = 0
    t0 = time.perf_counter()
    try:
        while done < spp:
            k = min(chunk, spp - done)
            pt.clear_buffer()
            pt.draw(ds, spp=k, seed=seed, sample_offset=done, **settings)
            rgba, n = pt.read()
            acc += rgba[..., :3].astype(np.float64)
            assert np.all(n == k)
            done += k
    finally:
        pt.close()
        ds.update(cam)
    return acc / spp, {"spp": spp, "tile": [x0, y0, tw, th], "seconds": time.perf_counter() - t0}
