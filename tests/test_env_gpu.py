"""Environment light on the GPU: the device-scan importance tables against
the oracle's serial restatement of kernel.cu:65-149, and image parity of
environment-lit renders (parity and corrected modes)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from firefly_b200 import scenes
from tests.conftest import cpu_threads

pytestmark = pytest.mark.gpu


def _tables(ds, w, h):
    import firefly_b200 as ff
    marginal = np.zeros(h, np.float64)
    cond = np.zeros((h, w), np.float64)
    pdf = np.zeros((h, w), np.float32)
    denom = np.zeros(1, np.float64)
    st = ff.lib().ff_scene_read_env_tables(ds.handle, marginal.ctypes.data_as(C.c_void_p),
                                           cond.ctypes.data_as(C.c_void_p), pdf.ctypes.data_as(C.c_void_p),
                                           denom.ctypes.data_as(C.c_void_p))
    assert st == 0
    return marginal, cond, pdf, float(denom[0])


@pytest.mark.parametrize("w,h", [(128, 64), (300, 150), (2048, 1024)])
def test_env_tables_match_oracle(ctx, oracle, w, h):
    import firefly_b200 as ff
    scn = scenes.sphere_under_sky(seed=1, env_w=w, env_h=h)
    ds = ff.dScene(ctx, scn)
    gm, gc, gp, gd = _tables(ds, w, h)
    rm, rc, rp, rd = oracle.env_build(scn.env_rgb)
    # The FP64 row sums and the denominator are reassociated into block
    # reductions (the CDFs are running sums in the reference's order), and the
    # float sine of a row (sin(M_PI * v), a float in the reference) can land
    # one float ulp away from the host libm's sinf (row 6 of 64 does: glibc
    # returns 0.2902847, the device's correctly rounded double sine gives
    # 0.29028466).  That row's marginal pdf then differs by up to one float
    # ulp (6e-8 relative) and the denominator by ~1e-10; the conditional CDFs
    # are normalised per row and agree to 1e-15.
    assert abs(gd - rd) <= 1e-8 * abs(rd)
    assert np.allclose(gm, rm, rtol=1.2e-7, atol=0)
    ok = np.isfinite(rc)
    assert np.array_equal(ok, np.isfinite(gc))        # rows of zero probability are NaN in both
    assert np.allclose(gc[ok], rc[ok], rtol=1e-12, atol=1e-300)
    assert np.allclose(gp, rp, rtol=1e-6, atol=0)       # the float pdf may differ in its last bits
    assert abs(gm[-1] - 1.0) < 1e-9                      # a normalised marginal CDF
    ds.close()


def _upper_bound(lst, vals):
    """upper_bound of Helpers.cu:16-31 for float32 draws: the binary search's
    end index (numpy's right-sided search where the list is sorted, the loop
    itself where it is not), then the reference's list[left <= val] step."""
    vals = np.asarray(vals, np.float32)
    n = len(lst)
    if np.all(lst[:-1] <= lst[1:]):
        left = np.searchsorted(lst, vals.astype(np.float64), side="right")
    else:
        left = np.empty(len(vals), np.int64)
        for i, v in enumerate(vals.astype(np.float64)):
            lo, hi = 0, n
            while lo < hi:
                mid = (hi - lo) // 2 + lo
                if v >= lst[mid]:
                    lo = mid + 1
                else:
                    hi = mid
            left[i] = lo
    idx = np.where(left.astype(np.float32) <= vals, 1, 0)
    return left + ((left < n) & (lst[idx] != 0.0))


def _picks_expected(marginal, cond, exy):
    h, w = cond.shape
    y = np.clip(_upper_bound(marginal, exy[:, 1]) - 1, 0, h - 1)
    x = np.empty(len(exy), np.int64)
    for row in np.unique(y):
        sel = y == row
        x[sel] = np.clip(_upper_bound(cond[row], exy[sel, 0]) - 1, 0, w - 1)
    return x, y


def _edge_draws(values, rng, n_random):
    """Uniform draws, the guide tables' bucket edges k / G, the table entries
    themselves as floats, their float neighbours, and 0 and 1."""
    edges = np.concatenate([np.arange(1025) / 1024.0, np.arange(513) / 512.0, values, [0.0, 1.0]]).astype(np.float32)
    edges = edges[(edges >= 0) & (edges <= 1)]
    near = np.concatenate([edges, np.nextafter(edges, np.float32(0)), np.nextafter(edges, np.float32(1))])
    return np.concatenate([rng.random(n_random, dtype=np.float32), near]).astype(np.float32)


@pytest.mark.parametrize("case", ["sky_sun_2048", "zero_rows_256"])
def test_env_pick_matches_full_search(ctx, case):
    """The light sample's texel (guided CDF searches, ff_debug_env_pick) is
    the one the reference's full upper_bound searches pick, draw for draw,
    on the device's own tables: at the C2 sky (2048 x 1024, 0.5 degree sun of
    5e4) and at a sky with black rows and black runs of texels (CDF plateaus,
    rows of zero probability whose conditional CDF is NaN)."""
    import firefly_b200 as ff
    rng = np.random.default_rng(7)
    if case == "sky_sun_2048":
        env = scenes.sky_env(2048, 1024, seed=0)
    else:
        env = scenes.sky_env(256, 128, seed=3, sun_radiance=500.0, sun_diameter_deg=3.0)
        env[40:56] = 0.0
        env[70:90, 10:120] = 0.0
    scn = scenes.sphere_under_sky(seed=0)
    scn.env_rgb = env
    h, w = env.shape[:2]
    ds = ff.dScene(ctx, scn)
    marginal, cond, _, _ = _tables(ds, w, h)
    ok = np.all(np.isfinite(cond), axis=1)
    # the CDFs are running sums: every finite row is sorted (the guide tables then apply)
    assert np.all(marginal[:-1] <= marginal[1:])
    assert np.all(cond[ok, :-1] <= cond[ok, 1:])
    # ey: draws and edges of the marginal; ex: draws and edges of the rows the
    # draws land in (plus the sun's row)
    ey = _edge_draws(marginal, rng, 200_000)
    rows = np.unique(np.clip(_upper_bound(marginal, ey[:2000]) - 1, 0, h - 1))
    ex_vals = _edge_draws(cond[rows[:16]].ravel(), rng, 200_000)
    m = max(len(ex_vals), len(ey))
    exy = np.stack([np.resize(ex_vals, m), np.resize(rng.permutation(ey), m)], axis=1).astype(np.float32)
    # every ex edge also against the row the sun sits in
    sun_row = int(np.argmax(np.diff(marginal, prepend=0.0)))
    ey_sun = np.float32(marginal[sun_row - 1] if sun_row > 0 else 0.0)
    exy = np.concatenate([exy, np.stack([ex_vals, np.full(len(ex_vals), ey_sun, np.float32)], axis=1)])
    exy = np.ascontiguousarray(exy, np.float32)
    xy = np.zeros((len(exy), 2), np.int32)
    st = ff.lib().ff_debug_env_pick(ds.handle, exy.ctypes.data_as(C.c_void_p), len(exy),
                                    xy.ctypes.data_as(C.c_void_p))
    assert st == 0
    x, y = _picks_expected(marginal, cond, exy)
    print(f"[env pick] {case}: {len(exy)} draws, {len(np.unique(y))} rows, {int((~ok).sum())} NaN rows")
    assert np.array_equal(xy[:, 1], y)
    assert np.array_equal(xy[:, 0], x)
    ds.close()


def test_env_render_parity(ctx, oracle):
    import firefly_b200 as ff
    scn = scenes.sphere_under_sky(seed=0, width=64, height=64)
    for mode in (ff.FF_MODE_PARITY, ff.FF_MODE_CORRECTED):
        ds = ff.dScene(ctx, scn)
        pt = ff.PathTracer(ctx, 64, 64)
        st = pt.draw(ds, spp=4, max_depth=4, rr_depth=3, seed=11, light=-1, mode=mode)
        rgba, n = pt.read()
        ref, (re, rs) = oracle.render(scn, 64, 64, 4, max_depth=4, rr_depth=3, seed=11, mode=mode, light=-1,
                                      threads=cpu_threads())
        got = rgba[..., :3].astype(np.float64)
        # parity mode keeps the reference's non-finite pixels (its env pdf divides
        # by sin(acos(wi.z)), which is 0 at the poles of the z axis): they must
        # occur at the same pixels on both sides
        bad_g, bad_r = ~np.isfinite(got), ~np.isfinite(ref)
        fin = ~(bad_g | bad_r)
        mre = float(np.abs(got[fin] - ref[fin]).sum() / np.abs(ref[fin]).sum())
        print(f"[parity] env mode={mode}: mre={mre:.3e} nonfinite gpu={int(bad_g.sum())} oracle={int(bad_r.sum())} "
              f"ext={st['extension_rays']}/{re} shadow={st['shadow_rays']}/{rs}")
        assert np.array_equal(bad_g, bad_r)
        assert bad_g.mean() < 0.01
        assert mre <= 1e-4
        assert np.all(n == 4)
        pt.close()
        ds.close()


def test_all_material_kinds_render(ctx):
    """Reduced at-scale scene (icosphere subdivided 4x, 32 materials of the
    five kinds, sky with sun): finite, non-negative, lit."""
    import firefly_b200 as ff
    scn = scenes.displaced_icosphere(subdiv=4, width=160, height=90, env_w=256, env_h=128)
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, 160, 90)
    st = pt.draw(ds, spp=4, max_depth=8, rr_depth=3, seed=0, light=-1, mode=ff.FF_MODE_CORRECTED)
    img = pt.image()
    assert np.all(np.isfinite(img)) and img.min() >= 0.0
    assert img.mean() > 0.0
    assert st["extension_rays"] > 160 * 90 * 4 and st["shadow_rays"] > 0
    pt.close()
    ds.close()
