"""Trace parity on the GPU: ff_trace (8-wide BVH, persistent kernel) against
the oracle's brute-force restatement of dTriangle::intersect / shadow_hit.

Closest-hit: prim, t, u and v must be bit-identical (ties to the lowest
original index).  Any-hit: the occluded / unoccluded answer must agree.
"""
from __future__ import annotations

import numpy as np
import pytest

from firefly_b200 import scenes
from tests.conftest import cpu_threads

pytestmark = pytest.mark.gpu


def _same_closest(got, ref):
    gp, rp = got["prim"], ref["prim"]
    bad = gp != rp
    hit = rp >= 0
    for f in ("t", "u", "v"):
        g = got[f].view(np.uint32)
        r = ref[f].view(np.uint32)
        bad |= hit & (g != r)
    return bad


def _check_closest(scn, dscene, oracle, rays):
    got = dscene.trace(rays, any_hit=False)
    ref = oracle.trace_brute(scn.triangle_soup(), rays, any_hit=False, threads=cpu_threads())
    bad = _same_closest(got, ref)
    n_bad = int(bad.sum())
    assert n_bad == 0, (f"{n_bad} of {len(rays)} closest hits differ; first: ray {np.argmax(bad)} "
                        f"got {got[np.argmax(bad)]} ref {ref[np.argmax(bad)]}")
    return got


def _check_any(scn, dscene, oracle, rays):
    got = dscene.trace(rays, any_hit=True)
    ref = oracle.trace_brute(scn.triangle_soup(), rays, any_hit=True, threads=cpu_threads())
    bad = (got["prim"] >= 0) != (ref["prim"] >= 0)
    n_bad = int(bad.sum())
    assert n_bad == 0, f"{n_bad} of {len(rays)} any-hit answers differ; first ray {np.argmax(bad)}"
    return got


@pytest.fixture(scope="module")
def room(ctx):
    import firefly_b200 as ff
    scn = scenes.small_room(seed=0)
    return scn, ff.dScene(ctx, scn)


def test_room_stats(room):
    scn, ds = room
    st = ds.stats()
    assert st["num_triangles"] == 4120
    assert 1 <= st["num_nodes"] <= 4120
    assert 1 <= st["bvh_depth"] <= 64


def test_closest_incoherent(room, oracle):
    scn, ds = room
    rays = scenes.incoherent_rays(scn, 200_000, seed=11)
    got = _check_closest(scn, ds, oracle, rays)
    assert (got["prim"] >= 0).mean() > 0.95   # closed room: nearly every ray hits


def test_closest_coherent(room, oracle):
    scn, ds = room
    rays = scenes.camera_rays(scn, 384, 384)
    _check_closest(scn, ds, oracle, rays)


def test_any_hit_random_tmax(room, oracle):
    scn, ds = room
    rays = scenes.with_random_tmax(scenes.incoherent_rays(scn, 200_000, seed=12), scn, seed=13)
    got = _check_any(scn, ds, oracle, rays)
    frac = (got["prim"] >= 0).mean()
    assert 0.05 < frac < 1.0


def test_any_hit_short_rays(room, oracle):
    scn, ds = room
    rays = scenes.incoherent_rays(scn, 100_000, seed=14)
    rays[:, 7] = np.random.default_rng(15).uniform(0.001, 2.0, len(rays)).astype(np.float32)
    _check_any(scn, ds, oracle, rays)


def test_tmin_interval(room, oracle):
    scn, ds = room
    rays = scenes.incoherent_rays(scn, 50_000, seed=16)
    rng = np.random.default_rng(17)
    rays[:, 3] = rng.uniform(0.0, 3.0, len(rays)).astype(np.float32)
    rays[:, 7] = (rays[:, 3] + rng.uniform(0.0, 8.0, len(rays))).astype(np.float32)
    _check_closest(scn, ds, oracle, rays)
    _check_any(scn, ds, oracle, rays)


def test_edge_cases(room, oracle):
    """Axis-aligned and zero-component directions, rays through vertices and
    along edges of the room's quads, origins on surfaces."""
    scn, ds = room
    P = scn.positions
    rng = np.random.default_rng(18)
    rays = []
    axes = np.eye(3, dtype=np.float32)
    for k in range(4000):
        o = rng.uniform(-4.9, 4.9, 3).astype(np.float32)
        o[1] = rng.uniform(0.1, 9.9)
        if k % 4 == 0:
            d = axes[k % 3] * (1 if k % 8 < 4 else -1)
        elif k % 4 == 1:
            target = P[rng.integers(0, len(P))]       # aim at a vertex exactly
            d = (target - o).astype(np.float64)
            d /= np.linalg.norm(d)
        elif k % 4 == 2:
            d = rng.normal(size=3)
            d[rng.integers(0, 3)] = 0.0                # one zero component
            d /= np.linalg.norm(d)
        else:
            o = P[rng.integers(0, 24)].copy()          # origin on a room corner
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
        rays.append([*o, 0.0, *np.asarray(d, np.float32), np.inf])
    rays = np.asarray(rays, np.float32)
    _check_closest(scn, ds, oracle, rays)
    _check_any(scn, ds, oracle, rays)


def test_degenerate_and_empty_scenes(ctx, oracle):
    import firefly_b200 as ff
    # one triangle
    scn = scenes.Scene(positions=np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32),
                       indices=np.array([[0, 1, 2]], np.uint32))
    ds = ff.dScene(ctx, scn)
    rng = np.random.default_rng(3)
    rays = np.zeros((5000, 8), np.float32)
    rays[:, 0:2] = rng.uniform(-0.5, 1.5, (5000, 2))
    rays[:, 2] = rng.choice([-1.0, 1.0], 5000)
    rays[:, 6] = -np.sign(rays[:, 2])
    rays[:, 7] = np.inf
    _check_closest(scn, ds, oracle, rays)
    _check_any(scn, ds, oracle, rays)
    # many coincident triangles: ties must go to the lowest index
    P = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    scn2 = scenes.Scene(positions=np.tile(P, (40, 1)), indices=np.arange(120, dtype=np.uint32).reshape(40, 3))
    ds2 = ff.dScene(ctx, scn2)
    got = _check_closest(scn2, ds2, oracle, rays)
    assert set(np.unique(got["prim"])) <= {-1, 0}
    # empty scene: every ray misses
    scn3 = scenes.Scene(positions=np.zeros((0, 3), np.float32), indices=np.zeros((0, 3), np.uint32))
    ds3 = ff.dScene(ctx, scn3)
    h = ds3.trace(rays[:100])
    assert np.all(h["prim"] == -1)
    # zero rays
    assert len(ds.trace(rays[:0])) == 0


def test_invalid_scene_rejected(ctx):
    import firefly_b200 as ff
    bad = scenes.Scene(positions=np.zeros((3, 3), np.float32), indices=np.array([[0, 1, 5]], np.uint32))
    with pytest.raises(ff.FireflyError) as e:
        ff.dScene(ctx, bad)
    assert e.value.status == 1
    nan = scenes.Scene(positions=np.array([[0, 0, 0], [np.nan, 0, 0], [0, 1, 0]], np.float32),
                       indices=np.array([[0, 1, 2]], np.uint32))
    with pytest.raises(ff.FireflyError):
        ff.dScene(ctx, nan)


def test_device_pointer_path_matches_host_path(room):
    import torch
    scn, ds = room
    rays = scenes.incoherent_rays(scn, 100_000, seed=19)
    host = ds.trace(rays)
    d_rays = torch.from_numpy(rays).cuda()
    d_hits = torch.empty((len(rays), 4), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ds.trace_device(d_rays.data_ptr(), len(rays), d_hits.data_ptr())
    ds.ctx.sync()
    dev = d_hits.cpu().numpy().view(np.uint8).view(host.dtype).reshape(-1)
    assert np.array_equal(dev.view(np.uint32), host.view(np.uint32))


def test_trace_count(ctx, room):
    """ff_trace_count: deterministic, the same from host and device rays,
    at least the root node per ray and a tested triangle per hit, and on a
    one-triangle scene at most one test per ray and node."""
    import firefly_b200 as ff
    import torch
    scn, ds = room
    rays = scenes.incoherent_rays(scn, 100_000, seed=23)
    n = len(rays)
    c1, c2 = ds.trace_count(rays), ds.trace_count(rays)
    assert c1 == c2
    d_rays = torch.from_numpy(rays).cuda()
    torch.cuda.synchronize()
    assert ds.trace_count(d_rays.data_ptr(), n) == c1
    assert c1["node_bytes"] == 80 and c1["tri_bytes"] == 48
    hits = ds.trace(rays)
    assert c1["nodes"] >= n and c1["tris"] >= int((hits["prim"] >= 0).sum())
    ca = ds.trace_count(rays, any_hit=True)
    assert ca["nodes"] >= n and ca["tris"] >= int((ds.trace(rays, any_hit=True)["prim"] >= 0).sum())
    print(f"[trace] room, incoherent: {c1['nodes'] / n:.2f} nodes, {c1['tris'] / n:.2f} tris per ray "
          f"({c1['fetch_bytes_per_ray']:.0f} B); any-hit {ca['fetch_bytes_per_ray']:.0f} B")

    one = scenes.Scene(positions=np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32),
                       indices=np.array([[0, 1, 2]], np.uint32))
    ds1 = ff.dScene(ctx, one)
    nn = ds1.stats()["num_nodes"]
    rng = np.random.default_rng(5)
    r1 = np.zeros((4096, 8), np.float32)
    r1[:, 0:2] = rng.uniform(-0.5, 1.5, (4096, 2))
    r1[:, 2] = 1.0
    r1[:, 6] = -1.0
    r1[:, 7] = np.inf
    c = ds1.trace_count(r1)
    h = ds1.trace(r1)
    assert len(r1) <= c["nodes"] <= nn * len(r1)
    assert int((h["prim"] >= 0).sum()) <= c["tris"] <= len(r1)
    empty = scenes.Scene(positions=np.zeros((0, 3), np.float32), indices=np.zeros((0, 3), np.uint32))
    ds0 = ff.dScene(ctx, empty)
    assert ds0.trace_count(r1[:10])["nodes"] == 0
    assert ds.trace_count(rays[:0])["rays"] == 0
