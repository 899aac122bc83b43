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
    hit = rp != -1          # two-sided traces report back faces as -2 - index
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


def _check_two_sided(scn, dscene, oracle, rays):
    got = dscene.trace(rays, two_sided=True)
    ref = oracle.trace_brute(scn.triangle_soup(), rays, two_sided=True, threads=cpu_threads())
    bad = _same_closest(got, ref)
    n_bad = int(bad.sum())
    assert n_bad == 0, (f"{n_bad} of {len(rays)} two-sided hits differ; first: ray {np.argmax(bad)} "
                        f"got {got[np.argmax(bad)]} ref {ref[np.argmax(bad)]}")
    return got


def test_two_sided_closest(room, oracle):
    """FF_TRACE_TWO_SIDED (the traversal of rays inside refracting objects):
    bit-exact against the oracle's mirrored culling test, back faces as
    prim = -2 - index, ties to the lowest index; a front-face answer equals
    the culling trace's answer for the same ray."""
    scn, ds = room
    P = np.asarray(scn.positions, np.float64)
    sphere = P[np.unique(np.asarray(scn.indices)[np.asarray(scn.material_ids) == 1])]
    c = sphere.mean(0)
    rad = float(np.linalg.norm(sphere - c, axis=1).max())
    rng = np.random.default_rng(41)
    rays = scenes.incoherent_rays(scn, 150_000, seed=42)
    # half the origins inside the sphere: their rays leave through back faces
    k = len(rays) // 2
    u = rng.normal(size=(k, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    rays[:k, 0:3] = (c + u * (0.95 * rad * rng.random((k, 1)) ** (1 / 3))).astype(np.float32)
    got = _check_two_sided(scn, ds, oracle, rays)
    back = got["prim"] < -1
    assert back[:k].mean() > 0.9 and back[k:].mean() > 0.01
    cull = ds.trace(rays)
    front = got["prim"] >= 0
    assert np.array_equal(got[front].view(np.uint32), cull[front].view(np.uint32))
    # edge cases of the mirrored test: the coincident-triangle tie, rays along
    # the axes from inside the sphere, and a tmin interval
    r2 = rays[:20_000].copy()
    axes = np.eye(3, dtype=np.float32)
    r2[:3000, 4:7] = axes[np.arange(3000) % 3] * np.where(np.arange(3000) % 2 == 0, 1, -1)[:, None]
    r2[3000:6000, 3] = rng.uniform(0.0, 1.0, 3000).astype(np.float32)
    _check_two_sided(scn, ds, oracle, r2)


def test_two_sided_ties_and_device_path(ctx, oracle):
    import firefly_b200 as ff
    import torch
    # 40 coincident copies of one triangle, half of them wound the other way:
    # every ray hits at the same t from either side; the lowest index wins
    P = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    I = np.arange(120, dtype=np.uint32).reshape(40, 3)
    I[1::2] = I[1::2][:, [0, 2, 1]]
    scn = scenes.Scene(positions=np.tile(P, (40, 1)), indices=I)
    ds = ff.dScene(ctx, scn)
    rng = np.random.default_rng(43)
    rays = np.zeros((8000, 8), np.float32)
    rays[:, 0:2] = rng.uniform(-0.5, 1.5, (8000, 2))
    rays[:, 2] = rng.choice([-1.0, 1.0], 8000)
    rays[:, 6] = -np.sign(rays[:, 2])
    rays[:, 7] = np.inf
    got = _check_two_sided(scn, ds, oracle, rays)
    hit = got["prim"] != -1
    # index 0 faces +z: rays from above see its front, rays from below its back
    assert set(np.unique(got["prim"][hit])) <= {0, -2}
    d_rays = torch.from_numpy(rays).cuda()
    d_hits = torch.empty((len(rays), 4), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ds.trace_device(d_rays.data_ptr(), len(rays), d_hits.data_ptr(), two_sided=True)
    ds.ctx.sync()
    dev = d_hits.cpu().numpy().view(np.uint8).view(got.dtype).reshape(-1)
    assert np.array_equal(dev.view(np.uint32), got.view(np.uint32))
    # any-hit rays are two-sided already: the flag is refused for them
    with pytest.raises(ff.FireflyError):
        ds.trace(rays, any_hit=True, two_sided=True)


def test_at_scale_mesh_bit_exact(ctx, oracle):
    """The at-scale mesh itself (icosphere subdivided 8x and displaced, in the
    room: 1,310,732 triangles; its 8-wide BVH quantises boxes on a far finer
    grid than the small room's): 1M incoherent rays and the 1920 x 1080
    camera frame's primary rays, closest hits bit for bit (ids, t, u, v;
    ties to the lowest index) against the oracle's CPU hierarchy, which
    decides every triangle with the same restated test as the brute force;
    any-hit answers for 500k rays with random tmax; two-sided closest hits
    for 500k rays from inside the sphere."""
    import firefly_b200 as ff
    scn = scenes.displaced_icosphere(subdiv=8, width=1920, height=1080, env_w=64, env_h=32)
    assert scn.num_triangles == 1_310_732
    ds = ff.dScene(ctx, scn)
    bvh = oracle.BVH(scn.triangle_soup())
    try:
        sets = {"incoherent": scenes.incoherent_rays(scn, 1_000_000, seed=51),
                "camera": scenes.camera_rays(scn, 1920, 1080)}
        for name, rays in sets.items():
            got = ds.trace(rays)
            ref = bvh.trace(rays, threads=cpu_threads())
            bad = _same_closest(got, ref)
            assert int(bad.sum()) == 0, (name, int(bad.sum()), got[np.argmax(bad)], ref[np.argmax(bad)])
            assert (got["prim"] >= 0).mean() > 0.5
        anyr = scenes.with_random_tmax(scenes.incoherent_rays(scn, 500_000, seed=52), scn, seed=53)
        ga, ra = ds.trace(anyr, any_hit=True), bvh.trace(anyr, any_hit=True, threads=cpu_threads())
        assert np.array_equal(ga["prim"] >= 0, ra["prim"] >= 0)
        P = np.asarray(scn.positions, np.float64)[24:]   # the sphere (after the room's 24 vertices)
        c = P.mean(0)
        rng = np.random.default_rng(54)
        inside = scenes.incoherent_rays(scn, 500_000, seed=55)
        inside[:, 0:3] = (c + rng.normal(size=(len(inside), 3)) * 0.3).astype(np.float32)
        g2, r2 = ds.trace(inside, two_sided=True), bvh.trace(inside, two_sided=True, threads=cpu_threads())
        bad = _same_closest(g2, r2)
        assert int(bad.sum()) == 0, int(bad.sum())
        assert (g2["prim"] < -1).mean() > 0.9
    finally:
        bvh.close()
        ds.close()


def test_traversal_pinned_by_oracle_restatement(ctx, oracle):
    """ff_trace_count's node and triangle counts, and ff_trace's answers, against
    the oracle's restatement of the device traversal (oracle/ffo_bvh8.c: the
    same box arithmetic, child order, stack and triangle tests) over the BVH
    read back from the device (ff_scene_read_bvh): the counts are equal ray
    set by ray set, closest hits bit for bit, and any-hit answers report the
    same occluder at the same t (the same traversal order finds it first)."""
    import firefly_b200 as ff
    for name, scn in (("room", scenes.small_room(seed=0)),
                      ("sphere in room", scenes.displaced_icosphere(subdiv=6, width=320, height=180,
                                                                    env_w=64, env_h=32))):
        ds = ff.dScene(ctx, scn)
        try:
            nodes, tris = ds.read_bvh()
            st = ds.stats()
            assert nodes.shape == (st["num_nodes"], 80) and tris.shape == (st["num_triangles"], 48)
            rng = np.random.default_rng(61)
            sets = [("incoherent", scenes.incoherent_rays(scn, 200_000, seed=62), False, False),
                    ("camera", scenes.camera_rays(scn, 320, 180), False, False),
                    ("any", scenes.with_random_tmax(scenes.incoherent_rays(scn, 200_000, seed=63), scn, seed=64),
                     True, False)]
            inside = scenes.incoherent_rays(scn, 100_000, seed=65)
            P = np.asarray(scn.positions, np.float64)[24:] if name != "room" else np.asarray(scn.positions)
            inside[:, 0:3] = (P.mean(0) + rng.normal(size=(len(inside), 3)) * 0.2).astype(np.float32)
            sets.append(("two-sided", inside, False, True))
            for label, rays, any_hit, two in sets:
                got = ds.trace(rays, any_hit=any_hit, two_sided=two)
                cnt = ds.trace_count(rays, any_hit=any_hit, two_sided=two)
                ref, n_nodes, n_tris, errors = oracle.bvh8_trace(nodes, tris, rays, any_hit=any_hit,
                                                                 two_sided=two, threads=cpu_threads())
                assert errors == 0
                assert (cnt["nodes"], cnt["tris"]) == (n_nodes, n_tris), (name, label, cnt, n_nodes, n_tris)
                bad = got["prim"] != ref["prim"]
                for f in ("t", "u", "v"):
                    bad |= got[f].view(np.uint32) != ref[f].view(np.uint32)
                assert int(bad.sum()) == 0, (name, label, int(bad.sum()), got[np.argmax(bad)], ref[np.argmax(bad)])
                print(f"[trace] {name}, {label}: {n_nodes / len(rays):.3f} nodes, {n_tris / len(rays):.3f} "
                      f"triangles per ray, equal on the device and in the restatement")
        finally:
            ds.close()
