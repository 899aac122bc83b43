"""Pins the oracle (oracle/ffo_*.c, the CPU restatement) to golden vectors
produced by the reference's own routines compiled for the host
(tests/golden/make_golden.py).  CPU only.

Bit-exact for intersection, hashing, draws, warps, sampling directions,
upper_bound and the environment tables; shading values within 2 float ulps
(the reference evaluates pow(x, 5) and pow(x, 2) with libm, the restatement
with multiplications; the results agree to the last bit in almost every case,
which the test also checks).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_vectors.npz"
P = C.c_void_p


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def lib(oracle):
    L = oracle.load()
    sig = {
        "ffo_probe_material": (None, [P, P, P, P, P]),
        "ffo_probe_diff_sample": (None, [P, C.c_float, C.c_float, P]),
        "ffo_probe_spec_sample": (None, [P, P, C.c_float, C.c_float, C.c_float, P]),
        "ffo_probe_concentric_disk": (None, [C.c_float, C.c_float, P]),
        "ffo_probe_upper_bound": (C.c_int, [P, C.c_int, C.c_float]),
        "ffo_probe_camera": (None, [P, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, P, P, P]),
        "ffo_probe_env": (None, [P, C.c_int, C.c_int, P, P, P, P, C.c_float, C.c_float, P, P]),
        "ffo_probe_area": (None, [P, P, P, P, P, P, P]),
        "ffo_probe_surface": (None, [P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


def p(a):
    return a.ctypes.data


def draw(lib, s):
    """The reference's random() for clock value s: float(wang_hash(s) * 2^-32),
    which the oracle's ffo_rand gives for key = s ^ wang_hash(0), dim 0."""
    return lib.ffo_rand(int(s) ^ lib.ffo_wang_hash(0), 0)


def ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7fffffff), a)
    b = np.where(b < 0, -(b & 0x7fffffff), b)
    return np.abs(a - b)


def test_ray_triangle_intersect(g, oracle):
    tris, rays, ref = g["tri_tris"], g["tri_rays"], g["tri_isect"]
    for i in range(len(tris)):
        ok, t, u, v = oracle.intersect_cull(tris[i, 0:3], tris[i, 3:6], tris[i, 6:9], rays[i, 0:3], rays[i, 4:7])
        assert ok == int(ref[i, 0]), i
        if ok:
            assert np.float32(t).view(np.uint32) == ref[i, 1:2].view(np.uint32)[0], i
            assert np.float32(u).view(np.uint32) == ref[i, 2:3].view(np.uint32)[0], i
            assert np.float32(v).view(np.uint32) == ref[i, 3:4].view(np.uint32)[0], i
    assert 500 < ref[:, 0].sum() < len(ref)


def test_shadow_hit(g, oracle):
    tris, rays, ref = g["tri_tris"], g["tri_rays"], g["tri_shadow"]
    for i in range(len(tris)):
        ok, t = oracle.shadow_hit(tris[i, 0:3], tris[i, 3:6], tris[i, 6:9], rays[i, 0:3], rays[i, 4:7])
        assert ok == int(ref[i, 0]), i
        if ok:
            assert np.float32(t) == ref[i, 1], i


def test_wang_hash_and_draws(g, lib):
    for s, h in zip(g["hash_in"], g["hash_out"]):
        assert lib.ffo_wang_hash(int(s)) == int(h)
    got = np.array([draw(lib, s) for s in g["hash_in"]], np.float32)
    assert np.array_equal(got.view(np.uint32), g["rand_out"].view(np.uint32))
    assert got.max() <= 1.0


def test_uniform_sample_square_draw_order(g, lib):
    # make_float2(random(), random()) in the reference's host build: x takes the second draw
    for s, ref in zip(g["square_seeds"], g["square_out"]):
        assert np.float32(draw(lib, s[1])) == ref[0]
        assert np.float32(draw(lib, s[0])) == ref[1]


def test_concentric_disk(g, lib):
    out = np.zeros(2, np.float32)
    for u, ref in zip(g["disk_in"], g["disk_out"]):
        lib.ffo_probe_concentric_disk(float(u[0]), float(u[1]), p(out))
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


def test_material_lobes(g, lib):
    mats, ns, wis, wos, ref = g["mat_params"], g["mat_n"], g["mat_wi"], g["mat_wo"], g["mat_out"]
    got = np.zeros_like(ref)
    for i in range(len(mats)):
        lib.ffo_probe_material(p(mats[i]), p(ns[i]), p(wis[i]), p(wos[i]), p(got[i]))
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(got))
    d = ulps(got[fin], ref[fin])
    assert d.max() <= 2, d.max()
    assert (d == 0).mean() > 0.995


def test_sampling_directions(g, lib):
    mats, ns, wos, seeds = g["mat_params"], g["mat_n"], g["mat_wo"], g["sample_seeds"]
    out = np.zeros(3, np.float32)
    for i in range(len(mats)):
        e0, e1 = draw(lib, seeds[i, 0]), draw(lib, seeds[i, 1])
        lib.ffo_probe_diff_sample(p(ns[i]), e0, e1, p(out))
        assert ulps(out, g["diff_sample_out"][i]).max() == 0, i
        lib.ffo_probe_spec_sample(p(ns[i]), p(wos[i]), float(mats[i, 6]), e0, e1, p(out))
        assert ulps(out, g["spec_sample_out"][i]).max() <= 1, i


def test_camera_rays(g, lib):
    out = np.zeros(6, np.float32)
    for inv, cin, ref, s in zip(g["cam_inv"], g["cam_in"], g["cam_out"], g["cam_seeds"]):
        lens, focal, W, H, px, py = cin
        jit = np.array([draw(lib, s[1]), draw(lib, s[0])], np.float32)
        lns = np.array([draw(lib, s[3]), draw(lib, s[2])], np.float32)
        lib.ffo_probe_camera(p(np.ascontiguousarray(inv)), float(lens), float(focal), 0.005, int(W), int(H), int(px),
                             int(py), p(jit), p(lns), p(out))
        assert ulps(out, ref).max() == 0


def test_environment_tables_and_sampling(g, lib, oracle):
    env = g["env_rgb"]
    m, c, pdf, den = oracle.env_build(env)
    assert np.array_equal(m, g["env_marginal"])
    assert np.array_equal(np.isnan(c), np.isnan(g["env_cond"]))
    ok = ~np.isnan(c)
    assert np.array_equal(c[ok], g["env_cond"][ok])
    assert np.array_equal(pdf, g["env_pdf"])
    assert den == g["env_denom"][0]
    out = np.zeros(10, np.float32)
    h, w = env.shape[:2]
    for pos, s, q, ref in zip(g["env_pos"], g["env_seeds"], g["env_q"], g["env_out"]):
        ex, ey = draw(lib, s[0]), draw(lib, s[1])
        lib.ffo_probe_env(p(env), w, h, p(m), p(np.ascontiguousarray(c)), p(pdf), p(pos), ex, ey, p(q), p(out))
        assert ulps(out, ref).max() == 0
    for v, ref in zip(g["ub_vals"], g["ub_out"]):
        assert lib.ffo_probe_upper_bound(p(m), h, float(v)) == ref


def test_area_light(g, lib, oracle):
    rect = g["area_rect"]
    L = oracle.ffo_area_light()
    for k in range(3):
        L.p0[k], L.a[k], L.b[k], L.normal[k], L.emissive[k] = rect[k], rect[3 + k], rect[6 + k], rect[9 + k], g["area_emissive"][k]
    L.radiance = 15.0
    out = np.zeros(11, np.float32)
    for pos, s, ray, ref in zip(g["area_pos"], g["area_seeds"], g["area_rays"], g["area_out"]):
        u = np.array([draw(lib, s[1]), draw(lib, s[0])], np.float32)
        up = np.array([draw(lib, s[3]), draw(lib, s[2])], np.float32)
        wi = ref[3:6].copy()
        lib.ffo_probe_area(C.byref(L), p(pos), p(u), p(wi), p(up), p(ray), p(out))
        assert ulps(out[:10], ref[:10]).max() == 0
        assert out[10] == ref[10]


def test_reference_bvh_agrees_with_brute_force(g, oracle):
    """The reference's own SAH BVH + intersect() against the oracle's brute
    force on 20,000 incoherent rays in the small room (original ids; the
    reference breaks exact ties in traversal order, the oracle to the lowest
    id, so only such ties could differ)."""
    from firefly_b200 import scenes
    scn = scenes.small_room(seed=0)
    ref = g["bvh_hits"]
    brute = oracle.trace_brute(scn.triangle_soup(), g["bvh_rays"])
    ref_prim = ref[:, 1].copy().view(np.int32)
    same = ref_prim == brute["prim"]
    assert same.mean() >= 0.9999, same.mean()
    hit = same & (brute["prim"] >= 0)
    assert np.array_equal(ref[hit, 0], brute["t"][hit])


def test_material_textures_and_normal_map(g, lib, oracle):
    """get_albedo / get_roughness / get_metallic / get_normal with every
    texture slot (base colour, roughness, metallic, packed metallic-roughness,
    tangent-space normal) at random texcoords (wrapping) and tangent frames,
    bit for bit against the reference's own routines."""
    texs = [np.ascontiguousarray(g[f"surf_tex{k}"]) for k in range(6)]
    tdesc = (oracle.ffo_texture * len(texs))()
    for i, t in enumerate(texs):
        tdesc[i].rgb, tdesc[i].width, tdesc[i].height = t.ctypes.data, t.shape[1], t.shape[0]
    mats, slots, isect, ref = g["surf_mat"], g["surf_slots"], g["surf_isect"], g["surf_out"]
    got = np.zeros_like(ref)
    for i in range(len(mats)):
        m = oracle.ffo_material()
        for k in range(3):
            m.base_color[k] = mats[i, k]
            m.fresnel[k] = mats[i, 3 + k]
        m.roughness, m.metallic, m.kind = float(mats[i, 6]), float(mats[i, 7]), 0
        (m.base_color_tex, m.roughness_tex, m.metallic_tex, m.metallic_roughness_tex,
         m.normal_tex) = (int(x) for x in slots[i])
        lib.ffo_probe_surface(C.byref(m), C.cast(tdesc, C.c_void_p), p(np.ascontiguousarray(isect[i])), p(got[i]))
    assert (slots[:, 4] >= 0).sum() > 100 and (slots[:, 3] >= 0).sum() > 100
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), ulps(got, ref).max()
