"""Generate tests/golden/ref_vectors.npz from the reference's own routines.

Runs the reference's device code compiled for the host (oracle/_ref/
libffref.so, built by `make -C oracle ref` from the reference checkout) on
seeded inputs and stores inputs and outputs.  tests/test_oracle_golden.py
then pins the oracle's restatement (oracle/ffo_*.c) to these vectors.

Usage: python tests/golden/make_golden.py      (needs the reference checkout)

The reference's random() hashes a clock() value; the host build's clock() is
redirected to a sequence set per call (oracle/compat/ffref_compat.h), so a
draw with "seed" s returns float(wang_hash(s) * 2^-32).
"""
from __future__ import annotations

import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "ref_vectors.npz"
P = C.c_void_p


def load_ref():
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref"], check=True)
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libffref.so"))
    sig = {
        "ffref_set_clock": (None, [P, C.c_int]),
        "ffref_clock_used": (C.c_int, []),
        "ffref_intersect": (C.c_int, [P, P, P]),
        "ffref_shadow_hit": (C.c_int, [P, P, P]),
        "ffref_wang_hash": (C.c_uint32, [C.c_uint32]),
        "ffref_rand_draw": (C.c_float, []),
        "ffref_uniform_sample_square": (None, [P]),
        "ffref_concentric_sample_disk": (None, [P, P]),
        "ffref_material_eval": (None, [P, P, P, P, P]),
        "ffref_diff_sample": (None, [P, P, P]),
        "ffref_spec_sample": (None, [P, P, P, P]),
        "ffref_gen_ray": (None, [P, C.c_float, C.c_float, C.c_int, C.c_int, C.c_float, C.c_float, P]),
        "ffref_env_create": (P, [P, C.c_int, C.c_int]),
        "ffref_env_tables": (None, [P, P, P, P, P]),
        "ffref_env_sample": (None, [P, P, P, P]),
        "ffref_env_eval": (None, [P, P, P, P]),
        "ffref_upper_bound": (C.c_int, [P, C.c_int, C.c_float]),
        "ffref_area_create": (P, [P, C.c_float, P]),
        "ffref_area_sample": (None, [P, P, P, P]),
        "ffref_area_eval": (None, [P, P, P, P, P, P]),
        "ffref_area_hit": (C.c_int, [P, P]),
        "ffref_bvh_build": (P, [P, C.c_int, C.POINTER(C.c_double)]),
        "ffref_bvh_trace": (None, [P, P, C.c_long, P, C.c_int, C.c_int]),
        "ffref_tex_create": (C.c_ulonglong, [P, C.c_int, C.c_int, C.c_int]),
        "ffref_surface": (None, [P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def p(a):
    return a.ctypes.data


def with_clock(lib, seeds, fn):
    seq = np.ascontiguousarray(seeds, np.uint32)
    lib.ffref_set_clock(p(seq), len(seq))
    r = fn()
    used = lib.ffref_clock_used()
    lib.ffref_set_clock(None, 0)
    return r, used


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def main():
    lib = load_ref()
    rng = np.random.default_rng(20241203)
    out = {}

    # ---- ray/triangle tests: aimed rays, plus edge cases
    n = 3000
    tris = rng.normal(size=(n, 9)).astype(np.float32)
    bary = rng.uniform(-0.15, 1.15, size=(n, 2))
    v0, v1, v2 = tris[:, 0:3], tris[:, 3:6], tris[:, 6:9]
    target = v0 + bary[:, :1] * (v1 - v0) + bary[:, 1:2] * (v2 - v0)
    orig = target + unit(rng, n) * rng.uniform(0.5, 5.0, (n, 1))
    d = target - orig
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 4:7], rays[:, 7] = orig, d, np.inf
    # edge cases in the last rows
    k = 0
    for i in range(n - 400, n):
        kind = k % 8
        t = tris[i]
        a, b, c = t[0:3], t[3:6], t[6:9]
        if kind == 0:   # at a vertex
            tgt = [a, b, c][k % 3]
        elif kind == 1:  # edge midpoint
            tgt = 0.5 * (a + b)
        elif kind == 2:  # parallel: direction inside the triangle's plane
            rays[i, 0:3] = a - (b - a)
            dd = b - a
            rays[i, 4:7] = dd / np.linalg.norm(dd)
            k += 1
            continue
        elif kind == 3:  # origin on the triangle (t = 0)
            rays[i, 0:3] = (a + b + c) / 3
            nn = np.cross(b - a, c - a)
            rays[i, 4:7] = -nn / np.linalg.norm(nn)
            k += 1
            continue
        elif kind == 4:  # degenerate triangle (collinear)
            tris[i, 6:9] = 2 * b - a
            tgt = b
        elif kind == 5:  # nearly edge-on
            nn = np.cross(b - a, c - a)
            nn /= np.linalg.norm(nn)
            tgt = (a + b + c) / 3
            rays[i, 0:3] = tgt + (b - a) * 3 + nn * 1e-3
            dd = tgt - rays[i, 0:3]
            rays[i, 4:7] = dd / np.linalg.norm(dd)
            k += 1
            continue
        elif kind == 6:  # back face
            tgt = (a + b + c) / 3
        else:            # zero direction components
            tgt = (a + 2 * b + 3 * c) / 6
            rays[i, 0:3] = tgt + np.array([0, 0, 2.0], np.float32)
            rays[i, 4:7] = [0, 0, -1]
            k += 1
            continue
        o = tgt + np.array([0.3, -0.7, 1.1], np.float32) * (1 if kind != 6 else -1)
        dd = tgt - o
        rays[i, 0:3], rays[i, 4:7] = o, dd / np.linalg.norm(dd)
        k += 1
    isect = np.zeros((n, 4), np.float32)
    shadow = np.zeros((n, 2), np.float32)
    for i in range(n):
        tuv = np.zeros(3, np.float32)
        ok = lib.ffref_intersect(p(tris[i]), p(rays[i]), p(tuv))
        isect[i] = [ok, *tuv]
        t1 = np.zeros(1, np.float32)
        ok2 = lib.ffref_shadow_hit(p(tris[i]), p(rays[i]), p(t1))
        shadow[i] = [ok2, t1[0]]
    out.update(tri_tris=tris, tri_rays=rays, tri_isect=isect, tri_shadow=shadow)

    # ---- sampler
    hs = np.concatenate([np.arange(200, dtype=np.uint32), rng.integers(0, 2**32, 800, dtype=np.uint64).astype(np.uint32)])
    out["hash_in"] = hs
    out["hash_out"] = np.array([lib.ffref_wang_hash(int(s)) for s in hs], np.uint32)
    draws = []
    for s in hs:
        v, used = with_clock(lib, [s], lambda: lib.ffref_rand_draw())
        draws.append(v)
    out["rand_out"] = np.array(draws, np.float32)
    sq_seeds = rng.integers(0, 2**32, size=(300, 2), dtype=np.uint64).astype(np.uint32)
    sq = []
    for s in sq_seeds:
        o2 = np.zeros(2, np.float32)
        with_clock(lib, s, lambda: lib.ffref_uniform_sample_square(p(o2)))
        sq.append(o2.copy())
    out.update(square_seeds=sq_seeds, square_out=np.array(sq, np.float32))
    du = rng.random(size=(500, 2)).astype(np.float32)
    du[:6] = [[0, 0], [1, 1], [0.5, 0.5], [0.5, 0.9], [0.9, 0.5], [0.25, 0.75]]
    disk = []
    for u in du:
        o2 = np.zeros(2, np.float32)
        lib.ffref_concentric_sample_disk(p(u), p(o2))
        disk.append(o2.copy())
    out.update(disk_in=du, disk_out=np.array(disk, np.float32))

    # ---- materials
    m = 2000
    mat8 = np.zeros((m, 8), np.float32)
    mat8[:, 0:3] = rng.uniform(0.05, 0.95, (m, 3))
    mat8[:, 3:6] = 0.04
    mat8[:, 6] = rng.uniform(0.05, 1.0, m)
    mat8[:, 7] = rng.choice([0.0, 0.0, 1.0, 0.37], m)
    nrm = unit(rng, m)
    wi = unit(rng, m)
    wo = unit(rng, m)
    flip = (wi * nrm).sum(1) < 0
    wi[flip & (rng.random(m) < 0.85)] *= -1
    flip = (wo * nrm).sum(1) < 0
    wo[flip & (rng.random(m) < 0.85)] *= -1
    mres = np.zeros((m, 19), np.float32)
    isx6 = np.zeros((m, 6), np.float32)
    isx6[:, 3:6] = nrm
    for i in range(m):
        lib.ffref_material_eval(p(mat8[i]), p(isx6[i]), p(wi[i]), p(wo[i]), p(mres[i]))
    out.update(mat_params=mat8, mat_n=nrm, mat_wi=wi, mat_wo=wo, mat_out=mres[:, :17])
    seeds = rng.integers(0, 2**32, size=(m, 2), dtype=np.uint64).astype(np.uint32)
    ds_out = np.zeros((m, 3), np.float32)
    ss_out = np.zeros((m, 3), np.float32)
    for i in range(m):
        with_clock(lib, seeds[i], lambda: lib.ffref_diff_sample(p(mat8[i]), p(isx6[i]), p(ds_out[i])))
        with_clock(lib, seeds[i], lambda: lib.ffref_spec_sample(p(mat8[i]), p(isx6[i]), p(wo[i]), p(ss_out[i])))
    out.update(sample_seeds=seeds, diff_sample_out=ds_out, spec_sample_out=ss_out)

    # ---- camera
    from firefly_b200 import scenes
    cams = []
    cam_out = []
    cam_in = []
    for i in range(400):
        lens = 0.0 if i % 2 == 0 else float(rng.uniform(0.01, 0.2))
        cam = scenes.make_camera(eye=rng.uniform(-3, 3, 3), center=rng.uniform(-1, 1, 3), fovy=float(rng.uniform(30, 90)),
                                 aspect=float(rng.uniform(0.5, 2.0)), lens_radius=lens, focal_distance=float(rng.uniform(0.5, 5)))
        inv = np.array(cam.inv_view_proj, np.float32)
        W, H = int(rng.integers(16, 2000)), int(rng.integers(16, 2000))
        px, py = int(rng.integers(0, W)), int(rng.integers(0, H))
        s4 = rng.integers(0, 2**32, 4, dtype=np.uint64).astype(np.uint32)
        o6 = np.zeros(6, np.float32)
        with_clock(lib, s4, lambda: lib.ffref_gen_ray(p(inv), cam.lens_radius, cam.focal_distance, W, H,
                                                      float(px), float(py), p(o6)))
        cams.append(inv)
        cam_in.append([lens, cam.focal_distance, W, H, px, py])
        cam_out.append(o6.copy())
        out.setdefault("cam_seeds", []).append(s4)
    out.update(cam_inv=np.array(cams, np.float32), cam_in=np.array(cam_in, np.float64),
               cam_out=np.array(cam_out, np.float32), cam_seeds=np.array(out["cam_seeds"], np.uint32))

    # ---- environment light
    env = scenes.sky_env(64, 32, seed=3, sun_radiance=500.0, sun_diameter_deg=8.0)
    h_env = lib.ffref_env_create(p(env), 64, 32)
    marg = np.zeros(32, np.float64)
    cond = np.zeros((32, 64), np.float64)
    pdf = np.zeros((32, 64), np.float32)
    den = np.zeros(1, np.float64)
    lib.ffref_env_tables(h_env, p(marg), p(cond), p(pdf), p(den))
    ne = 600
    epos = rng.uniform(-2, 2, (ne, 3)).astype(np.float32)
    eseeds = rng.integers(0, 2**32, (ne, 2), dtype=np.uint64).astype(np.uint32)
    eq = unit(rng, ne)
    esamp = np.zeros((ne, 10), np.float32)
    for i in range(ne):
        wi3 = np.zeros(3, np.float32)
        sp3 = np.zeros(3, np.float32)
        with_clock(lib, eseeds[i], lambda: lib.ffref_env_sample(h_env, p(epos[i]), p(wi3), p(sp3)))
        L3 = np.zeros(3, np.float32)
        pd = np.zeros(1, np.float32)
        lib.ffref_env_eval(h_env, p(eq[i]), p(L3), p(pd))
        esamp[i] = [*wi3, *sp3, *L3, pd[0]]
    ub_vals = rng.random(500).astype(np.float32)
    ub_vals[:4] = [0.0, 1.0, marg[5], marg[-1]]
    ub = np.array([lib.ffref_upper_bound(p(marg), 32, float(v)) for v in ub_vals], np.int32)
    out.update(env_rgb=env, env_marginal=marg, env_cond=cond, env_pdf=pdf, env_denom=den, env_pos=epos,
               env_seeds=eseeds, env_q=eq, env_out=esamp, ub_vals=ub_vals, ub_out=ub)

    # ---- area light
    rect = np.array([-1.0, 9.99, -1.0, 2.0, 0.0, 0.0, 0.0, 0.0, 2.0, 0.0, -1.0, 0.0], np.float32)
    em = np.array([1.0, 0.9, 0.8], np.float32)
    h_area = lib.ffref_area_create(p(rect), 15.0, p(em))
    na = 600
    apos = rng.uniform(-4, 4, (na, 3)).astype(np.float32)
    apos[:, 1] = rng.uniform(0.5, 9.5, na)
    aseeds = rng.integers(0, 2**32, (na, 4), dtype=np.uint64).astype(np.uint32)
    aout = np.zeros((na, 11), np.float32)
    arays = np.zeros((na, 8), np.float32)
    for i in range(na):
        wi3 = np.zeros(3, np.float32)
        sp3 = np.zeros(3, np.float32)
        with_clock(lib, aseeds[i, :2], lambda: lib.ffref_area_sample(h_area, p(apos[i]), p(wi3), p(sp3)))
        L3 = np.zeros(3, np.float32)
        pd = np.zeros(1, np.float32)
        with_clock(lib, aseeds[i, 2:], lambda: lib.ffref_area_eval(h_area, p(apos[i]), p(wi3), p(sp3), p(L3), p(pd)))
        tgt = rect[0:3] + rng.uniform(-0.2, 1.2) * rect[3:6] + rng.uniform(-0.2, 1.2) * rect[6:9]
        dd = tgt - apos[i]
        arays[i, 0:3], arays[i, 4:7] = apos[i], dd / np.linalg.norm(dd)
        hit = lib.ffref_area_hit(h_area, p(arays[i]))
        aout[i] = [*sp3, *wi3, *L3, pd[0], hit]
    out.update(area_rect=rect, area_emissive=em, area_pos=apos, area_seeds=aseeds, area_rays=arays, area_out=aout)

    # ---- BVH trace of the reference (SAH BVH + intersect()) on the small room
    scn = scenes.small_room(seed=0)
    soup = scn.triangle_soup()
    ms = C.c_double()
    hb = lib.ffref_bvh_build(p(soup), len(soup), C.byref(ms))
    br = scenes.incoherent_rays(scn, 20000, seed=99)
    bh = np.zeros((len(br), 2), np.float32)
    lib.ffref_bvh_trace(hb, p(br), len(br), p(bh), 0, 8)
    out.update(bvh_rays=br, bvh_hits=bh)

    # ---- material texture reads (get_albedo / get_roughness / get_metallic /
    # get_normal): random textures, materials with random slots, intersections
    # with random texcoords (wrapping) and orthonormal-ish frames
    srng = np.random.default_rng(777)
    ntex = 6
    stex = [srng.uniform(0.0, 1.0, (int(srng.integers(2, 9)), int(srng.integers(2, 9)), 3)).astype(np.float32)
            for _ in range(ntex - 1)]
    stex.append(scenes.normal_texture(16, seed=5))
    tex_ids = [lib.ffref_tex_create(p(np.ascontiguousarray(t)), t.shape[1], t.shape[0], 3) for t in stex]
    ns = 400
    smat = np.zeros((ns, 8), np.float32)
    smat[:, 0:3] = srng.uniform(0.1, 0.9, (ns, 3))
    smat[:, 3:6] = 0.04
    smat[:, 6] = srng.uniform(0.05, 1.0, ns)
    smat[:, 7] = srng.uniform(0.0, 1.0, ns)
    sslots = np.where(srng.uniform(size=(ns, 5)) < 0.5, srng.integers(0, ntex - 1, (ns, 5)), -1).astype(np.int32)
    sslots[:, 4] = np.where(srng.uniform(size=ns) < 0.6, ntex - 1, -1)   # normal slot: the normal texture
    sisect = np.zeros((ns, 11), np.float32)
    sisect[:, 0:2] = srng.uniform(-0.5, 1.5, (ns, 2))
    nrm = unit(srng, ns)
    tan = unit(srng, ns)
    tan = tan - nrm * (tan * nrm).sum(1, keepdims=True)
    tan /= np.linalg.norm(tan, axis=1, keepdims=True)
    sisect[:, 2:5], sisect[:, 5:8], sisect[:, 8:11] = nrm, tan, np.cross(nrm, tan)
    sout = np.zeros((ns, 8), np.float32)
    for i in range(ns):
        ids = np.array([tex_ids[k] if k >= 0 else -1 for k in sslots[i]], np.int32)
        lib.ffref_surface(p(smat[i]), p(ids), p(sisect[i]), p(sout[i]))
    out.update(surf_mat=smat, surf_slots=sslots, surf_isect=sisect, surf_out=sout,
               **{f"surf_tex{k}": t for k, t in enumerate(stex)})

    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e6:.2f} MB)")


if __name__ == "__main__":
    main()
