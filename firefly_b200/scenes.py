"""Procedural scenes and ray sets of the benchmark workloads (numpy, seeded).

The reference's own scenes are glTF files loaded through assimp
(CUDA-RayTracer/Scene.cpp:20-65); they are not part of the hot path and the
workloads here are procedural instead:

* ``small_room``: a closed box of 12 quads (24 triangles) around a UV sphere
  of 64 x 32 segments (4,096 triangles, the pole quads degenerate) at a seeded
  centre and radius, one rectangular area light of radiance 15, albedos
  uniform in [0.2, 0.8] per object.  4,120 triangles.
* ``displaced_icosphere``: an icosphere subdivided 8 times (1,310,720
  triangles) displaced by 4-octave value noise inside a 12-triangle room,
  triangles grouped into 4 material classes by a seeded 3D noise, and a
  synthetic 2048 x 1024 equirectangular sky with a sun disc.
* ray sets for the trace micro-benchmark: coherent pinhole camera rays and
  incoherent rays (origins uniform in the scene box, directions uniform on
  the sphere), closest-hit and any-hit with tmax ~ U[0.1, 10] x diagonal.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A


# ----------------------------------------------------------------- camera
def look_at(eye, center, up) -> np.ndarray:
    """Right-handed view matrix (OpenGL convention), row-major math matrix."""
    eye, center, up = (np.asarray(v, np.float64) for v in (eye, center, up))
    f = center - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = s, u, -f
    m[0, 3], m[1, 3], m[2, 3] = -s @ eye, -u @ eye, f @ eye
    return m


def perspective(fovy_deg: float, aspect: float, near: float, far: float) -> np.ndarray:
    """OpenGL perspective projection (clip z in [-1, 1]), row-major math matrix."""
    t = math.tan(math.radians(fovy_deg) / 2)
    m = np.zeros((4, 4))
    m[0, 0] = 1 / (aspect * t)
    m[1, 1] = 1 / t
    m[2, 2] = -(far + near) / (far - near)
    m[2, 3] = -2 * far * near / (far - near)
    m[3, 2] = -1
    return m


def make_camera(eye, center, up=(0, 1, 0), fovy=45.0, aspect=1.0, near=0.1, far=100.0,
                lens_radius=0.0, focal_distance=1.0, exposure=1.0, pixel_jitter=0.005) -> A.ff_camera:
    """ff_camera with inv_view_proj[4*i + j] = (row j, column i) of inverse(P V),
    the column-major order the reference's Matrix4x4 m[i][j] holds."""
    inv = np.linalg.inv(perspective(fovy, aspect, near, far) @ look_at(eye, center, up))
    cam = A.ff_camera()
    flat = inv.T.astype(np.float32).ravel()
    for k in range(16):
        cam.inv_view_proj[k] = float(flat[k])
    cam.lens_radius = lens_radius
    cam.focal_distance = focal_distance
    cam.exposure = exposure
    cam.pixel_jitter = pixel_jitter
    return cam


# ------------------------------------------------------------------ meshes
def box_room(lo, hi, inward=True):
    """Closed box of 12 quads (each face split in two), 24 triangles, wound so
    that the geometric normal e1 x e2 points into the box (front faces seen
    from inside under the reference's culling test)."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    P, I = [], []

    def quad(a, b, c, d):
        base = len(P)
        P.extend([a, b, c, d])
        if inward:
            I.extend([[base, base + 1, base + 2], [base, base + 2, base + 3]])
        else:
            I.extend([[base, base + 2, base + 1], [base, base + 3, base + 2]])

    x0, y0, z0 = lo
    x1, y1, z1 = hi
    xm, ym, zm = (lo + hi) / 2
    # floor (y = y0), normal +y: ccw seen from above
    quad([x0, y0, z0], [x0, y0, zm], [x1, y0, zm], [x1, y0, z0])
    quad([x0, y0, zm], [x0, y0, z1], [x1, y0, z1], [x1, y0, zm])
    # ceiling (y = y1), normal -y
    quad([x0, y1, z0], [x1, y1, z0], [x1, y1, zm], [x0, y1, zm])
    quad([x0, y1, zm], [x1, y1, zm], [x1, y1, z1], [x0, y1, z1])
    # wall x = x0, normal +x
    quad([x0, y0, z0], [x0, y1, z0], [x0, y1, zm], [x0, y0, zm])
    quad([x0, y0, zm], [x0, y1, zm], [x0, y1, z1], [x0, y0, z1])
    # wall x = x1, normal -x
    quad([x1, y0, z0], [x1, y0, zm], [x1, y1, zm], [x1, y1, z0])
    quad([x1, y0, zm], [x1, y0, z1], [x1, y1, z1], [x1, y1, zm])
    # wall z = z0, normal +z
    quad([x0, y0, z0], [x1, y0, z0], [x1, ym, z0], [x0, ym, z0])
    quad([x0, ym, z0], [x1, ym, z0], [x1, y1, z0], [x0, y1, z0])
    # wall z = z1, normal -z
    quad([x0, y0, z1], [x0, ym, z1], [x1, ym, z1], [x1, y0, z1])
    quad([x0, ym, z1], [x0, y1, z1], [x1, y1, z1], [x1, ym, z1])
    P = np.asarray(P, np.float32)
    I = np.asarray(I, np.uint32)
    # verify the winding once: normals must point toward the centre
    c = (lo + hi) / 2
    tri = P[I]
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    toc = c - tri.mean(axis=1)
    sgn = np.sign((n * toc).sum(1))
    assert np.all(sgn == (1 if inward else -1))
    return P, I


def uv_sphere(center, radius, seg_u=64, seg_v=32):
    """UV sphere of seg_u x seg_v quads, two triangles each (the pole quads
    keep a degenerate triangle), wound outward; per-vertex normals."""
    center = np.asarray(center, np.float64)
    th = np.linspace(0, math.pi, seg_v + 1)          # polar
    ph = np.linspace(0, 2 * math.pi, seg_u + 1)      # azimuth
    T, PH = np.meshgrid(th, ph, indexing="ij")       # (seg_v+1, seg_u+1)
    n = np.stack([np.sin(T) * np.cos(PH), np.cos(T), np.sin(T) * np.sin(PH)], -1)
    P = (center + radius * n).reshape(-1, 3).astype(np.float32)
    N = n.reshape(-1, 3).astype(np.float32)
    idx = []
    W = seg_u + 1
    for i in range(seg_v):
        for j in range(seg_u):
            a = i * W + j
            b = a + 1
            c = a + W
            d = c + 1
            idx.append([a, b, d])
            idx.append([a, d, c])
    I = np.asarray(idx, np.uint32)
    # orient outward
    tri = P[I].astype(np.float64)
    nn = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    out = tri.mean(1) - center
    flip = (nn * out).sum(1) < 0
    I[flip] = I[flip][:, [0, 2, 1]]
    return P, I, N


@dataclass
class Scene:
    positions: np.ndarray
    indices: np.ndarray
    normals: np.ndarray | None = None
    texcoords: np.ndarray | None = None
    material_ids: np.ndarray | None = None
    materials: list = field(default_factory=list)
    area_lights: list = field(default_factory=list)
    directional_lights: list = field(default_factory=list)   # light indices after the area lights
    env_rgb: np.ndarray | None = None
    env_color: tuple = (0.0, 0.0, 0.0)
    textures: list = field(default_factory=list)   # (h, w, 3) float32 arrays, indexed by ff_material.*_tex
    tangents: np.ndarray | None = None     # (V, 3) per-vertex tangent frame for normal textures, or None
    bitangents: np.ndarray | None = None
    camera: A.ff_camera | None = None
    width: int = 256
    height: int = 256

    @property
    def num_triangles(self) -> int:
        return int(self.indices.shape[0])

    def triangle_soup(self) -> np.ndarray:
        """(T, 9) float32 v0 v1 v2 per triangle, in the caller's order."""
        return np.ascontiguousarray(self.positions[self.indices].reshape(-1, 9), dtype=np.float32)

    def bounds(self):
        return self.positions.min(0), self.positions.max(0)


def directional_light(direction, emissive=(1.0, 1.0, 1.0), radiance=1.0) -> A.ff_directional_light:
    """A directional light shining from `direction` (toward the light)."""
    L = A.ff_directional_light()
    for k in range(3):
        L.direction[k] = float(direction[k])
        L.emissive[k] = float(emissive[k])
    L.radiance = float(radiance)
    return L


def material(base_color, kind=A.FF_MAT_MIX, roughness=1.0, metallic=0.0, ior=1.5, fresnel=0.04,
             emissive=(0, 0, 0), radiance=0.0, base_color_tex=-1, roughness_tex=-1, metallic_tex=-1,
             metallic_roughness_tex=-1, normal_tex=-1) -> A.ff_material:
    m = A.ff_material()
    for k in range(3):
        m.base_color[k] = float(base_color[k])
        m.emissive[k] = float(emissive[k])
        m.fresnel[k] = float(fresnel)
    m.roughness = roughness
    m.metallic = metallic
    m.radiance = radiance
    m.ior = ior
    m.kind = kind
    m.base_color_tex = base_color_tex
    m.roughness_tex = roughness_tex
    m.metallic_tex = metallic_tex
    m.metallic_roughness_tex = metallic_roughness_tex
    m.normal_tex = normal_tex
    return m


def area_light(p0, a, b, normal, radiance=15.0, emissive=(1, 1, 1)) -> A.ff_area_light:
    L = A.ff_area_light()
    for k in range(3):
        L.p0[k], L.a[k], L.b[k], L.normal[k], L.emissive[k] = p0[k], a[k], b[k], normal[k], emissive[k]
    L.radiance = radiance
    return L


def small_room(seed: int = 0, width: int = 256, height: int = 256, kind=A.FF_MAT_MIX,
               lens_radius: float = 0.0) -> Scene:
    """The plain-tracer room: 24-triangle box, 4,096-triangle UV sphere, one area light."""
    rng = np.random.default_rng(seed)
    lo, hi = np.array([-5, 0, -5], np.float32), np.array([5, 10, 5], np.float32)
    rP, rI = box_room(lo, hi)
    radius = float(rng.uniform(1.0, 2.0))
    center = np.array([rng.uniform(-2.5, 2.5), rng.uniform(radius + 0.5, 5.0), rng.uniform(-2.5, 2.5)])
    sP, sI, sN = uv_sphere(center, radius)
    tri = rP[rI].astype(np.float64)
    rn = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    rn /= np.linalg.norm(rn, axis=1, keepdims=True)
    # room vertices are not shared between faces: per-vertex normal = face normal
    rN = np.zeros_like(rP)
    for t, (i0, i1, i2) in enumerate(rI):
        rN[[i0, i1, i2]] = rn[t]
    P = np.concatenate([rP, sP]).astype(np.float32)
    N = np.concatenate([rN, sN]).astype(np.float32)
    I = np.concatenate([rI, sI + len(rP)]).astype(np.uint32)
    mat_ids = np.concatenate([np.zeros(len(rI), np.uint32), np.ones(len(sI), np.uint32)])
    albedo = rng.uniform(0.2, 0.8, size=(2, 3))
    mats = [material(albedo[0], kind=kind), material(albedo[1], kind=kind)]
    light = area_light(p0=(-1.0, 9.99, -1.0), a=(2.0, 0.0, 0.0), b=(0.0, 0.0, 2.0), normal=(0.0, -1.0, 0.0),
                       radiance=15.0)
    cam = make_camera(eye=(0.0, 5.0, 4.9), center=(center[0], center[1], center[2]), fovy=60.0,
                      aspect=width / height, near=0.05, far=50.0, lens_radius=lens_radius)
    return Scene(positions=P, indices=I, normals=N, material_ids=mat_ids, materials=mats, area_lights=[light],
                 env_color=(0.0, 0.0, 0.0), camera=cam, width=width, height=height)


# -------------------------------------------------------------- ray sets
def camera_rays(scene: Scene, width: int, height: int) -> np.ndarray:
    """Coherent primary rays through pixel centres of a pinhole camera
    (n x 8 float32, ff_ray layout), computed in float64 then rounded."""
    inv = np.asarray(scene.camera.inv_view_proj, np.float64).reshape(4, 4).T  # math matrix
    ys, xs = np.meshgrid(np.arange(height, dtype=np.float64), np.arange(width, dtype=np.float64), indexing="ij")
    nx = 2.0 * ((xs + 0.5) / width) - 1.0
    ny = 1.0 - 2.0 * ((ys + 0.5) / height)
    def unproject(z):
        v = np.stack([nx, ny, np.full_like(nx, z), np.ones_like(nx)], -1) @ inv.T
        return v[..., :3] / v[..., 3:]
    pn, pf = unproject(-1.0), unproject(1.0)
    d = pf - pn
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    rays = np.zeros((height * width, 8), np.float32)
    rays[:, 0:3] = pn.reshape(-1, 3)
    rays[:, 3] = 0.0
    rays[:, 4:7] = d.reshape(-1, 3)
    rays[:, 7] = np.inf
    return rays


def incoherent_rays(scene: Scene, n: int, seed: int = 1) -> np.ndarray:
    """Origins uniform in the scene box, directions uniform on the sphere."""
    rng = np.random.default_rng(seed)
    lo, hi = scene.bounds()
    o = rng.uniform(lo, hi, size=(n, 3))
    z = 1.0 - 2.0 * rng.random(n)
    phi = 2.0 * math.pi * rng.random(n)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], -1)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def with_random_tmax(rays: np.ndarray, scene: Scene, seed: int = 2) -> np.ndarray:
    """Any-hit variant: tmax ~ U[0.1, 10] x scene diagonal."""
    rng = np.random.default_rng(seed)
    lo, hi = scene.bounds()
    diag = float(np.linalg.norm(hi.astype(np.float64) - lo))
    out = rays.copy()
    out[:, 7] = (rng.uniform(0.1, 10.0, size=len(rays)) * diag).astype(np.float32)
    return out


# ------------------------------------------------------- environment maps
def sky_env(width: int = 2048, height: int = 1024, seed: int = 0, sun_dir=(0.35, 0.8, 0.25),
            sun_radiance: float = 5e4, sun_diameter_deg: float = 0.5) -> np.ndarray:
    """Synthetic equirectangular sky, (height, width, 3) float32, row y at v = y/height.

    A vertical gradient (zenith blue to a bright horizon, darker ground) times
    log-normal(0, 0.5) per-texel noise, plus a sun disc of the given angular
    diameter and radiance.  Texel directions follow the reference's
    spherical mapping: u = atan2(z, x)/2pi + 0.5, v = asin(y)/pi + 0.5."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    U, Vv = np.meshgrid(u, v)
    phi = (U - 0.5) * 2 * math.pi
    lat = (Vv - 0.5) * math.pi
    dy = np.sin(lat)
    dx = np.cos(lat) * np.cos(phi)
    dz = np.cos(lat) * np.sin(phi)
    t = np.clip(dy, -1, 1)
    zenith = np.array([0.25, 0.45, 0.95])
    horizon = np.array([0.9, 0.9, 1.0])
    ground = np.array([0.25, 0.22, 0.2])
    up = np.clip(t, 0, 1)[..., None]
    sky = np.where(t[..., None] >= 0, horizon * (1 - up) + zenith * up, ground * (0.5 + 0.5 * (1 + t[..., None])))
    noise = rng.lognormal(0.0, 0.5, size=(height, width, 1))
    img = sky * noise
    s = np.asarray(sun_dir, np.float64)
    s /= np.linalg.norm(s)
    cosang = dx * s[0] + dy * s[1] + dz * s[2]
    half = math.radians(sun_diameter_deg) / 2
    # at least the texel nearest the sun direction lights up, so the sun survives any resolution
    disc = cosang >= math.cos(half)
    su = math.atan2(s[2], s[0]) / (2 * math.pi) + 0.5
    sv = math.asin(s[1]) / math.pi + 0.5
    disc[min(height - 1, int(sv * height)), min(width - 1, int(su * width))] = True
    img[disc] = sun_radiance
    return img.astype(np.float32)


def sphere_under_sky(seed: int = 0, width: int = 64, height: int = 64, env_w: int = 128, env_h: int = 64,
                     kind=A.FF_MAT_MIX) -> Scene:
    """Open scene for the environment light: a ground quad and a UV sphere
    under a synthetic sky."""
    rng = np.random.default_rng(seed)
    gP = np.array([[-20, 0, -20], [-20, 0, 20], [20, 0, 20], [20, 0, -20]], np.float32)
    gI = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    gN = np.tile(np.array([0, 1, 0], np.float32), (4, 1))
    radius = float(rng.uniform(1.0, 1.5))
    sP, sI, sN = uv_sphere((0.0, radius, 0.0), radius, seg_u=32, seg_v=16)
    P = np.concatenate([gP, sP])
    N = np.concatenate([gN, sN])
    I = np.concatenate([gI, sI + len(gP)]).astype(np.uint32)
    mat_ids = np.concatenate([np.zeros(len(gI), np.uint32), np.ones(len(sI), np.uint32)])
    albedo = rng.uniform(0.2, 0.8, size=(2, 3))
    mats = [material(albedo[0], kind=kind, roughness=0.8), material(albedo[1], kind=kind, roughness=0.5)]
    cam = make_camera(eye=(0.0, 2.5, 6.0), center=(0.0, radius, 0.0), fovy=50.0, aspect=width / height,
                      near=0.05, far=100.0)
    env = sky_env(env_w, env_h, seed=seed, sun_radiance=200.0, sun_diameter_deg=4.0)
    return Scene(positions=P.astype(np.float32), indices=I, normals=N.astype(np.float32), material_ids=mat_ids,
                 materials=mats, env_rgb=env, camera=cam, width=width, height=height)


# ----------------------------------------------------- at-scale workload
def icosphere(subdiv: int):
    """Unit icosphere: 20 * 4^subdiv triangles, outward winding."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    V = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(subdiv):
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * len(V) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // len(V), uniq % len(V)
        mid = V[a] + V[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(V)
        V = np.concatenate([V, mid])
        nf = len(F)
        m01, m12, m20 = inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base
        F = np.concatenate([np.stack([F[:, 0], m01, m20], 1), np.stack([F[:, 1], m12, m01], 1),
                            np.stack([F[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return V, F


def value_noise3(p: np.ndarray, seed: int, octaves: int = 4) -> np.ndarray:
    """Fractal value noise in [-1, 1]: lattice values hashed from integer
    coordinates, smoothstep-interpolated, octaves at doubling frequency and
    halving amplitude."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1.0, 1.0, size=256)
    perm = rng.permutation(256)

    def lattice(ix, iy, iz):
        h = perm[(perm[(perm[ix & 255] + iy) & 255] + iz) & 255]
        return table[h]

    total = np.zeros(len(p))
    amp, freq, norm = 1.0, 1.0, 0.0
    for _ in range(octaves):
        q = p * freq
        i = np.floor(q).astype(np.int64)
        f = q - i
        s = f * f * (3 - 2 * f)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = ((s[:, 0] if dx else 1 - s[:, 0]) * (s[:, 1] if dy else 1 - s[:, 1]) *
                         (s[:, 2] if dz else 1 - s[:, 2]))
                    acc += w * lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def displaced_icosphere(subdiv: int = 8, seed: int = 0, width: int = 1920, height: int = 1080,
                        env_w: int = 2048, env_h: int = 1024) -> Scene:
    """The at-scale workload: an icosphere subdivided `subdiv` times (8 ->
    1,310,720 triangles) displaced radially by 4-octave value noise of
    amplitude 0.1 x radius, inside a 12-triangle room (floor, four walls and
    half a ceiling, open to the sky over the other half), triangles grouped by
    a seeded 3D noise into 4 material classes (diffuse, GGX conductor with
    roughness U[0.05, 0.6], thin GGX dielectric of IOR 1.5, diffuse under a
    GGX coat), a 2048 x 1024 sky with a 0.5 degree sun of radiance 5e4."""
    rng = np.random.default_rng(seed)
    V, F = icosphere(subdiv)
    radius, center = 2.0, np.array([0.0, 2.4, 0.0])
    disp = value_noise3(V * 2.0 + 10.0, seed + 1, octaves=4)
    Pv = center + V * (radius * (1.0 + 0.1 * disp))[:, None]
    # vertex normals of the displaced surface (area-weighted face normals)
    tri = Pv[F]
    fn = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    Nv = np.zeros_like(Pv)
    for k in range(3):
        np.add.at(Nv, F[:, k], fn)
    Nv /= np.linalg.norm(Nv, axis=1, keepdims=True)
    # room: 12 triangles (floor, four walls, half a ceiling), normals inward
    lo, hi = np.array([-8.0, 0.0, -8.0]), np.array([8.0, 9.0, 8.0])
    room_tris, room_P = [], []

    def quad(a, b, c, d):
        base = len(room_P)
        room_P.extend([a, b, c, d])
        room_tris.extend([[base, base + 1, base + 2], [base, base + 2, base + 3]])

    x0, y0, z0 = lo
    x1, y1, z1 = hi
    quad([x0, y0, z0], [x0, y0, z1], [x1, y0, z1], [x1, y0, z0])          # floor, normal +y
    quad([x0, y0, z0], [x0, y1, z0], [x0, y1, z1], [x0, y0, z1])          # x = x0, normal +x
    quad([x1, y0, z0], [x1, y0, z1], [x1, y1, z1], [x1, y1, z0])          # x = x1, normal -x
    quad([x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0])          # z = z0, normal +z
    quad([x0, y0, z1], [x0, y1, z1], [x1, y1, z1], [x1, y0, z1])          # z = z1, normal -z
    quad([x0, y1, 0.0], [x1, y1, 0.0], [x1, y1, z1], [x0, y1, z1])        # ceiling over z > 0, normal -y
    rP = np.asarray(room_P, np.float64)
    rI = np.asarray(room_tris, np.int64)
    rt = rP[rI]
    rn = np.cross(rt[:, 1] - rt[:, 0], rt[:, 2] - rt[:, 0])
    rn /= np.linalg.norm(rn, axis=1, keepdims=True)
    inward = ((lo + hi) / 2 - rt.mean(1)) * rn
    assert np.all(inward.sum(1) > 0), "room triangles must face inward"
    rN = np.zeros_like(rP)
    for t_, (i0, i1, i2) in enumerate(rI):
        rN[[i0, i1, i2]] = rn[t_]
    P = np.concatenate([rP, Pv]).astype(np.float32)
    N = np.concatenate([rN, Nv]).astype(np.float32)
    I = np.concatenate([rI, F + len(rP)]).astype(np.uint32)
    # materials: 0 = room (the reference's mix material); classes 1..4 x 8 variants
    mats = [material((0.7, 0.7, 0.68), kind=A.FF_MAT_MIX, roughness=0.9)]
    kinds = [A.FF_MAT_DIFFUSE, A.FF_MAT_CONDUCTOR, A.FF_MAT_DIELECTRIC, A.FF_MAT_COAT]
    variants = 8
    for kd in kinds:
        for _ in range(variants):
            alb = rng.uniform(0.2, 0.9, 3)
            if kd == A.FF_MAT_DIFFUSE:
                mats.append(material(alb, kind=kd, roughness=1.0))
            elif kd == A.FF_MAT_CONDUCTOR:
                mats.append(material(alb, kind=kd, roughness=float(rng.uniform(0.05, 0.6)), metallic=1.0))
            elif kd == A.FF_MAT_DIELECTRIC:
                mats.append(material((0.95, 0.97, 1.0), kind=kd, roughness=float(rng.uniform(0.05, 0.3)), ior=1.5))
            else:
                mats.append(material(alb, kind=kd, roughness=float(rng.uniform(0.05, 0.3)), ior=1.5))
    cen = Pv[F].mean(axis=1)
    cls_noise = value_noise3(cen * 1.5 + 3.0, seed + 2, octaves=2)
    q = np.quantile(cls_noise, [0.25, 0.5, 0.75])
    cls = np.searchsorted(q, cls_noise)
    var = (np.arange(len(F)) * 2654435761 % 2**32 >> 16) % variants
    sphere_mat = 1 + cls * variants + var
    mat_ids = np.concatenate([np.zeros(len(rI), np.uint32), sphere_mat.astype(np.uint32)])
    cam = make_camera(eye=(0.0, 3.2, 7.4), center=(0.0, 2.2, 0.0), fovy=50.0, aspect=width / height,
                      near=0.05, far=100.0)
    env = sky_env(env_w, env_h, seed=seed)
    return Scene(positions=P, indices=I, normals=N, material_ids=mat_ids, materials=mats, env_rgb=env,
                 camera=cam, width=width, height=height)


def perlin2(res: int, seed: int, octaves: int = 5, base: int = 4) -> np.ndarray:
    """Seeded 2D gradient (Perlin) noise fBm on a res x res grid, in [-1, 1] roughly."""
    rng = np.random.default_rng(seed)
    out = np.zeros((res, res))
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = base * 2 ** o
        ang = rng.uniform(0, 2 * math.pi, size=(cells + 1, cells + 1))
        gx, gy = np.cos(ang), np.sin(ang)
        t = (np.arange(res) + 0.5) / res * cells
        i0 = np.floor(t).astype(int)
        f = t - i0
        fy, fx = np.meshgrid(f, f, indexing="ij")
        iy, ix = np.meshgrid(i0, i0, indexing="ij")

        def dotg(dy, dx):
            return gx[iy + dy, ix + dx] * (fx - dx) + gy[iy + dy, ix + dx] * (fy - dy)
        sx = fx * fx * fx * (fx * (fx * 6 - 15) + 10)
        sy = fy * fy * fy * (fy * (fy * 6 - 15) + 10)
        n0 = dotg(0, 0) * (1 - sx) + dotg(0, 1) * sx
        n1 = dotg(1, 0) * (1 - sx) + dotg(1, 1) * sx
        out += amp * (n0 * (1 - sy) + n1 * sy)
        total += amp
        amp *= 0.5
    return out / total * 1.5


def albedo_texture(res: int = 512, seed: int = 0) -> np.ndarray:
    """Seeded Perlin RGB albedo in [0.1, 0.9], (res, res, 3) float32."""
    ch = [np.clip(0.5 + 0.4 * perlin2(res, seed * 3 + c), 0.1, 0.9) for c in range(3)]
    return np.stack(ch, -1).astype(np.float32)


def roughness_texture(res: int = 512, seed: int = 0, lo: float = 0.1, hi: float = 0.6) -> np.ndarray:
    """Seeded Perlin roughness in [lo, hi], (res, res, 3) float32; a
    material's roughness_tex reads channel 0 (the three channels are equal)."""
    r = np.clip(0.5 * (lo + hi) + 0.5 * (hi - lo) * perlin2(res, seed * 3 + 101), lo, hi)
    return np.repeat(r[..., None], 3, -1).astype(np.float32)


def textured_room(seed: int = 0, width: int = 512, height: int = 512, albedo=None, env=None, tex_res: int = 512,
                  env_w: int = 256, env_h: int = 128, kind=A.FF_MAT_DIFFUSE, sphere_kind=None,
                  roughness=None, sphere_metallic: float = 1.0, packed: bool = False) -> Scene:
    """The small room opened to the sky (no ceiling) for inverse rendering:
    floor, walls and sphere carry one albedo texture (texture 0); the
    environment map lights the room.  `albedo` (res, res, 3) and `env`
    (env_h, env_w, 3) default to the hidden parameters: a seeded Perlin
    albedo in [0.1, 0.9] and a synthetic sky.

    With `sphere_kind` (a GGX kind: FF_MAT_MIX, CONDUCTOR, DIELECTRIC, COAT)
    the sphere gets its own material of that kind, base colour 0.8 and
    metallic `sphere_metallic`, whose roughness reads texture 1:
    `roughness` (res, res, 3), by default a seeded Perlin roughness in
    [0.1, 0.6].  With `packed` texture 1 is instead the sphere's glTF
    metallic-roughness texture: channel x zero, y the roughness, z
    `sphere_metallic`."""
    rng = np.random.default_rng(seed)
    lo, hi = np.array([-5, 0, -5], np.float32), np.array([5, 10, 5], np.float32)
    rP, rI = box_room(lo, hi)
    keep = [0, 1, 4, 5, 6, 7, 8, 9, 10, 11]          # quads of box_room without the ceiling (2, 3)
    tri_keep = np.concatenate([[2 * q, 2 * q + 1] for q in keep])
    rI = rI[tri_keep]
    # per-face uv: project on the two axes spanning each quad
    rUV = np.zeros((len(rP), 2), np.float32)
    for q in keep:
        vs = np.unique(rI[2 * keep.index(q):2 * keep.index(q) + 2].ravel())
        p = rP[vs]
        span = p.max(0) - p.min(0)
        axes = np.argsort(-span)[:2]
        rUV[vs] = (p[:, axes] - lo[axes]) / (hi[axes] - lo[axes])
    tri = rP[rI].astype(np.float64)
    rn = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    rn /= np.linalg.norm(rn, axis=1, keepdims=True)
    rN = np.zeros_like(rP)
    for t, (i0, i1, i2) in enumerate(rI):
        rN[[i0, i1, i2]] = rn[t]
    radius = float(rng.uniform(1.0, 2.0))
    center = np.array([rng.uniform(-2.5, 2.5), rng.uniform(radius + 0.5, 5.0), rng.uniform(-2.5, 2.5)])
    sP, sI, sN = uv_sphere(center, radius)
    d = (sP - center) / radius
    sUV = np.stack([np.arctan2(d[:, 2], d[:, 0]) / (2 * math.pi) + 0.5, np.arccos(np.clip(d[:, 1], -1, 1)) / math.pi],
                   -1).astype(np.float32)
    P = np.concatenate([rP, sP]).astype(np.float32)
    N = np.concatenate([rN, sN]).astype(np.float32)
    UV = np.concatenate([rUV, sUV]).astype(np.float32)
    I = np.concatenate([rI, sI + len(rP)]).astype(np.uint32)
    mat_ids = np.zeros(len(I), np.uint32)
    mats = [material((0.5, 0.5, 0.5), kind=kind, roughness=1.0, base_color_tex=0)]
    tex = albedo_texture(tex_res, seed) if albedo is None else np.asarray(albedo, np.float32)
    textures = [tex]
    if sphere_kind is not None:
        mat_ids[len(rI):] = 1
        rough = roughness_texture(tex_res, seed) if roughness is None else np.asarray(roughness, np.float32)
        if packed:
            rough = np.stack([np.zeros_like(rough[..., 0]), rough[..., 0],
                              np.full_like(rough[..., 0], sphere_metallic)], -1).astype(np.float32)
        mats.append(material((0.8, 0.8, 0.8), kind=sphere_kind, roughness=0.5, metallic=sphere_metallic,
                             roughness_tex=-1 if packed else 1, metallic_roughness_tex=1 if packed else -1))
        textures.append(rough)
    sky = sky_env(env_w, env_h, seed=seed, sun_radiance=300.0, sun_diameter_deg=6.0) if env is None else env
    cam = make_camera(eye=(0.0, 8.0, 4.9), center=(center[0], center[1], center[2]), fovy=70.0, aspect=width / height,
                      near=0.05, far=60.0)
    return Scene(positions=P, indices=I, normals=N, texcoords=UV, material_ids=mat_ids, materials=mats,
                 env_rgb=np.asarray(sky, np.float32), textures=textures, camera=cam, width=width, height=height)


def vertex_tangents(positions, indices, texcoords, normals):
    """Per-vertex tangent frame for normal textures: per triangle, dP/du and
    dP/dv from the uv differences of its edges, summed at its vertices, then
    made orthogonal to the vertex normal (Gram-Schmidt) and normalised; the
    bitangent keeps the sign of dP/dv.  Returns (tangents, bitangents), both
    (V, 3) float32."""
    P = np.asarray(positions, np.float64)
    I = np.asarray(indices, np.int64)
    UV = np.asarray(texcoords, np.float64)
    N = np.asarray(normals, np.float64).copy()
    # vertices no triangle uses may carry a zero normal: any unit normal does
    N[np.linalg.norm(N, axis=1) < 1e-12] = (0.0, 0.0, 1.0)
    e1, e2 = P[I[:, 1]] - P[I[:, 0]], P[I[:, 2]] - P[I[:, 0]]
    d1, d2 = UV[I[:, 1]] - UV[I[:, 0]], UV[I[:, 2]] - UV[I[:, 0]]
    det = d1[:, 0] * d2[:, 1] - d2[:, 0] * d1[:, 1]
    r = np.where(np.abs(det) > 1e-20, 1.0 / np.where(det == 0, 1.0, det), 0.0)[:, None]
    T = (e1 * d2[:, 1:2] - e2 * d1[:, 1:2]) * r
    B = (e2 * d1[:, 0:1] - e1 * d2[:, 0:1]) * r
    Tv, Bv = np.zeros_like(P), np.zeros_like(P)
    for k in range(3):
        np.add.at(Tv, I[:, k], T)
        np.add.at(Bv, I[:, k], B)
    Tv -= N * (Tv * N).sum(1, keepdims=True)
    # vertices without a uv gradient (poles, degenerate mappings): any tangent
    bad = np.linalg.norm(Tv, axis=1) < 1e-12
    alt = np.where(np.abs(N[:, :1]) > 0.5, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    Tv[bad] = np.cross(N[bad], alt[bad])
    Tv /= np.linalg.norm(Tv, axis=1, keepdims=True)
    Bn = np.cross(N, Tv)
    sign = np.where((Bn * Bv).sum(1, keepdims=True) < 0.0, -1.0, 1.0)
    return Tv.astype(np.float32), (Bn * sign).astype(np.float32)


def normal_texture(res: int = 64, seed: int = 0, strength: float = 0.6) -> np.ndarray:
    """Tangent-space normal texture of a seeded bump field, stored as
    0.5 + 0.5 * n (the usual 8-bit-style encoding), (res, res, 3) float32."""
    h = perlin2(res, seed * 7 + 3)
    gy, gx = np.gradient(h * res * strength / 8.0)
    n = np.stack([-gx, -gy, np.ones_like(h)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    return (0.5 + 0.5 * n).astype(np.float32)


def pbr_textured_room(seed: int = 0, width: int = 64, height: int = 64, tex_res: int = 64, env=None,
                      derive_tangents: bool = False) -> Scene:
    """The room open to the sky with every material texture kind:
    walls and floor FF_MAT_MIX with a base-colour texture (0), a packed
    metallic-roughness texture (1: roughness in y, metallic in z) and a normal
    texture (2); the sphere a GGX conductor with a roughness texture (3), a
    metallic texture (4) and the normal texture.  Per-vertex tangents come with
    the scene unless derive_tangents (the library then derives them)."""
    base = textured_room(seed=seed, width=width, height=height, tex_res=tex_res, env=env, env_w=64, env_h=32,
                         sphere_kind=A.FF_MAT_CONDUCTOR)
    rng = np.random.default_rng(seed + 17)
    rough = np.clip(0.35 + 0.25 * perlin2(tex_res, seed * 5 + 11), 0.05, 0.9)
    metal = np.clip(0.5 + 0.5 * perlin2(tex_res, seed * 5 + 12), 0.0, 1.0)
    mr = np.stack([np.zeros_like(rough), rough, metal], -1).astype(np.float32)
    nt = normal_texture(tex_res, seed)
    r1 = np.repeat(np.clip(0.2 + 0.3 * perlin2(tex_res, seed * 5 + 13), 0.05, 0.9)[..., None], 3, -1)
    m1 = np.repeat(np.clip(0.7 + 0.3 * perlin2(tex_res, seed * 5 + 14), 0.0, 1.0)[..., None], 3, -1)
    mats = [material((0.5, 0.5, 0.5), kind=A.FF_MAT_MIX, roughness=1.0, base_color_tex=0,
                     metallic_roughness_tex=1, normal_tex=2),
            material(tuple(rng.uniform(0.5, 0.9, 3)), kind=A.FF_MAT_CONDUCTOR, roughness=0.5, metallic=1.0,
                     roughness_tex=3, metallic_tex=4, normal_tex=2)]
    scn = Scene(positions=base.positions, indices=base.indices, normals=base.normals, texcoords=base.texcoords,
                material_ids=base.material_ids, materials=mats, env_rgb=base.env_rgb,
                textures=[base.textures[0], mr, nt, r1.astype(np.float32), m1.astype(np.float32)],
                camera=base.camera, width=width, height=height)
    if not derive_tangents:
        scn.tangents, scn.bitangents = vertex_tangents(scn.positions, scn.indices, scn.texcoords, scn.normals)
    return scn
