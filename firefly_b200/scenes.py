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
    env_rgb: np.ndarray | None = None
    env_color: tuple = (0.0, 0.0, 0.0)
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


def material(base_color, kind=A.FF_MAT_MIX, roughness=1.0, metallic=0.0, ior=1.5, fresnel=0.04,
             emissive=(0, 0, 0), radiance=0.0) -> A.ff_material:
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
    m.base_color_tex = -1
    m.roughness_tex = -1
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
