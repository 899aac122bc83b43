"""glTF 2.0 scene import (JSON .gltf with external or data-URI buffers, or
binary .glb) into a firefly_b200.scenes.Scene.

Replaces the reference's assimp import (CUDA-RayTracer/Scene.cpp:20-221:
Scene::load walks the node tree accumulating transforms, load_mesh reads
positions, normals, texture coordinates and indices with
aiProcess_Triangulate | aiProcess_GenSmoothNormals | aiProcess_FlipUVs, and
materials keep the glTF metallic-roughness factors, dScene.cpp:82-214).
Here: triangle primitives (mode 4) of every mesh instanced by the default
scene's nodes, with node matrices or TRS composed root to leaf; positions
transformed by the node matrix and normals by its inverse transpose;
missing normals generated as area-weighted vertex normals; texture
coordinates flipped in v (1 - v) as aiProcess_FlipUVs does; one material per
glTF material (base colour, roughness and metallic factors, and the base
colour, metallic-roughness and normal textures, Scene.cpp:206-212); tangent
frames from TANGENT attributes (bitangent = cross(N, T) * w); the first
perspective camera found becomes the scene camera.

Images (PNG, JPEG: whatever PIL decodes) become float RGB textures of
byte / 255 (16-bit images / 65535), rows flipped as the reference's loader
flips them (stbi_set_flip_vertically_on_load, dTexture.cu:115-117; with the
uv flip the two cancel).  A texture replaces its factor, as the reference's
get_* functions read it (dMaterial.cu:10-60); no sRGB decoding is applied
(the reference's loader applies none).  The reference decodes with
stb_image, which is not in its checkout: the decoded values are not pinned.
"""
from __future__ import annotations

import base64
import json
import math
import struct
from pathlib import Path

import numpy as np

from . import _abi as A
from . import scenes

_COMPONENT = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_NCOMP = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT4": 16}


def _load(path: Path):
    data = path.read_bytes()
    if data[:4] == b"glTF":
        version, length = struct.unpack_from("<II", data, 4)
        if version != 2:
            raise ValueError(f"unsupported glb version {version}")
        off, doc, bin_chunk = 12, None, None
        while off < length:
            clen, ctype = struct.unpack_from("<II", data, off)
            chunk = data[off + 8:off + 8 + clen]
            if ctype == 0x4E4F534A:
                doc = json.loads(chunk.decode("utf-8"))
            elif ctype == 0x004E4942:
                bin_chunk = chunk
            off += 8 + clen
        if doc is None:
            raise ValueError("glb without a JSON chunk")
        return doc, bin_chunk
    return json.loads(data.decode("utf-8")), None


def _buffers(doc, base: Path, bin_chunk):
    out = []
    for i, b in enumerate(doc.get("buffers", [])):
        uri = b.get("uri")
        if uri is None:
            if bin_chunk is None:
                raise ValueError(f"buffer {i} has no uri and there is no binary chunk")
            out.append(bin_chunk)
        elif uri.startswith("data:"):
            out.append(base64.b64decode(uri.split(",", 1)[1]))
        else:
            out.append((base / uri).read_bytes())
    return out


def _accessor(doc, bufs, idx: int) -> np.ndarray:
    acc = doc["accessors"][idx]
    dtype = np.dtype(_COMPONENT[acc["componentType"]])
    n = _NCOMP[acc["type"]]
    count = acc["count"]
    if "bufferView" not in acc:
        return np.zeros((count, n), dtype)
    bv = doc["bufferViews"][acc["bufferView"]]
    buf = bufs[bv["buffer"]]
    start = bv.get("byteOffset", 0) + acc.get("byteOffset", 0)
    stride = bv.get("byteStride", 0) or dtype.itemsize * n
    raw = np.frombuffer(buf, np.uint8, count=(count - 1) * stride + dtype.itemsize * n, offset=start)
    rows = np.lib.stride_tricks.as_strided(raw, shape=(count, dtype.itemsize * n), strides=(stride, 1))
    out = np.ascontiguousarray(rows).view(dtype).reshape(count, n)
    if acc.get("normalized") and dtype.kind in "iu":
        out = out.astype(np.float32) / float(np.iinfo(dtype).max)
    return out


def _node_matrix(node) -> np.ndarray:
    if "matrix" in node:
        return np.asarray(node["matrix"], np.float64).reshape(4, 4).T   # column-major in the file
    t = np.asarray(node.get("translation", [0, 0, 0]), np.float64)
    x, y, z, w = node.get("rotation", [0, 0, 0, 1])
    s = np.asarray(node.get("scale", [1, 1, 1]), np.float64)
    r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    m = np.eye(4)
    m[:3, :3] = r * s[None, :]
    m[:3, 3] = t
    return m


def _smooth_normals(P: np.ndarray, I: np.ndarray) -> np.ndarray:
    tri = P[I].astype(np.float64)
    fn = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])      # area-weighted
    N = np.zeros_like(P, dtype=np.float64)
    for k in range(3):
        np.add.at(N, I[:, k], fn)
    ln = np.linalg.norm(N, axis=1, keepdims=True)
    return (N / np.where(ln > 0, ln, 1.0)).astype(np.float32)


def _image(doc, bufs, base: Path, idx: int) -> np.ndarray:
    """Image idx decoded to float32 (h, w, 3), rows flipped as stb flips them."""
    import io

    from PIL import Image
    img = doc["images"][idx]
    if "bufferView" in img:
        bv = doc["bufferViews"][img["bufferView"]]
        raw = bufs[bv["buffer"]][bv.get("byteOffset", 0):bv.get("byteOffset", 0) + bv["byteLength"]]
    elif img.get("uri", "").startswith("data:"):
        raw = base64.b64decode(img["uri"].split(",", 1)[1])
    else:
        raw = (base / img["uri"]).read_bytes()
    im = Image.open(io.BytesIO(raw))
    a = np.asarray(im)
    scale = 65535.0 if a.dtype == np.uint16 or im.mode.startswith("I;16") else 255.0
    a = a.astype(np.float64) / scale
    if a.ndim == 2:
        a = np.repeat(a[..., None], 3, -1)
    elif a.shape[2] == 2:            # luminance + alpha
        a = np.repeat(a[..., :1], 3, -1)
    a = a[..., :3]
    return np.ascontiguousarray(a[::-1]).astype(np.float32)


def load(path, width: int = 512, height: int = 512, kind=A.FF_MAT_MIX) -> scenes.Scene:
    """A scenes.Scene from a glTF 2.0 file (lights come from the caller)."""
    path = Path(path)
    doc, bin_chunk = _load(path)
    bufs = _buffers(doc, path.parent, bin_chunk)
    textures, tex_slot = [], {}

    def slot(info):
        """Scene texture index of a glTF textureInfo, -1 when absent."""
        if not info or "index" not in info:
            return -1
        src = doc["textures"][info["index"]].get("source")
        if src is None:
            return -1
        if src not in tex_slot:
            tex_slot[src] = len(textures)
            textures.append(_image(doc, bufs, path.parent, src))
        return tex_slot[src]

    mats = []
    for m in doc.get("materials", []):
        pbr = m.get("pbrMetallicRoughness", {})
        bc = pbr.get("baseColorFactor", [1, 1, 1, 1])
        mats.append(scenes.material(bc[:3], kind=kind, roughness=float(pbr.get("roughnessFactor", 1.0)),
                                    metallic=float(pbr.get("metallicFactor", 1.0)),
                                    base_color_tex=slot(pbr.get("baseColorTexture")),
                                    metallic_roughness_tex=slot(pbr.get("metallicRoughnessTexture")),
                                    normal_tex=slot(m.get("normalTexture"))))
    default_mat = len(mats)
    mats.append(scenes.material((0.8, 0.8, 0.8), kind=kind))
    Ps, Ns, UVs, Is, Ms, Ts, Bs, Ls = [], [], [], [], [], [], [], []
    any_tangents = False
    base = 0
    camera = None
    scene_idx = doc.get("scene", 0)
    roots = doc["scenes"][scene_idx]["nodes"] if doc.get("scenes") else list(range(len(doc.get("nodes", []))))
    stack = [(r, np.eye(4)) for r in reversed(roots)]
    while stack:
        ni, parent = stack.pop()
        node = doc["nodes"][ni]
        M = parent @ _node_matrix(node)
        for c in reversed(node.get("children", [])):
            stack.append((c, M))
        if "camera" in node and camera is None:
            cam = doc["cameras"][node["camera"]]
            if cam.get("type") == "perspective":
                p = cam["perspective"]
                eye = M[:3, 3]
                fwd = -M[:3, 2] / np.linalg.norm(M[:3, 2])
                up = M[:3, 1] / np.linalg.norm(M[:3, 1])
                camera = scenes.make_camera(eye=tuple(eye), center=tuple(eye + fwd), up=tuple(up),
                                            fovy=math.degrees(p["yfov"]), aspect=width / height,
                                            near=p.get("znear", 0.01), far=p.get("zfar", 1000.0))
        if "mesh" not in node:
            continue
        nrm_m = np.linalg.inv(M[:3, :3]).T
        for prim in doc["meshes"][node["mesh"]]["primitives"]:
            if prim.get("mode", 4) != 4:
                continue
            at = prim["attributes"]
            P = _accessor(doc, bufs, at["POSITION"]).astype(np.float64)
            I = (_accessor(doc, bufs, prim["indices"]).reshape(-1).astype(np.int64) if "indices" in prim
                 else np.arange(len(P), dtype=np.int64))
            I = I.reshape(-1, 3)
            Pw = (P @ M[:3, :3].T + M[:3, 3]).astype(np.float32)
            if "NORMAL" in at:
                N = _accessor(doc, bufs, at["NORMAL"]).astype(np.float64) @ nrm_m.T
                N /= np.maximum(np.linalg.norm(N, axis=1, keepdims=True), 1e-30)
                N = N.astype(np.float32)
            else:
                N = _smooth_normals(Pw, I)
            if "TEXCOORD_0" in at:
                UV = _accessor(doc, bufs, at["TEXCOORD_0"]).astype(np.float32).copy()
                UV[:, 1] = 1.0 - UV[:, 1]                       # aiProcess_FlipUVs
            else:
                UV = np.zeros((len(P), 2), np.float32)
            if "TANGENT" in at:
                T4 = _accessor(doc, bufs, at["TANGENT"]).astype(np.float64)
                T = T4[:, :3] @ M[:3, :3].T
                T /= np.maximum(np.linalg.norm(T, axis=1, keepdims=True), 1e-30)
                B = np.cross(N.astype(np.float64), T) * np.where(T4[:, 3:4] < 0.0, -1.0, 1.0)
                Ts.append(T.astype(np.float32))
                Bs.append(B.astype(np.float32))
                any_tangents = True
            else:
                Ts.append(None)
                Bs.append(None)
            Ps.append(Pw)
            Ns.append(N)
            UVs.append(UV)
            Is.append(I + base)
            Ls.append(I)
            Ms.append(np.full(len(I), prim.get("material", default_mat), np.uint32))
            base += len(P)
    if not Ps:
        raise ValueError("the glTF scene has no triangle primitives")
    tangents = bitangents = None
    if any_tangents:
        # primitives without TANGENT get the uv-derived frame
        for k in range(len(Ts)):
            if Ts[k] is None:
                Ts[k], Bs[k] = scenes.vertex_tangents(Ps[k], Ls[k], UVs[k], Ns[k])
        tangents, bitangents = np.concatenate(Ts), np.concatenate(Bs)
    return scenes.Scene(positions=np.concatenate(Ps), indices=np.concatenate(Is).astype(np.uint32),
                        normals=np.concatenate(Ns), texcoords=np.concatenate(UVs),
                        material_ids=np.concatenate(Ms), materials=mats, camera=camera, width=width, height=height,
                        textures=textures, tangents=tangents, bitangents=bitangents)


def save(path, scene: scenes.Scene):
    """Write the scene's mesh, tangent frame, material factors and its base
    colour, metallic-roughness and normal textures (PNG, 8 bits per channel)
    as a .glb (one node, one mesh, one primitive per material): the inverse of
    load() for tests and for exporting procedural scenes.  Single-channel
    roughness and metallic textures have no core glTF slot and are left out."""
    path = Path(path)
    blobs, views, accessors, prims = [], [], [], []

    def add(arr: np.ndarray, comp: int, typ: str, target=None, minmax=False):
        raw = np.ascontiguousarray(arr).tobytes()
        off = sum(len(b) for b in blobs)
        pad = (-len(raw)) % 4
        blobs.append(raw + b"\0" * pad)
        v = {"buffer": 0, "byteOffset": off, "byteLength": len(raw)}
        if target:
            v["target"] = target
        views.append(v)
        a = {"bufferView": len(views) - 1, "componentType": comp, "count": int(arr.shape[0]), "type": typ}
        if minmax:
            a["min"] = [float(x) for x in arr.min(0)]
            a["max"] = [float(x) for x in arr.max(0)]
        accessors.append(a)
        return len(accessors) - 1

    pos = add(scene.positions.astype(np.float32), 5126, "VEC3", 34962, True)
    attrs = {"POSITION": pos}
    if scene.normals is not None:
        attrs["NORMAL"] = add(scene.normals.astype(np.float32), 5126, "VEC3", 34962)
    if scene.texcoords is not None:
        uv = scene.texcoords.astype(np.float32).copy()
        uv[:, 1] = 1.0 - uv[:, 1]
        attrs["TEXCOORD_0"] = add(uv, 5126, "VEC2", 34962)
    if getattr(scene, "tangents", None) is not None and scene.normals is not None:
        T = np.asarray(scene.tangents, np.float64)
        w = np.where((np.cross(np.asarray(scene.normals, np.float64), T) * np.asarray(scene.bitangents, np.float64))
                     .sum(1, keepdims=True) < 0.0, -1.0, 1.0)
        attrs["TANGENT"] = add(np.concatenate([T, w], 1).astype(np.float32), 5126, "VEC4", 34962)
    mids = scene.material_ids if scene.material_ids is not None else np.zeros(scene.num_triangles, np.uint32)
    for m in np.unique(mids):
        idx = scene.indices[mids == m].reshape(-1).astype(np.uint32)
        prims.append({"attributes": attrs, "indices": add(idx, 5125, "SCALAR", 34963), "material": int(m), "mode": 4})
    images, textures, img_of = [], [], {}

    def tex_ref(k):
        """glTF textureInfo for scene texture k (PNG of round(255 t), rows
        flipped back), or None."""
        if k < 0:
            return None
        if k not in img_of:
            import io

            from PIL import Image
            t = np.clip(np.asarray(scene.textures[k], np.float64)[::-1], 0.0, 1.0)
            buf = io.BytesIO()
            Image.fromarray(np.round(t * 255.0).astype(np.uint8), "RGB").save(buf, format="PNG")
            raw = buf.getvalue()
            off = sum(len(b) for b in blobs)
            blobs.append(raw + b"\0" * ((-len(raw)) % 4))
            views.append({"buffer": 0, "byteOffset": off, "byteLength": len(raw)})
            images.append({"bufferView": len(views) - 1, "mimeType": "image/png"})
            textures.append({"source": len(images) - 1})
            img_of[k] = len(textures) - 1
        return {"index": img_of[k]}

    mats = []
    for m in scene.materials:
        pbr = {"baseColorFactor": [float(m.base_color[0]), float(m.base_color[1]), float(m.base_color[2]), 1.0],
               "roughnessFactor": float(m.roughness), "metallicFactor": float(m.metallic)}
        if tex_ref(m.base_color_tex):
            pbr["baseColorTexture"] = tex_ref(m.base_color_tex)
        if tex_ref(m.metallic_roughness_tex):
            pbr["metallicRoughnessTexture"] = tex_ref(m.metallic_roughness_tex)
        mat = {"pbrMetallicRoughness": pbr}
        if tex_ref(m.normal_tex):
            mat["normalTexture"] = tex_ref(m.normal_tex)
        mats.append(mat)
    binary = b"".join(blobs)
    doc = {"asset": {"version": "2.0", "generator": "firefly_b200.gltf"}, "scene": 0, "scenes": [{"nodes": [0]}],
           "nodes": [{"mesh": 0}], "meshes": [{"primitives": prims}], "materials": mats,
           "buffers": [{"byteLength": len(binary)}], "bufferViews": views, "accessors": accessors}
    if images:
        doc["images"], doc["textures"] = images, textures
    js = json.dumps(doc).encode("utf-8")
    js += b" " * ((-len(js)) % 4)
    out = struct.pack("<III", 0x46546C67, 2, 12 + 8 + len(js) + 8 + len(binary))
    out += struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(binary), 0x004E4942) + binary
    path.write_bytes(out)
