"""glTF 2.0 import (the scene-import step of the reference's Scene::load):
a round trip through .glb, node transforms (TRS and matrices) applied to
positions and normals, generated normals, flipped texture v, cameras, image
textures and tangent frames."""
import base64
import json
import math

import numpy as np

from firefly_b200 import gltf, scenes

ROOT = __import__("pathlib").Path(__file__).resolve().parent.parent


def _tri_set(P, I):
    return sorted(tuple(np.round(P[t].ravel(), 5)) for t in I)


def test_glb_round_trip(tmp_path):
    scn = scenes.small_room(seed=0, width=64, height=64)
    p = tmp_path / "room.glb"
    gltf.save(p, scn)
    got = gltf.load(p, 64, 64)
    assert got.num_triangles == scn.num_triangles
    assert _tri_set(got.positions, got.indices) == _tri_set(scn.positions, scn.indices)
    # material factors and the per-triangle assignment survive
    for m_src, m_got in zip(scn.materials, got.materials):
        assert np.allclose(list(m_src.base_color), list(m_got.base_color))
        assert m_src.roughness == m_got.roughness
    src_by_tri = {tuple(np.round(scn.positions[t].ravel(), 5)): m for t, m in zip(scn.indices, scn.material_ids)}
    for t, m in zip(got.indices, got.material_ids):
        assert src_by_tri[tuple(np.round(got.positions[t].ravel(), 5))] == m
    assert np.allclose(np.linalg.norm(got.normals, axis=1), 1.0, atol=1e-5)


def test_gltf_node_transforms_normals_uvs_camera(tmp_path):
    P = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    UV = np.array([[0, 0], [1, 0], [0, 1]], np.float32)
    I = np.array([0, 1, 2], np.uint16)
    blob = P.tobytes() + UV.tobytes() + I.tobytes() + b"\0\0"
    uri = "data:application/octet-stream;base64," + base64.b64encode(blob).decode()
    c = math.sqrt(0.5)
    doc = {
        "asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": [0, 2]}],
        "nodes": [{"translation": [1, 2, 3], "children": [1]},
                  {"rotation": [0, 0, c, c], "scale": [2, 2, 2], "mesh": 0},
                  {"matrix": [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 1, 10, 1], "camera": 0}],
        "cameras": [{"type": "perspective", "perspective": {"yfov": 0.8, "znear": 0.1, "zfar": 100}}],
        "meshes": [{"primitives": [{"attributes": {"POSITION": 0, "TEXCOORD_0": 1}, "indices": 2}]}],
        "buffers": [{"byteLength": len(blob), "uri": uri}],
        "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": 36},
                        {"buffer": 0, "byteOffset": 36, "byteLength": 24},
                        {"buffer": 0, "byteOffset": 60, "byteLength": 6}],
        "accessors": [{"bufferView": 0, "componentType": 5126, "count": 3, "type": "VEC3"},
                      {"bufferView": 1, "componentType": 5126, "count": 3, "type": "VEC2"},
                      {"bufferView": 2, "componentType": 5123, "count": 3, "type": "SCALAR"}],
    }
    p = tmp_path / "tri.gltf"
    p.write_text(json.dumps(doc))
    s = gltf.load(p, 32, 32)
    # scale 2, 90 degrees about z, then + (1, 2, 3)
    want = np.array([[1, 2, 3], [1, 4, 3], [-1, 2, 3]], np.float32)
    assert np.allclose(s.positions, want, atol=1e-5)
    assert np.allclose(s.normals, [[0, 0, 1]] * 3, atol=1e-6)          # generated, area-weighted
    assert np.allclose(s.texcoords, [[0, 1], [1, 1], [0, 0]])           # v flipped
    assert s.material_ids.tolist() == [0] and len(s.materials) == 1     # the default material
    assert s.camera is not None
    rays = scenes.camera_rays(s, 32, 32).reshape(32, 32, 8)
    assert np.allclose(rays[16, 16, :3], [0, 1, 10], atol=0.2)          # camera at (0, 1, 10) looking down -z
    assert rays[16, 16, 6] < -0.99


def _quantised_pbr_room():
    scn = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=32)
    # 8-bit texels, so that the PNG round trip is exact
    scn.textures = [(np.round(np.clip(t, 0.0, 1.0) * 255.0) / 255.0).astype(np.float32) for t in scn.textures]
    for m in scn.materials:       # single-channel textures have no core glTF slot
        m.roughness_tex = -1
        m.metallic_tex = -1
    return scn


def test_glb_textures_and_tangents_round_trip(tmp_path):
    scn = _quantised_pbr_room()
    p = tmp_path / "pbr.glb"
    gltf.save(p, scn)
    got = gltf.load(p, 48, 48)
    for m_src, m_got in zip(scn.materials, got.materials):
        for slot in ("base_color_tex", "metallic_roughness_tex", "normal_tex"):
            a, b = getattr(m_src, slot), getattr(m_got, slot)
            assert (a < 0) == (b < 0), slot
            if a >= 0:
                assert np.array_equal(scn.textures[a], got.textures[b]), slot
    V = len(scn.positions)
    used = np.unique(scn.indices)
    # every primitive repeats the vertex arrays; the first copy maps 1:1
    assert np.abs(got.tangents[:V][used] - scn.tangents[used]).max() < 1e-6
    assert np.abs(got.bitangents[:V][used] - scn.bitangents[used]).max() < 1e-6


def test_gltf_external_png_rows_and_scaling(tmp_path):
    """An image file referenced by uri: texel values byte / 255, rows stored
    bottom-up as the reference's loader flips them, so that with the flipped
    texture v the image's top row is read at glTF v = 0."""
    from PIL import Image
    h, w = 4, 3
    img = np.zeros((h, w, 3), np.uint8)
    img[..., 0] = np.arange(h)[:, None] * 60          # red grows down the image
    img[..., 1] = np.arange(w)[None, :] * 100         # green grows to the right
    img[..., 2] = 255
    Image.fromarray(img, "RGB").save(tmp_path / "t.png")
    P = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    uv = np.array([[0, 0], [1, 0], [0, 1]], np.float32)
    blob = P.tobytes() + uv.tobytes()
    doc = {"asset": {"version": "2.0"}, "scenes": [{"nodes": [0]}], "nodes": [{"mesh": 0}],
           "meshes": [{"primitives": [{"attributes": {"POSITION": 0, "TEXCOORD_0": 1}, "material": 0}]}],
           "materials": [{"pbrMetallicRoughness": {"baseColorTexture": {"index": 0}}}],
           "textures": [{"source": 0}], "images": [{"uri": "t.png"}],
           "buffers": [{"byteLength": len(blob), "uri": "data:application/octet-stream;base64,"
                        + base64.b64encode(blob).decode()}],
           "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": 36},
                           {"buffer": 0, "byteOffset": 36, "byteLength": 24}],
           "accessors": [{"bufferView": 0, "componentType": 5126, "count": 3, "type": "VEC3"},
                         {"bufferView": 1, "componentType": 5126, "count": 3, "type": "VEC2"}]}
    (tmp_path / "s.gltf").write_text(json.dumps(doc))
    got = gltf.load(tmp_path / "s.gltf", 8, 8)
    assert got.materials[0].base_color_tex == 0
    tex = got.textures[0]
    assert tex.shape == (h, w, 3) and tex.dtype == np.float32
    assert np.array_equal(tex, (img[::-1] / 255.0).astype(np.float32))
    # the flipped v of the first vertex (glTF v = 0) is 1: the top image row sits at texture row h - 1
    assert got.texcoords[0, 1] == 1.0


def test_committed_fixture_decodes_to_known_texels():
    """tests/golden/room_pbr.glb (made by tests/golden/make_gltf_fixture.py)
    holds textures whose texels are integer formulas of (x, y): the import
    must give exactly formula / 255 with the rows flipped as the reference's
    loader flips them (stbi_set_flip_vertically_on_load, dTexture.cu:115-117),
    the material slots of the file, and its geometry."""
    from firefly_b200 import gltf
    from tests.golden.make_gltf_fixture import formula_bytes
    scn = gltf.load(ROOT / "tests" / "golden" / "room_pbr.glb", 48, 48)
    assert len(scn.textures) == 3
    for k in range(3):
        want = formula_bytes(k)[::-1].astype(np.float32) / 255.0
        assert np.array_equal(scn.textures[k], want), k
    m0 = scn.materials[0]
    assert (m0.base_color_tex, m0.metallic_roughness_tex, m0.normal_tex) == (0, 1, 2)
    assert scn.num_triangles == 4116
    assert scn.tangents is not None and np.isfinite(scn.tangents).all()
