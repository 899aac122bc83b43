"""Writes tests/golden/room_pbr.glb, the committed glTF fixture of the import
tests (tests/test_gltf_cpu.py, tests/test_render_gpu.py).

The scene is scenes.pbr_textured_room(seed=3, tex_res=16) -- the room open to
the sky with a base-colour, a packed metallic-roughness and a normal texture
on the walls and floor, a conductor sphere with the normal texture -- whose
texels are replaced by integer formulas of (x, y), so that every decoded
texel has a known value: texel (x, y) of texture k (row y counted from the
top of the image file) is FORMULAS[k](x, y) / 255.  The file is written with
firefly_b200.gltf.save (PNG, 8 bits per channel).

Usage: python tests/golden/make_gltf_fixture.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

RES = 16


def formula_bytes(k: int) -> np.ndarray:
    """uint8 (RES, RES, 3) image of texture k, row 0 = the image file's top row."""
    y, x = np.meshgrid(np.arange(RES), np.arange(RES), indexing="ij")
    if k == 0:      # base colour
        c = [(37 * x + 11 * y + 20) % 256, (13 * x + 71 * y + 90) % 256, (x * y * 7 + 40) % 256]
    elif k == 1:    # metallic-roughness: x unused, roughness y in [30, 250], metallic z in {0, 255}
        c = [np.zeros_like(x), 30 + (17 * x + 29 * y) % 221, np.where((x + y) % 3 == 0, 255, 0)]
    else:           # tangent-space normal: z dominant
        c = [128 + (x - RES // 2) * 5, 128 + (y - RES // 2) * 5, np.full_like(x, 235)]
    return np.stack(c, -1).astype(np.uint8)


def main() -> None:
    from firefly_b200 import gltf, scenes
    scn = scenes.pbr_textured_room(seed=3, width=48, height=48, tex_res=RES)
    # gltf.save writes texture rows flipped back (the loader flips them as
    # stb does): a scene texture is the file image upside down
    scn.textures = [(formula_bytes(k)[::-1].astype(np.float32) / 255.0) for k in range(3)]
    scn.materials[1].roughness_tex = -1
    scn.materials[1].metallic_tex = -1
    gltf.save(HERE / "room_pbr.glb", scn)
    print(HERE / "room_pbr.glb")


if __name__ == "__main__":
    main()
