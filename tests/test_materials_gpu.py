"""GPU parity of the material kinds without a reference counterpart: the
rough GGX dielectric (Walter et al. 2007; refraction into and out of
objects, with two-sided closest hits for rays inside them) and the diffuse
base under a GGX coat, against the oracle's restatement (oracle/ffo_render.c)
with the same per-pixel sampler seeds.  Tolerance: mean relative error
<= 1e-4 of the per-pixel mean radiance, and the same ray counts to 1e-3 (the
same paths were traced).
"""
from __future__ import annotations

import numpy as np
import pytest

from firefly_b200 import scenes
from tests.conftest import cpu_threads
from tests.test_render_gpu import MRE_TOL, _parity

pytestmark = pytest.mark.gpu


def _room_with_sphere(kind, seed, w, h, roughness, albedo=(0.9, 0.95, 1.0), ior=1.5):
    scn = scenes.small_room(seed=seed, width=w, height=h)
    scn.materials[1] = scenes.material(albedo, kind=kind, roughness=roughness, ior=ior)
    return scn


@pytest.mark.parametrize("roughness", [0.1, 0.45])
@pytest.mark.parametrize("mode", [0, 1])
def test_dielectric_sphere_parity(ctx, oracle, mode, roughness):
    import firefly_b200 as ff
    scn = _room_with_sphere(ff.FF_MAT_DIELECTRIC, 0, 64, 64, roughness)
    got, ref, stats, mre = _parity(ctx, oracle, scn, 64, 64, 8, max_depth=8, rr_depth=3, seed=3, mode=mode)
    assert (ref.sum(-1) > 0).mean() > 0.5


def test_coat_sphere_parity(ctx, oracle):
    import firefly_b200 as ff
    for mode in (0, 1):
        scn = _room_with_sphere(ff.FF_MAT_COAT, 1, 48, 48, 0.3, albedo=(0.7, 0.3, 0.2))
        _parity(ctx, oracle, scn, 48, 48, 6, max_depth=6, seed=4, mode=mode)


def test_dielectric_ior_and_tint(ctx, oracle):
    """Another index (water) and a coloured transmission, under the room's
    light and a directional light chosen per vertex."""
    import firefly_b200 as ff
    scn = _room_with_sphere(ff.FF_MAT_DIELECTRIC, 2, 48, 48, 0.25, albedo=(1.0, 0.6, 0.3), ior=1.33)
    scn.directional_lights = [scenes.directional_light((0.3, 1.0, 0.2), radiance=2.0)]
    _parity(ctx, oracle, scn, 48, 48, 6, max_depth=8, seed=5, mode=ff.FF_MODE_CORRECTED, light=ff.FF_LIGHT_ALL)


def test_reduced_at_scale_scene_parity(ctx, oracle):
    """The at-scale scene reduced (icosphere subdivided 4x: 5,132 triangles
    with the room, 32 materials of all five kinds, 256 x 128 sky with the
    sun) at 160 x 90, 4 spp, depth 8, corrected mode, against the oracle."""
    import firefly_b200 as ff
    scn = scenes.displaced_icosphere(subdiv=4, width=160, height=90, env_w=256, env_h=128)
    kinds = {int(m.kind) for m in scn.materials}
    assert kinds == {0, 1, 2, 3, 4}
    got, ref, stats, mre = _parity(ctx, oracle, scn, 160, 90, 4, light=-1, max_depth=8, rr_depth=3, seed=0,
                                   mode=ff.FF_MODE_CORRECTED)
    assert np.all(np.isfinite(got)) and got.min() >= 0.0
