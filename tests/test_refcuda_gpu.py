"""The reference's own GPU traversal (CUDA-RayTracer/dTriangle.cu's
intersect / intersect_shadows, built unmodified for sm_100a by
`make -C oracle refcuda`) against ff_trace on the same rays.  The reference's
device build contracts its float dot and cross products into FMAs (nvcc's
default), so a ray whose hit lies within rounding of a triangle edge can
land on the neighbour; everything else must agree."""
import numpy as np
import pytest

from firefly_b200 import scenes

pytestmark = pytest.mark.gpu


def test_reference_gpu_traversal_agrees(ctx):
    from oracle import ffrefcuda
    if not ffrefcuda.available():
        pytest.skip("oracle/_ref/libffrefcuda.so was not built")
    import firefly_b200 as ff
    scn = scenes.small_room(seed=0)
    ds = ff.dScene(ctx, scn)
    bvh = ffrefcuda.RefGpuBVH(scn.triangle_soup())
    cam = scenes.camera_rays(scn, 256, 256)
    inc = scenes.incoherent_rays(scn, 1 << 16, seed=3)
    for name, rays in (("camera", cam), ("incoherent", inc)):
        ours = ds.trace(rays)
        t, prim, ms = bvh.trace(rays)
        same = ours["prim"] == prim
        frac = float(same.mean())
        dt = np.abs(ours["t"][same & (prim >= 0)] - t[same & (prim >= 0)])
        rel = float((dt / np.maximum(t[same & (prim >= 0)], 1e-30)).max()) if dt.size else 0.0
        print(f"[refcuda] {name}: {len(rays)} rays, ids agree {frac:.6f}, max rel t diff {rel:.2e}, "
              f"{len(rays) / (ms / 1e3) / 1e6:.1f} Mrays/s")
        assert frac > 0.999
        assert rel < 1e-5
    rays = scenes.with_random_tmax(inc, scn, seed=4)
    occ_ours = ds.trace(rays, any_hit=True)["prim"] >= 0
    _, occ, _ = bvh.trace(rays, any_hit=True)
    frac = float(np.mean(occ_ours == (occ > 0)))
    print(f"[refcuda] any-hit: agree {frac:.6f}")
    assert frac > 0.999
    bvh.close()
    ds.close()
