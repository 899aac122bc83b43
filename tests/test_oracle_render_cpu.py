"""The oracle's full render (its restatement of the reference's stages in
plain C) against the reference's own path tracer compiled for the host
(oracle/_ref: the reference's BVH, materials, lights and sampler routines,
with the wf_* stage logic restated in the harness).  The host-compiled
reference draws from a free-running clock, so the two are compared as
estimators of the same image: per-pixel means at 1024 spp."""
import numpy as np
import pytest

from firefly_b200 import scenes
from tests.conftest import cpu_threads


def test_oracle_render_agrees_with_host_compiled_reference(oracle):
    from oracle import ffref
    if not ffref.available():
        pytest.skip("oracle/_ref was not built (no reference checkout)")
    W = H = 24
    spp = 1024
    scn = scenes.small_room(seed=0, width=W, height=H)
    ref, (re, rs, rn), _ = ffref.render(scn, W, H, spp, max_depth=5, rr_depth=3, light=0, threads=cpu_threads(),
                                         want_image=True)
    ours, (oe, os_) = oracle.render(scn, W, H, spp, max_depth=5, rr_depth=3, seed=7, mode=0, light=0,
                                    threads=cpu_threads())
    ref = ref.astype(np.float64) / spp
    ours = ours.astype(np.float64) / spp
    ok = np.isfinite(ref).all(-1) & np.isfinite(ours).all(-1)
    assert ok.mean() > 0.99
    rel_mean = abs(ours[ok].mean() - ref[ok].mean()) / ref[ok].mean()
    # two independent 1024-spp estimates: per-pixel relative squared differences
    rel = ((ours[ok] - ref[ok]) ** 2 / (ref[ok] ** 2 + 1e-2)).mean()
    print(f"[oracle] render vs host-compiled reference: mean {ours[ok].mean():.4f} vs {ref[ok].mean():.4f} "
          f"(rel {rel_mean:.4f}), relMSE {rel:.2e}; rays {oe}+{os_} vs {re}+{rs}")
    assert rel_mean < 0.01
    assert rel < 5e-3
    # same ray budget per sample to within the noise of the path lengths
    assert abs(oe / re - 1) < 0.02 and abs(os_ / rs - 1) < 0.02
