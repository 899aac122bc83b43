"""Headless image output: PNG and PFM writers round-trip."""
import numpy as np

from firefly_b200 import image


def test_png_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    for c in (3, 4):
        img = rng.integers(0, 256, (17, 23, c), dtype=np.uint8)
        image.write_png(tmp_path / f"a{c}.png", img)
        assert np.array_equal(image.read_png(tmp_path / f"a{c}.png"), img)


def test_pfm_round_trip(tmp_path):
    img = np.random.default_rng(1).normal(size=(9, 13, 3)).astype(np.float32)
    image.write_pfm(tmp_path / "a.pfm", img)
    assert np.array_equal(image.read_pfm(tmp_path / "a.pfm"), img)
