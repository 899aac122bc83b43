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


def _rgbe_to_float(rgbe):
    e = rgbe[..., 3].astype(np.int32)
    s = np.where(e > 0, np.ldexp(np.float32(1.0), e - 136), np.float32(0.0)).astype(np.float32)
    return rgbe[..., :3].astype(np.float32) * s[..., None]


def test_hdr_round_trip_and_orientation(tmp_path):
    from firefly_b200 import image
    rng = np.random.default_rng(0)
    rgbe = rng.integers(0, 256, (5, 9, 4)).astype(np.uint8)
    rgbe[..., 3] = rng.integers(120, 140, (5, 9))
    rgbe[0, 0, 3] = 0                                    # an exponent of 0 decodes to black
    # a float image that RGBE represents exactly: the largest channel carries the exponent
    rgbe[..., 0] = np.maximum(rgbe[..., 0], 128)
    rgbe[..., 1:3] = np.minimum(rgbe[..., 1:3], rgbe[..., :1])
    want = _rgbe_to_float(rgbe)[::-1]                    # row 0 = the file's bottom row
    image.write_hdr(tmp_path / "a.hdr", want)
    got = image.read_hdr(tmp_path / "a.hdr")
    assert got.dtype == np.float32 and got.shape == (5, 9, 3)
    assert np.array_equal(got, want)


def _rle_channel(vals):
    # runs of equal bytes (length >= 3) as run packets, the rest as literals
    out, i, n = bytearray(), 0, len(vals)
    while i < n:
        j = i
        while j < n and vals[j] == vals[i] and j - i < 127:
            j += 1
        if j - i >= 3:
            out += bytes([128 + (j - i), vals[i]])
            i = j
        else:
            k = i
            while k < n and k - i < 128 and not (k + 2 < n and vals[k] == vals[k + 1] == vals[k + 2]):
                k += 1
            k = max(k, i + 1)
            out += bytes([k - i]) + bytes(vals[i:k])
            i = k
    return bytes(out)


def test_hdr_run_length_scanlines(tmp_path):
    """New-style run-length scanlines (2, 2, w >> 8, w & 255, then each of the
    four channels as runs and literals) decode like the flat file."""
    from firefly_b200 import image
    rng = np.random.default_rng(1)
    h, w = 4, 40
    rgbe = rng.integers(0, 256, (h, w, 4)).astype(np.uint8)
    rgbe[:, 10:30, :] = rgbe[:, 10:11, :]                # long runs
    rgbe[..., 3] = rng.integers(125, 135)
    body = bytearray()
    for y in range(h):
        body += bytes([2, 2, w >> 8, w & 255])
        for c in range(4):
            body += _rle_channel(list(rgbe[y, :, c]))
    head = f"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y {h} +X {w}\n".encode()
    (tmp_path / "r.hdr").write_bytes(head + bytes(body))
    (tmp_path / "f.hdr").write_bytes(head + rgbe.tobytes())
    a, b = image.read_hdr(tmp_path / "r.hdr"), image.read_hdr(tmp_path / "f.hdr")
    assert np.array_equal(a, b)
    assert np.array_equal(a, _rgbe_to_float(rgbe)[::-1])


def test_reference_environment_maps_decode():
    """The reference's own environment maps (hrdi/*.hdr, run-length encoded)
    decode: the sky's upper half, at the end of the rows, outshines its
    lower half."""
    import pytest

    from firefly_b200 import image
    from oracle import REF_DIR
    d = REF_DIR.parent / "hrdi"
    if not d.is_dir():
        pytest.skip("reference checkout not present")
    for f in sorted(d.glob("*.hdr")):
        a = image.read_hdr(f)
        assert a.ndim == 3 and a.shape[2] == 3 and a.shape[1] == 2 * a.shape[0]
        assert np.isfinite(a).all() and a.min() >= 0.0 and a.max() > 1.0
    sky = image.read_hdr(d / "HDR_029_Sky_Cloudy_Env.hdr")
    assert sky[sky.shape[0] // 2:].mean() > 2 * sky[:sky.shape[0] // 2].mean()
