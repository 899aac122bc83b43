"""Headless image output, in place of the reference's GL display surface
(wf_logic writes the tonemapped char4 into a GL texture, CUDA-RayTracer/
kernel.cu:447-454): 8-bit PNG of ff_film_tonemap's RGBA and float PFM of the
mean radiance, with standard-library encoders only.  Also the Radiance .hdr
environment maps the reference loads with stb_image (load_texture_float,
dTexture.cu:188-196): read_hdr / write_hdr."""
from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np


def write_png(path, rgba8: np.ndarray):
    """(h, w, 4) or (h, w, 3) uint8 -> PNG (colour type 6 or 2, no filter)."""
    img = np.ascontiguousarray(rgba8, np.uint8)
    h, w, c = img.shape
    if c not in (3, 4):
        raise ValueError("need 3 or 4 channels")
    raw = b"".join(b"\0" + img[y].tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)
    hdr = struct.pack(">IIBBBBB", w, h, 8, 6 if c == 4 else 2, 0, 0, 0)
    Path(path).write_bytes(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", hdr) + chunk(b"IDAT", zlib.compress(raw, 6)) +
                           chunk(b"IEND", b""))


def read_png(path) -> np.ndarray:
    """Reader for the files write_png produces (filter type 0 only)."""
    data = Path(path).read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    off, idat = 8, b""
    w = h = ctype = None
    while off < len(data):
        (n,) = struct.unpack(">I", data[off:off + 4])
        tag, body = data[off + 4:off + 8], data[off + 8:off + 8 + n]
        if tag == b"IHDR":
            w, h, _, ctype = struct.unpack(">IIBB", body[:10])
        elif tag == b"IDAT":
            idat += body
        off += 12 + n
    c = 4 if ctype == 6 else 3
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + w * c)
    if np.any(raw[:, 0] != 0):
        raise ValueError("only unfiltered rows are supported")
    return raw[:, 1:].reshape(h, w, c)


def write_pfm(path, rgb: np.ndarray):
    """(h, w, 3) float -> little-endian PFM (rows bottom to top)."""
    img = np.ascontiguousarray(np.asarray(rgb, np.float32)[::-1])
    h, w = img.shape[:2]
    Path(path).write_bytes(f"PF\n{w} {h}\n-1.0\n".encode() + img.astype("<f4").tobytes())


def read_pfm(path) -> np.ndarray:
    data = Path(path).read_bytes()
    parts = data.split(b"\n", 3)
    w, h = map(int, parts[1].split())
    scale = float(parts[2])
    arr = np.frombuffer(parts[3], "<f4" if scale < 0 else ">f4").reshape(h, w, 3)
    return arr[::-1].astype(np.float32)


def read_hdr(path) -> np.ndarray:
    """Radiance RGBE (.hdr) image as float32 (h, w, 3), decoded as stb_image
    decodes it for the reference's environment maps (load_texture_float,
    dTexture.cu:188-196): value = byte * 2^(e - 136), 0 where e = 0, and the
    rows flipped (stbi_set_flip_vertically_on_load), so row 0 is the image's
    bottom row.  Flat and run-length-encoded scanlines, -Y H +X W layout."""
    data = Path(path).read_bytes()
    if not (data.startswith(b"#?RADIANCE") or data.startswith(b"#?RGBE")):
        raise ValueError("not a Radiance .hdr file")
    pos = 0
    fmt = None
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end].strip()
        pos = end + 1
        if not line:
            break
        if line.startswith(b"FORMAT="):
            fmt = line[7:]
    if fmt not in (None, b"32-bit_rle_rgbe"):
        raise ValueError(f"unsupported .hdr format {fmt!r}")
    end = data.index(b"\n", pos)
    res = data[pos:end].split()
    pos = end + 1
    if len(res) != 4 or res[0] != b"-Y" or res[2] != b"+X":
        raise ValueError(f"unsupported .hdr orientation {res!r}")
    h, w = int(res[1]), int(res[3])
    out = np.zeros((h, w, 4), np.uint8)
    buf = np.frombuffer(data, np.uint8)
    for y in range(h):
        if 8 <= w < 32768 and pos + 4 <= len(buf) and buf[pos] == 2 and buf[pos + 1] == 2 and not (buf[pos + 2] & 0x80):
            if (int(buf[pos + 2]) << 8 | int(buf[pos + 3])) != w:
                raise ValueError("run-length scanline width mismatch")
            pos += 4
            for c in range(4):
                x = 0
                while x < w:
                    count = int(buf[pos])
                    pos += 1
                    if count > 128:
                        count -= 128
                        if x + count > w:
                            raise ValueError("run overruns the scanline")
                        out[y, x:x + count, c] = buf[pos]
                        pos += 1
                    else:
                        if count == 0 or x + count > w:
                            raise ValueError("bad literal run")
                        out[y, x:x + count, c] = buf[pos:pos + count]
                        pos += count
                    x += count
        else:
            n = 4 * w
            if pos + n > len(buf):
                raise ValueError("truncated .hdr data")
            out[y] = buf[pos:pos + n].reshape(w, 4)
            pos += n
    e = out[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(np.float32(1.0), e - 136), np.float32(0.0)).astype(np.float32)
    rgb = out[..., :3].astype(np.float32) * scale[..., None]
    return np.ascontiguousarray(rgb[::-1])


def write_hdr(path, rgb: np.ndarray):
    """Float (h, w, 3) array, row 0 at the bottom as read_hdr returns it, as a
    flat (unencoded) Radiance RGBE file."""
    a = np.ascontiguousarray(np.asarray(rgb, np.float64)[::-1])
    m = a.max(-1)
    mant, e = np.frexp(m)
    scale = np.where(m > 1e-32, mant * 256.0 / np.where(m > 1e-32, m, 1.0), 0.0)
    rgbe = np.zeros(a.shape[:2] + (4,), np.uint8)
    rgbe[..., :3] = np.clip(np.floor(a * scale[..., None]), 0, 255).astype(np.uint8)
    rgbe[..., 3] = np.where(m > 1e-32, e + 128, 0).astype(np.uint8)
    head = f"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y {a.shape[0]} +X {a.shape[1]}\n".encode()
    Path(path).write_bytes(head + rgbe.tobytes())
