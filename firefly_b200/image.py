"""Headless image output, in place of the reference's GL display surface
(wf_logic writes the tonemapped char4 into a GL texture, CUDA-RayTracer/
kernel.cu:447-454): 8-bit PNG of ff_film_tonemap's RGBA and float PFM of the
mean radiance, with standard-library encoders only."""
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
