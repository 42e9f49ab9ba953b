"""PNG files of rendered frames: what ``RgbImage::save`` writes for the
reference's ``gr-renderer --output x.png`` (crates/gr-renderer/src/main.rs:137,
through the ``image`` crate 0.25.10, a dependency not vendored with the
reference).

Encoder: 8-bit truecolour (colour type 2), no interlace, one IDAT of the
zlib-deflated scanlines, each with filter type 0 (None) or 1 (Sub), whichever
sums smaller as signed bytes (the minimum-sum-of-absolute-differences
heuristic of the PNG specification, section 12.8).  The decoder reads
colour types 2 and 6 at 8 bits, all five filter types, and checks every
chunk CRC; tests use it to read frames back.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

_SIG = b"\x89PNG\r\n\x1a\n"


def _chunk(kind: bytes, data: bytes) -> bytes:
    return (struct.pack(">I", len(data)) + kind + data +
            struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF))


def encode_png(img: np.ndarray, level: int = 6) -> bytes:
    """(height, width, 3) uint8 to PNG bytes."""
    img = np.ascontiguousarray(img)
    if img.dtype != np.uint8 or img.ndim != 3 or img.shape[2] != 3:
        raise ValueError("encode_png wants a (height, width, 3) uint8 array")
    h, w = img.shape[:2]
    if h < 1 or w < 1:
        raise ValueError("empty image")
    rows = img.reshape(h, w * 3)
    sub = rows.copy()
    sub[:, 3:] = rows[:, 3:] - rows[:, :-3]  # uint8 arithmetic wraps mod 256
    cost_none = np.abs(rows.view(np.int8).astype(np.int32)).sum(axis=1)
    cost_sub = np.abs(sub.view(np.int8).astype(np.int32)).sum(axis=1)
    use_sub = cost_sub < cost_none
    raw = np.empty((h, 1 + w * 3), np.uint8)
    raw[:, 0] = np.where(use_sub, 1, 0)
    raw[:, 1:] = np.where(use_sub[:, None], sub, rows)
    ihdr = struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)
    return (_SIG + _chunk(b"IHDR", ihdr) +
            _chunk(b"IDAT", zlib.compress(raw.tobytes(), level)) + _chunk(b"IEND", b""))


def write_png(path, img: np.ndarray) -> None:
    data = encode_png(img)
    with open(path, "wb") as f:
        f.write(data)


def _paeth(a: int, b: int, c: int) -> int:
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    if pa <= pb and pa <= pc:
        return a
    return b if pb <= pc else c


def decode_png(data: bytes) -> np.ndarray:
    """PNG bytes (8-bit RGB or RGBA, not interlaced) to (height, width, C) uint8."""
    if data[:8] != _SIG:
        raise ValueError("not a PNG file")
    pos = 8
    header = None
    idat = bytearray()
    while pos + 8 <= len(data):
        n, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        crc = data[pos + 8 + n:pos + 12 + n]
        if len(body) != n or len(crc) != 4:
            raise ValueError("truncated PNG chunk")
        if struct.unpack(">I", crc)[0] != zlib.crc32(kind + body) & 0xFFFFFFFF:
            raise ValueError("PNG chunk CRC mismatch")
        pos += 12 + n
        if kind == b"IHDR":
            header = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat += body
        elif kind == b"IEND":
            break
    if header is None:
        raise ValueError("PNG without IHDR")
    w, h, depth, ctype, _, _, interlace = header
    if depth != 8 or ctype not in (2, 6) or interlace != 0:
        raise ValueError("unsupported PNG form")
    bpp = 3 if ctype == 2 else 4
    raw = np.frombuffer(zlib.decompress(bytes(idat)), np.uint8)
    stride = w * bpp
    if raw.size != h * (stride + 1):
        raise ValueError("PNG data size mismatch")
    raw = raw.reshape(h, stride + 1)
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        ft = raw[y, 0]
        f = raw[y, 1:].astype(np.int32)
        if ft == 0:  # None
            cur = f
        elif ft == 1:  # Sub: running sum along the row, per channel
            cur = np.cumsum(f.reshape(w, bpp), axis=0).reshape(-1) % 256
        elif ft == 2:  # Up
            cur = (f + prev) % 256
        elif ft == 3 or ft == 4:  # Average, Paeth
            cur = np.zeros(stride, np.int32)
            for x in range(stride):
                a = int(cur[x - bpp]) if x >= bpp else 0
                b = int(prev[x])
                if ft == 3:
                    cur[x] = (f[x] + ((a + b) >> 1)) & 255
                else:
                    c = int(prev[x - bpp]) if x >= bpp else 0
                    cur[x] = (f[x] + _paeth(a, b, c)) & 255
        else:
            raise ValueError("bad PNG filter type")
        out[y] = cur
        prev = cur.astype(np.int32)
    return out.reshape(h, w, bpp)


def read_png(path) -> np.ndarray:
    with open(path, "rb") as f:
        return decode_png(f.read())
