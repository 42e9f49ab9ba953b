"""Radiance ``.hdr`` (RGBE) images: the file format ``HdriSky::from_file``
reads (crates/raytracer/src/curved/sky.rs:59-71, through the ``image``
crate 0.25.10, a dependency not vendored with the reference).

Format (Greg Ward, "Real Pixels", Graphics Gems II, 1991; the Radiance
file format): text header lines up to an empty line, a resolution line
``-Y <height> +X <width>`` (top row first), then one scanline per row of
4-byte RGBE pixels.  A scanline is either flat, in the old run-length form
(a pixel (1, 1, 1, n) repeats the previous pixel n << shift times, shift
growing by 8 over consecutive repeats), or in the adaptive form: the bytes
(2, 2, width >> 8, width & 255), then each of the four channels run-length
coded on its own (a count byte above 128 repeats the next byte count - 128
times, otherwise count literal bytes follow).

Decoding to linear float, as the ``image`` crate does: a channel is
``c * 2**(e - 136)``, and 0 when ``e == 0``.
"""
from __future__ import annotations

import numpy as np


def rgbe_to_float(rgbe: np.ndarray) -> np.ndarray:
    """(..., 4) uint8 RGBE texels to (..., 3) float32."""
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e == 0, np.float32(0.0),
                     np.ldexp(np.float32(1.0), e - 136).astype(np.float32))
    return (rgbe[..., :3].astype(np.float32) * scale[..., None]).astype(np.float32)


def float_to_rgbe(rgb: np.ndarray) -> np.ndarray:
    """(..., 3) float to (..., 4) uint8 RGBE: the largest channel m sets
    e = frexp(m) exponent + 128, channels scaled by 256 / 2**frexp(m)
    exponent and truncated; m below 1e-32 encodes as zeros (Ward's
    ``setcolr``)."""
    rgb = np.asarray(rgb, np.float64)
    m = rgb.max(axis=-1)
    mant, ex = np.frexp(m)
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    ok = m >= 1e-32
    scale = np.where(ok, mant * 256.0 / np.where(ok, m, 1.0), 0.0)
    out[..., :3] = np.where(ok[..., None], np.clip(rgb * scale[..., None], 0, 255), 0).astype(np.uint8)
    out[..., 3] = np.where(ok, ex + 128, 0).astype(np.uint8)
    return out


def _read_scanline(buf: bytes, pos: int, width: int) -> tuple[np.ndarray, int]:
    if 8 <= width <= 0x7FFF and pos + 4 <= len(buf) and buf[pos] == 2 and buf[pos + 1] == 2 \
            and ((buf[pos + 2] << 8) | buf[pos + 3]) == width and buf[pos + 2] < 128:
        pos += 4
        line = np.empty((4, width), np.uint8)
        for c in range(4):
            x = 0
            while x < width:
                if pos >= len(buf):
                    raise ValueError("truncated .hdr scanline")
                count = buf[pos]
                pos += 1
                if count > 128:
                    count -= 128
                    if x + count > width or pos >= len(buf):
                        raise ValueError("bad run in .hdr scanline")
                    line[c, x:x + count] = buf[pos]
                    pos += 1
                else:
                    if count == 0 or x + count > width or pos + count > len(buf):
                        raise ValueError("bad literal in .hdr scanline")
                    line[c, x:x + count] = np.frombuffer(buf, np.uint8, count, pos)
                    pos += count
                x += count
        return line.T.copy(), pos
    # flat or old run-length pixels
    line = np.empty((width, 4), np.uint8)
    x = 0
    shift = 0
    while x < width:
        if pos + 4 > len(buf):
            raise ValueError("truncated .hdr scanline")
        px = buf[pos:pos + 4]
        pos += 4
        if px[0] == 1 and px[1] == 1 and px[2] == 1:
            if x == 0:
                raise ValueError("run without a pixel to repeat in .hdr scanline")
            count = px[3] << shift
            if x + count > width:
                raise ValueError("bad run in .hdr scanline")
            line[x:x + count] = line[x - 1]
            x += count
            shift += 8
        else:
            line[x] = np.frombuffer(px, np.uint8)
            x += 1
            shift = 0
    return line, pos


def decode_hdr(data: bytes) -> np.ndarray:
    """A Radiance file's bytes to (height, width, 3) float32, row 0 first in
    the file (the top of the image)."""
    pos = 0
    first = True
    while True:
        end = data.find(b"\n", pos)
        if end < 0:
            raise ValueError("no .hdr header end")
        line = data[pos:end].rstrip(b"\r")
        pos = end + 1
        if first:
            if not line.startswith(b"#?"):
                raise ValueError("not a Radiance .hdr file")
            first = False
            continue
        if line == b"":
            break
        if line.startswith(b"FORMAT=") and line != b"FORMAT=32-bit_rle_rgbe":
            raise ValueError("unsupported .hdr format " + line.decode(errors="replace"))
    end = data.find(b"\n", pos)
    if end < 0:
        raise ValueError("no .hdr resolution line")
    parts = data[pos:end].split()
    pos = end + 1
    if len(parts) != 4 or parts[0] != b"-Y" or parts[2] != b"+X":
        raise ValueError("unsupported .hdr orientation " + data[pos:end].decode(errors="replace"))
    height, width = int(parts[1]), int(parts[3])
    if height < 1 or width < 1:
        raise ValueError("empty .hdr image")
    rgbe = np.empty((height, width, 4), np.uint8)
    for y in range(height):
        rgbe[y], pos = _read_scanline(data, pos, width)
    return rgbe_to_float(rgbe)


def read_hdr(path) -> np.ndarray:
    with open(path, "rb") as f:
        return decode_hdr(f.read())


def _rle_channel(row: np.ndarray) -> bytes:
    out = bytearray()
    n = len(row)
    x = 0
    while x < n:
        run = 1
        while x + run < n and run < 127 and row[x + run] == row[x]:
            run += 1
        if run >= 4:
            out += bytes((128 + run, int(row[x])))
            x += run
            continue
        lit = x
        while lit < n and lit - x < 128:
            if lit + 3 < n and row[lit] == row[lit + 1] == row[lit + 2] == row[lit + 3]:
                break
            lit += 1
        out.append(lit - x)
        out += bytes(row[x:lit])
        x = lit
    return bytes(out)


def encode_hdr(rgb: np.ndarray, rle: bool = True) -> bytes:
    """(height, width, 3) float to Radiance bytes (adaptive run-length
    scanlines when `rle` and 8 <= width <= 32767, flat otherwise)."""
    rgbe = float_to_rgbe(rgb)
    h, w = rgbe.shape[:2]
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n")
    out += f"-Y {h} +X {w}\n".encode()
    for y in range(h):
        if rle and 8 <= w <= 0x7FFF:
            out += bytes((2, 2, w >> 8, w & 255))
            for c in range(4):
                out += _rle_channel(rgbe[y, :, c])
        else:
            out += rgbe[y].tobytes()
    return bytes(out)


def write_hdr(path, rgb: np.ndarray, rle: bool = True) -> None:
    with open(path, "wb") as f:
        f.write(encode_hdr(rgb, rle))
