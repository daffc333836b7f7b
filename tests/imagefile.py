"""Minimal readers for the two files the reference's CLI writes, used to compare outputs.

* Radiance RGBE `.hdr` (flat or new-style run-length scanlines), decoded as
  mantissa * 2^(exponent - 136), the convention of the reader the reference links.
* 8-bit RGB/RGBA PNG, non-interlaced, with the five PNG row filters.
"""
import struct
import zlib

import numpy as np


def read_hdr_rgbe(path):
    """The raw RGBE quads of a Radiance file, shape (H, W, 4), uint8."""
    data = open(path, "rb").read()
    pos = 0
    width = height = None
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end].decode("ascii", "replace")
        pos = end + 1
        if line.startswith("-Y "):
            parts = line.split()
            height, width = int(parts[1]), int(parts[3])
            break
    out = np.zeros((height, width, 4), np.uint8)
    for y in range(height):
        if (width >= 8 and width < 32768 and data[pos] == 2 and data[pos + 1] == 2
                and (data[pos + 2] << 8 | data[pos + 3]) == width):
            pos += 4
            for c in range(4):
                x = 0
                while x < width:
                    n = data[pos]
                    pos += 1
                    if n > 128:
                        n -= 128
                        out[y, x:x + n, c] = data[pos]
                        pos += 1
                    else:
                        out[y, x:x + n, c] = np.frombuffer(data, np.uint8, n, pos)
                        pos += n
                    x += n
        else:
            out[y] = np.frombuffer(data, np.uint8, width * 4, pos).reshape(width, 4)
            pos += width * 4
    return out


def rgbe_to_float(q):
    q = q.astype(np.int32)
    scale = np.where(q[..., 3] > 0, np.ldexp(1.0, q[..., 3] - 136), 0.0).astype(np.float32)
    return q[..., :3].astype(np.float32) * scale[..., None]


def read_hdr(path):
    return rgbe_to_float(read_hdr_rgbe(path))


def read_png(path):
    """8-bit RGB or RGBA PNG pixels, shape (H, W, channels), uint8."""
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n", "not a PNG file"
    pos, idat = 8, b""
    width = height = channels = None
    while pos < len(data):
        length, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + length]
        if kind == b"IHDR":
            width, height, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
            assert depth == 8 and interlace == 0 and ctype in (2, 6)
            channels = 3 if ctype == 2 else 4
        elif kind == b"IDAT":
            idat += body
        pos += 12 + length
    raw = np.frombuffer(zlib.decompress(idat), np.uint8)
    stride = width * channels
    out = np.zeros((height, stride), np.int32)
    prev = np.zeros(stride, np.int32)
    for y in range(height):
        f = raw[y * (stride + 1)]
        row = raw[y * (stride + 1) + 1:(y + 1) * (stride + 1)].astype(np.int32)
        cur = np.zeros(stride, np.int32)
        if f == 0:
            cur = row
        elif f == 2:
            cur = (row + prev) & 255
        else:
            for x in range(stride):
                a = cur[x - channels] if x >= channels else 0
                b = prev[x]
                c = prev[x - channels] if x >= channels else 0
                if f == 1:
                    p = a
                elif f == 3:
                    p = (a + b) >> 1
                else:
                    pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                    p = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                cur[x] = (row[x] + p) & 255
        out[y] = cur
        prev = cur
    return out.astype(np.uint8).reshape(height, width, channels)
