"""Minimal PNG reader for the tests: 8-bit RGB or RGBA, non-interlaced, any
of the five row filters (the CLI writes unfiltered stored blocks; the
reference renderer's stb writer picks a filter per row)."""
import struct
import zlib

import numpy as np


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    if pa <= pb and pa <= pc:
        return a
    return b if pb <= pc else c


def read_png(path):
    """-> uint8 array (H, W, channels)."""
    data = open(path, "rb").read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat, hdr = 8, b"", None
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if zlib.crc32(data[pos + 4:pos + 8 + n]) != struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]:
            raise ValueError(f"bad CRC in chunk {kind!r}")
        if kind == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat += body
        elif kind == b"IEND":
            break
        pos += 12 + n
    W, H, depth, ctype, _, _, interlace = hdr
    if depth != 8 or ctype not in (2, 6) or interlace != 0:
        raise ValueError("only 8-bit RGB/RGBA non-interlaced PNG files are read here")
    ch = 3 if ctype == 2 else 4
    raw = zlib.decompress(idat)
    stride = W * ch
    out = np.zeros((H, stride), np.uint8)
    prev = [0] * stride
    for y in range(H):
        f = raw[y * (stride + 1)]
        line = list(raw[y * (stride + 1) + 1:(y + 1) * (stride + 1)])
        cur = [0] * stride
        for i in range(stride):
            a = cur[i - ch] if i >= ch else 0
            b = prev[i]
            c = prev[i - ch] if i >= ch else 0
            x = line[i]
            if f == 1:
                x += a
            elif f == 2:
                x += b
            elif f == 3:
                x += (a + b) // 2
            elif f == 4:
                x += _paeth(a, b, c)
            elif f != 0:
                raise ValueError(f"unknown PNG filter {f}")
            cur[i] = x & 0xFF
        out[y] = cur
        prev = cur
    return out.reshape(H, W, ch)
