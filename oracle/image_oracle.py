"""TEST INFRASTRUCTURE ONLY -- CPU restatement of the reference's image
readers (stereonet.py:244-324 read_pnm, 3421-3601 zlib_decompress /
_unfilter / read_png, 3604-3612 read_image).

DEFLATE itself is delegated to Python's zlib module (an independent
implementation of RFC 1951), fed the raw stream after the two zlib header
bytes so that, like the reference's inflate (stereonet.py:3335-3418), the
Adler-32 trailer is not checked.  The zlib header checks (3421-3433), the
row filters (3436-3496), sample extraction and the FP64 arithmetic
(3556-3598, 290-322) are restated here.  tests/golden/images.npz (made by
running the reference) pins it.  Only tests use this module.
"""

from __future__ import annotations

import zlib

import numpy as np

PNG_SIGNATURE = b"\x89PNG\r\n\x1a\n"


def zlib_decompress(data: bytes) -> bytes:
    """stereonet.py:3421-3433."""
    if len(data) < 2:
        raise ValueError("zlib stream too short")
    cmf, flg = data[0], data[1]
    if cmf & 0x0F != 8:
        raise ValueError("unsupported zlib compression method")
    if ((cmf << 8) | flg) % 31 != 0:
        raise ValueError("zlib header checksum failed")
    if flg & 0x20:
        raise ValueError("zlib preset dictionary not supported")
    d = zlib.decompressobj(-15)
    try:
        return d.decompress(data[2:])
    except zlib.error as e:
        raise ValueError("corrupt DEFLATE stream: %s" % e) from None


def unfilter(raw: bytes, height: int, bpp: int, stride: int) -> np.ndarray:
    """stereonet.py:3456-3496 -> uint8 [height][stride]."""
    out = np.zeros((height, stride), dtype=np.int64)
    pos = 0
    for y in range(height):
        ft = raw[pos]
        row = np.frombuffer(raw[pos + 1:pos + 1 + stride], dtype=np.uint8).astype(np.int64)
        pos += 1 + stride
        up = out[y - 1] if y > 0 else np.zeros(stride, dtype=np.int64)
        o = out[y]
        if ft == 0:
            o[:] = row
        elif ft == 2:
            o[:] = (row + up) & 0xFF
        elif ft in (1, 3, 4):
            for i in range(stride):
                a = int(o[i - bpp]) if i >= bpp else 0
                b = int(up[i])
                c = int(up[i - bpp]) if i >= bpp else 0
                if ft == 1:
                    pr = a
                elif ft == 3:
                    pr = (a + b) >> 1
                else:
                    p = a + b - c
                    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                    pr = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                o[i] = (int(row[i]) + pr) & 0xFF
        else:
            raise ValueError("unknown PNG filter type %d on row %d" % (ft, y))
    return out.astype(np.uint8)


def _gray(r, g, b):
    return 0.299 * r + 0.587 * g + 0.114 * b


def _pack(r, g, b):
    rgb = np.empty(3 * r.size, dtype=np.float64)
    rgb[0::3], rgb[1::3], rgb[2::3] = r, g, b
    return rgb


def read_png_bytes(data: bytes):
    """stereonet.py:3499-3601 on the file's bytes -> (gray, rgb, W, H)."""
    if data[:8] != PNG_SIGNATURE:
        raise ValueError("not a PNG file")
    pos, idat, palette = 8, bytearray(), None
    W = H = depth = ct = interlace = 0
    while pos < len(data):
        n = int.from_bytes(data[pos:pos + 4], "big")
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if tag == b"IHDR":
            W, H = int.from_bytes(body[0:4], "big"), int.from_bytes(body[4:8], "big")
            depth, ct, interlace = body[8], body[9], body[12]
        elif tag == b"PLTE":
            palette = body
        elif tag == b"IDAT":
            idat += body
        elif tag == b"IEND":
            break
    if interlace:
        raise ValueError("Adam7 interlaced PNG is not supported")
    if depth not in (1, 2, 4, 8, 16):
        raise ValueError("unsupported PNG bit depth %d" % depth)
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}.get(ct)
    if ch is None:
        raise ValueError("unsupported PNG colour type %d" % ct)
    stride = (W * ch * depth + 7) // 8
    raw = unfilter(zlib_decompress(bytes(idat)), H, max(1, ch * depth // 8), stride)
    if depth == 8:
        s = raw[:, :W * ch].reshape(H * W, ch).astype(np.float64)
    elif depth == 16:
        w = raw[:, :2 * W * ch].reshape(H * W * ch, 2).astype(np.int64)
        s = ((w[:, 0] << 8) | w[:, 1]).reshape(H * W, ch).astype(np.float64)
    else:
        bit = np.arange(W) * depth
        byte = raw[:, bit >> 3].astype(np.int64)
        s = ((byte >> (8 - depth - (bit & 7))) & ((1 << depth) - 1)).reshape(H * W, 1)
    inv = 1.0 / 65535.0 if depth == 16 else 1.0 / ((1 << depth) - 1)
    if ct == 3:
        if palette is None:
            raise ValueError("indexed PNG with no PLTE chunk")
        p = 3 * s[:, 0].astype(np.int64)
        if p.size and p.max() + 2 >= len(palette):
            raise ValueError("palette index out of range")
        pal = np.frombuffer(palette, dtype=np.uint8).astype(np.float64)
        r, g, b = pal[p] / 255.0, pal[p + 1] / 255.0, pal[p + 2] / 255.0
    elif ct in (0, 4):
        r = g = b = s[:, 0] * inv
    else:
        r, g, b = s[:, 0] * inv, s[:, 1] * inv, s[:, 2] * inv
    return _gray(r, g, b), _pack(r, g, b), W, H


def _pnm_tokens(data: bytes, i: int):
    """stereonet.py:244-262."""
    toks, n = [], len(data)
    while len(toks) < 3 and i < n:
        c = data[i]
        if c == 35:
            while i < n and data[i] not in (10, 13):
                i += 1
        elif c in (32, 9, 10, 13):
            i += 1
        else:
            j = i
            while j < n and data[j] not in (32, 9, 10, 13):
                j += 1
            toks.append(data[i:j].decode("ascii"))
            i = j
    return toks, i


def read_pnm_bytes(data: bytes):
    """stereonet.py:265-324 on the file's bytes -> (gray, rgb, W, H)."""
    magic = data[:2]
    if magic not in (b"P2", b"P3", b"P5", b"P6"):
        raise ValueError("not a PGM/PPM file")
    toks, pos = _pnm_tokens(data, 2)
    W, H, maxval = int(toks[0]), int(toks[1]), int(toks[2])
    inv = 1.0 / maxval
    ch = 3 if magic in (b"P3", b"P6") else 1
    count = W * H * ch
    if magic in (b"P2", b"P3"):
        s = np.array([int(t) for t in data[pos:].split()[:count]], dtype=np.float64)
    else:
        pos += 1
        if maxval < 256:
            s = np.frombuffer(data[pos:pos + count], dtype=np.uint8).astype(np.float64)
        else:
            w = np.frombuffer(data[pos:pos + 2 * count], dtype=np.uint8).astype(np.int64)
            s = ((w[0::2] << 8) | w[1::2]).astype(np.float64)
    if s.size != count:
        raise ValueError("truncated PGM/PPM payload")
    v = s * inv
    if ch == 3:
        r, g, b = v[0::3], v[1::3], v[2::3]
        return _gray(r, g, b), v, W, H
    return v, _pack(v, v, v), W, H


def read_image_bytes(data: bytes):
    """stereonet.py:3604-3612."""
    if data[:8] == PNG_SIGNATURE:
        return read_png_bytes(data)
    return read_pnm_bytes(data)


def raw_to_float(raw: np.ndarray, desc):
    """The FP64 step of read_png / read_pnm (stereonet.py:3556-3598,
    290-322) applied to the raw samples the host decoder produced
    ([H][stride] uint8 with the sv_raw_image description)."""
    W, H, ch, depth = desc.width, desc.height, desc.channels, desc.depth
    if depth == 8:
        s = raw[:, :W * ch].reshape(H * W, ch).astype(np.float64)
    elif depth == 16:
        w = raw[:, :2 * W * ch].reshape(H * W * ch, 2).astype(np.int64)
        s = ((w[:, 0] << 8) | w[:, 1]).reshape(H * W, ch).astype(np.float64)
    else:
        bit = np.arange(W) * depth
        byte = raw[:, bit >> 3].astype(np.int64)
        s = ((byte >> (8 - depth - (bit & 7))) & ((1 << depth) - 1)).reshape(H * W, 1)
    if desc.colortype == 3:
        p = 3 * s[:, 0].astype(np.int64)
        pal = np.frombuffer(bytes(desc.palette), dtype=np.uint8).astype(np.float64)
        r, g, b = pal[p] / 255.0, pal[p + 1] / 255.0, pal[p + 2] / 255.0
    elif desc.colortype in (0, 4):
        r = g = b = s[:, 0] * desc.inv
    else:
        r, g, b = s[:, 0] * desc.inv, s[:, 1] * desc.inv, s[:, 2] * desc.inv
    gray = r if (desc.kind == 2 and desc.colortype == 0) else _gray(r, g, b)
    return gray, _pack(r, g, b)
