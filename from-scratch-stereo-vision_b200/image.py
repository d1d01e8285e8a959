"""Input images for the path: read_png, read_pnm and read_image with the
reference's signatures (stereonet.py:265-324, 3499-3601, 3604-3612).

The file is decoded on the host by the C library (inflate, PNG row
filters, Netpbm payloads) into raw 8/16-bit samples; only those cross to
the GPU, where one kernel forms the FP64 gray and interleaved RGB images
bit-identical to the reference's.  Like the reference, every reader
returns ``(gray, rgb, width, height)``; ``out`` chooses the container:
"list" (the reference's, the default so existing callers keep working),
"numpy", or "cuda" (FP64 device tensors that feed the GPU path without
leaving the device).  Files the reference rejects raise ValueError.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from .refine import _device, _ptr, _stream

PNG_SIGNATURE = b"\x89PNG\r\n\x1a\n"


def _decode(data: bytes, out: str, what: str):
    if out not in ("list", "numpy", "cuda"):
        raise ValueError("out must be 'list', 'numpy' or 'cuda'")
    lib = _lib.load()
    desc = _lib.RawImage()
    _lib.check(lib.sv_image_info(data, len(data), ctypes.byref(desc)), what)
    nbytes = desc.stride * desc.height
    raw = torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)
    _lib.check(lib.sv_image_decode_raw(data, len(data), ctypes.c_void_p(raw.data_ptr()), nbytes,
                                       ctypes.byref(desc)), what)
    dev = _device()
    raw_d = raw.to(dev, non_blocking=True)
    W, H = desc.width, desc.height
    gray = torch.empty(W * H, dtype=torch.float64, device=dev)
    rgb = torch.empty(3 * W * H, dtype=torch.float64, device=dev)
    _lib.check(lib.sv_raw_to_float(_ptr(raw_d), ctypes.byref(desc), _ptr(gray), _ptr(rgb),
                                   ctypes.c_void_p(_stream())), what)
    if out == "cuda":
        # the pinned staging buffer must outlive the asynchronous copy
        torch.cuda.current_stream().synchronize()
        return gray, rgb, W, H
    g, c = gray.cpu().numpy(), rgb.cpu().numpy()
    if out == "numpy":
        return g, c, W, H
    return g.tolist(), c.tolist(), W, H


def _read(path: str) -> bytes:
    with open(path, "rb") as f:
        return f.read()


def decode_image(data: bytes, out: str = "list"):
    """A PNG or PGM/PPM held in memory, chosen by the magic bytes."""
    return _decode(bytes(data), out, "decode_image")


def read_png(path, out: str = "list"):
    """stereonet.py:3499-3601 -> (gray, rgb, width, height)."""
    data = _read(path)
    if data[:8] != PNG_SIGNATURE:
        raise ValueError("not a PNG file: " + str(path))
    return _decode(data, out, "read_png")


def read_pnm(path, out: str = "list"):
    """stereonet.py:265-324 -> (gray, rgb, width, height)."""
    data = _read(path)
    if data[:2] not in (b"P2", b"P3", b"P5", b"P6"):
        raise ValueError("not a PGM/PPM file: " + str(path))
    return _decode(data, out, "read_pnm")


def read_image(path, out: str = "list"):
    """stereonet.py:3604-3612: PNG or Netpbm by the magic bytes."""
    data = _read(path)
    if data[:8] == PNG_SIGNATURE:
        return _decode(data, out, "read_png")
    if data[:2] not in (b"P2", b"P3", b"P5", b"P6"):
        raise ValueError("not a PGM/PPM file: " + str(path))
    return _decode(data, out, "read_pnm")


def _decode_many(blobs, out, threads, what):
    """Host decode of every file on `threads` threads, then one H2D copy and
    one conversion launch per file on the current stream."""
    lib = _lib.load()
    n = len(blobs)
    descs = (_lib.RawImage * n)()
    for i, b in enumerate(blobs):
        _lib.check(lib.sv_image_info(b, len(b), ctypes.byref(descs[i])), "%s[%d]" % (what, i))
    sizes = [d.stride * d.height for d in descs]
    raws = [torch.empty(max(sz, 1), dtype=torch.uint8, pin_memory=True) for sz in sizes]
    c_data = (ctypes.c_char_p * n)(*blobs)
    c_sizes = (ctypes.c_size_t * n)(*[len(b) for b in blobs])
    c_raw = (ctypes.c_void_p * n)(*[r.data_ptr() for r in raws])
    c_rb = (ctypes.c_size_t * n)(*sizes)
    st = (ctypes.c_int * n)()
    _lib.check(lib.sv_image_decode_batch(n, c_data, c_sizes, c_raw, c_rb, descs, st,
                                         int(threads)), what)
    dev = _device()
    res = []
    for i in range(n):
        W, H = descs[i].width, descs[i].height
        raw_d = raws[i].to(dev, non_blocking=True)
        gray = torch.empty(W * H, dtype=torch.float64, device=dev)
        rgb = torch.empty(3 * W * H, dtype=torch.float64, device=dev)
        _lib.check(lib.sv_raw_to_float(_ptr(raw_d), ctypes.byref(descs[i]), _ptr(gray), _ptr(rgb),
                                       ctypes.c_void_p(_stream())), what)
        res.append((gray, rgb, W, H))
    torch.cuda.current_stream().synchronize()
    if out == "cuda":
        return res
    conv = (lambda t: t.cpu().numpy()) if out == "numpy" else (lambda t: t.cpu().numpy().tolist())
    return [(conv(g), conv(c), W, H) for g, c, W, H in res]


def read_images(paths, out: str = "list", threads: int = 0):
    """read_image of several files (e.g. the two views of a pair, or a test
    split), decoded concurrently on host threads (default: one per file, up
    to the CPU count).  Returns a list of (gray, rgb, width, height)."""
    if out not in ("list", "numpy", "cuda"):
        raise ValueError("out must be 'list', 'numpy' or 'cuda'")
    blobs = [_read(p) for p in paths]
    for p, b in zip(paths, blobs):
        if b[:8] != PNG_SIGNATURE and b[:2] not in (b"P2", b"P3", b"P5", b"P6"):
            raise ValueError("not a PGM/PPM file: " + str(p))
    if not blobs:
        return []
    threads = threads or min(len(blobs), os.cpu_count() or 1)
    return _decode_many(blobs, out, threads, "read_images")


def decode_raw(data: bytes):
    """Host decode only: (raw samples as a numpy uint8 array [H][stride],
    sv_raw_image).  No GPU is touched."""
    lib = _lib.load()
    desc = _lib.RawImage()
    _lib.check(lib.sv_image_info(data, len(data), ctypes.byref(desc)), "decode_raw")
    raw = np.empty(max(desc.stride * desc.height, 1), dtype=np.uint8)
    _lib.check(lib.sv_image_decode_raw(data, len(data), raw.ctypes.data_as(ctypes.c_void_p),
                                       raw.size, ctypes.byref(desc)), "decode_raw")
    return raw[:desc.stride * desc.height].reshape(desc.height, desc.stride), desc
