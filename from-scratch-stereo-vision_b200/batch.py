"""lr_refine over many pairs of uneven sizes at once (sv_batch_lr_refine).

``lr_refine_batch(pairs, tol=1.0, **kw)`` takes a list of
``(left, right, disp0, W, H)`` tuples with the reference's argument meaning
(stereonet.py:5343-5391) and returns a list of ``(disparity, status)``, each
bit-identical to ``refine.lr_refine`` on that pair alone.  ``BatchRefiner``
is the device-resident form: the images, disparities and outputs stay in
HBM and one call enqueues the whole batch (seven launches; the SGM stage is
a persistent kernel over a device-side queue of scanline tasks).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .refine import _device, _image, _kind, _params, _ptr, _ret, _stream, _to_dev, _finite_disp


class PairDesc(ctypes.Structure):
    _fields_ = [("left", ctypes.c_void_p), ("right", ctypes.c_void_p),
                ("disp0", ctypes.c_void_p), ("out", ctypes.c_void_p),
                ("status", ctypes.c_void_p), ("W", ctypes.c_int), ("H", ctypes.c_int)]


class BatchRefiner:
    """lr_refine for a fixed list of (W, H) sizes; buffers allocated once."""

    def __init__(self, sizes, dtype=torch.uint8, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                 paths=8, uniq=0.0):
        self.lib = _lib.load()
        self.sizes = [(int(W), int(H)) for W, H in sizes]
        self.tol = float(tol)
        self.p = _params(R=R, P1=P1, P2=P2, rx=rx, ry=ry, paths=paths, uniq=uniq)
        self.code = {torch.uint8: _lib.SV_U8, torch.float32: _lib.SV_F32,
                     torch.float64: _lib.SV_F64}[dtype]
        dev = _device()
        self.left = [torch.empty(W * H, dtype=dtype, device=dev) for W, H in self.sizes]
        self.right = [torch.empty(W * H, dtype=dtype, device=dev) for W, H in self.sizes]
        self.disp0 = [torch.empty(W * H, dtype=torch.float64, device=dev) for W, H in self.sizes]
        self.out = [torch.empty(W * H, dtype=torch.float64, device=dev) for W, H in self.sizes]
        self.status = [torch.empty(W * H, dtype=torch.uint8, device=dev) for W, H in self.sizes]
        self.descs = (PairDesc * len(self.sizes))()
        for i, (W, H) in enumerate(self.sizes):
            self.descs[i] = PairDesc(self.left[i].data_ptr(), self.right[i].data_ptr(),
                                     self.disp0[i].data_ptr(), self.out[i].data_ptr(),
                                     self.status[i].data_ptr(), W, H)
        self.need = self.lib.sv_batch_lr_refine_workspace_size(self.descs, len(self.sizes),
                                                               ctypes.byref(self.p))
        if self.need == 0:
            _lib.raise_last("lr_refine_batch")
        self.ws = torch.empty(self.need, dtype=torch.uint8, device=dev)

    @property
    def pixels(self) -> int:
        return sum(W * H for W, H in self.sizes)

    def run(self, stream=None) -> None:
        _lib.check(self.lib.sv_batch_lr_refine(self.descs, len(self.sizes), self.code, self.tol,
                                               ctypes.byref(self.p), _ptr(self.ws), self.need,
                                               _stream() if stream is None else stream),
                   "lr_refine_batch")

    def data_status(self) -> None:
        rc = self.lib.sv_workspace_status(_ptr(self.ws), ctypes.c_void_p(_stream()))
        _lib.check(rc, "lr_refine_batch")


def lr_refine_batch(pairs, tol=1.0, **kw):
    """[(left, right, disp0, W, H), ...] -> [(disparity, status), ...]."""
    if not pairs:
        return []
    imgs = []
    for (left, right, disp0, W, H) in pairs:
        _finite_disp(disp0)
        tl, code = _image(left, W * H, "left")
        tr = _image(right, W * H, "right")[0].to(tl.dtype)
        imgs.append((tl, tr, _to_dev(disp0, W * H, torch.float64, name="disp0")))
    dtype = imgs[0][0].dtype
    b = BatchRefiner([(p[3], p[4]) for p in pairs], dtype=dtype, tol=tol, **kw)
    for i, (tl, tr, td) in enumerate(imgs):
        b.left[i].copy_(tl.to(dtype))
        b.right[i].copy_(tr.to(dtype))
        b.disp0[i].copy_(td)
    b.run()
    b.data_status()
    return [(_ret(b.out[i], pairs[i][0]), _ret(b.status[i], pairs[i][0], as_int=True))
            for i in range(len(pairs))]
