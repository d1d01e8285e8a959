"""The disparity hot path for one rectified pair, device resident.

``PairPipeline`` runs ``predict_auto`` (stereonet.py:3872-3929) and then
``lr_refine`` with ``refine_disparity``'s parameters (R=10, P1=12, P2=150,
9x7 census, tol=2.0; stereonet.py:5865-5872) on a W x H pair.  All buffers
and workspaces are allocated once per size; ``run_device`` only enqueues
kernels (plus the one 8-byte read per predict_auto pass that the work-width
choice needs), ``run_host`` adds the host->device copy of the two images and
the device->host copy of the refined disparity and status.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .network import _precision, gpu_net
from .refine import LRRefiner, _ptr, _stream


class PairPipeline:
    def __init__(self, W: int, H: int, net, image_dtype=torch.uint8, R=10, P1=12.0, P2=150.0,
                 rx=4, ry=3, tol=2.0, probe_width=64, max_width=320, passes=3,
                 target_peak=None, device=None, precision="fp32"):
        self.lib = _lib.load()
        self.precision = _precision(precision)
        self.W, self.H = W, H
        self.dev = torch.device("cuda", torch.cuda.current_device()) if device is None else device
        # A stream of its own: work on it can be captured, so each predict_auto
        # pass replays as one CUDA graph after its first run.
        self.stream = torch.cuda.Stream(device=self.dev)
        self.net = gpu_net(net)
        self.tp = float(self.net.target_peak if target_peak is None else target_peak)
        self.probe_width, self.max_width, self.passes = probe_width, max_width, passes
        self.code = {torch.uint8: _lib.SV_U8, torch.float32: _lib.SV_F32,
                     torch.float64: _lib.SV_F64}[image_dtype]
        N = W * H
        self.left = torch.empty(N, dtype=image_dtype, device=self.dev)
        self.right = torch.empty(N, dtype=image_dtype, device=self.dev)
        self.disp0 = torch.empty(N, dtype=torch.float64, device=self.dev)
        self.disp_work = torch.empty(max(N, 64 * 64), dtype=torch.float64, device=self.dev)
        self.out = torch.empty(N, dtype=torch.float64, device=self.dev)
        self.status = torch.empty(N, dtype=torch.uint8, device=self.dev)
        self.pneed = self.lib.sv_predict_workspace_size(self.net.handle, W, H, max_width)
        self.pws = torch.empty(max(self.pneed, 256), dtype=torch.uint8, device=self.dev)
        self.refiner = LRRefiner(W, H, R=R, P1=P1, P2=P2, rx=rx, ry=ry, tol=tol)
        self._Ww, self._Hw = ctypes.c_int(), ctypes.c_int()
        self._trace = (ctypes.c_int * (passes + 2))()
        # pinned host staging for run_host
        self.h_left = torch.empty(N, dtype=image_dtype, pin_memory=True)
        self.h_right = torch.empty(N, dtype=image_dtype, pin_memory=True)
        self.h_out = torch.empty(N, dtype=torch.float64, pin_memory=True)
        self.h_status = torch.empty(N, dtype=torch.uint8, pin_memory=True)

    # ------------------------------------------------------------------
    def predict(self, stream=None) -> None:
        s = self.stream.cuda_stream if stream is None else stream
        _lib.check(self.lib.sv_predict_auto(
            self.net.handle, _ptr(self.left), _ptr(self.right), self.code, self.W, self.H,
            self.tp, self.probe_width, self.max_width, self.passes, self.precision,
            _ptr(self.disp0), _ptr(self.disp_work), ctypes.byref(self._Ww),
            ctypes.byref(self._Hw), self._trace, _ptr(self.pws), self.pneed, s), "predict_auto")

    def confidence(self, stream=None):
        """The network's spread and peak probability of the last predict()'s
        final pass, at W x H (FP64 device tensors self.spread, self.pmax)."""
        if not hasattr(self, "spread"):
            N = self.W * self.H
            self.spread = torch.empty(N, dtype=torch.float64, device=self.dev)
            self.pmax = torch.empty(N, dtype=torch.float64, device=self.dev)
        Ww, Hw = self.work_size
        s = self.stream.cuda_stream if stream is None else stream
        _lib.check(self.lib.sv_predict_confidence(
            self.net.handle, self.W, self.H, Ww, Hw, self.probe_width, self.max_width,
            _ptr(self.pws), self.pneed, _ptr(self.spread), _ptr(self.pmax), s),
            "predict_confidence")
        return self.spread, self.pmax

    def refine(self, stream=None) -> None:
        self.refiner.run(self.left, self.right, self.disp0, self.out, self.status,
                         self.stream.cuda_stream if stream is None else stream)

    def run_device(self, stream=None) -> None:
        """predict_auto + lr_refine on the images already in self.left/right
        (on self.stream unless a stream handle is given), one library call:
        the refinement launches follow the last work-width read directly."""
        s = self.stream.cuda_stream if stream is None else stream
        r = self.refiner
        _lib.check(self.lib.sv_predict_refine(
            self.net.handle, _ptr(self.left), _ptr(self.right), self.code, self.W, self.H,
            self.tp, self.probe_width, self.max_width, self.passes, self.precision,
            _ptr(self.disp0), _ptr(self.disp_work), ctypes.byref(self._Ww),
            ctypes.byref(self._Hw), self._trace, _ptr(self.pws), self.pneed, r.tol,
            ctypes.byref(r.p), _ptr(self.out), _ptr(self.status), _ptr(r.ws), r.need, s),
            "predict_refine")

    def run_host(self, left: torch.Tensor, right: torch.Tensor):
        """End to end from pinned host images: H2D, the path, D2H of the
        refined disparity and status, all on self.stream.  Returns the pinned
        host tensors."""
        with torch.cuda.stream(self.stream):
            self.left.copy_(left, non_blocking=True)
            self.right.copy_(right, non_blocking=True)
            self.run_device()
            self.h_out.copy_(self.out, non_blocking=True)
            self.h_status.copy_(self.status, non_blocking=True)
        self.stream.synchronize()
        return self.h_out, self.h_status

    @property
    def work_size(self):
        return self._Ww.value, self._Hw.value

    @property
    def work_trace(self):
        return [int(t) for t in self._trace if t > 0]

    def h2d_bytes(self) -> int:
        return 2 * self.left.numel() * self.left.element_size()

    def d2h_bytes(self) -> int:
        return self.out.numel() * 8 + self.status.numel()
