"""StereoNet training on the GPU.

``Trainer`` keeps the parameters, the gradient and Adam's state in device
memory and runs ``train_grads`` (stereonet.py:1619-1653) over a batch of
crops in one call, the batch gradient being the mean of the per-sample
gradients -- what the reference's harness computes with one CPU process per
sample and a pickle round trip per step (train_parallel.py:129-156) -- and
then ``Adam.step`` (1368-1387) on the device.

``train_grads(net, sample)`` and ``train_step(net, opt, sample)`` are
drop-ins with the reference's signatures: ``net`` is the reference's
``StereoNet``, ``sample`` its dict (left, right, disp, valid, W, H); the
gradient is left in the network's own gradient lists (so the reference's
``Adam.step`` and ``flat_grads`` see it) and the return value is the
reference's ``(total, prediction, targets)``.  Arithmetic is FP32 with FP64
weight-gradient sums; the result agrees with the FP64 reference to the
tolerance the tests state, not bit for bit.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .network import _weights_of
from .refine import _device, _ptr, _stream


class Trainer:
    """Device-resident StereoNet trainer (one per network and device)."""

    def __init__(self, net, lr: float = 1.0e-3):
        self.lib = _lib.load()
        w = _weights_of(net)
        self.arch = w.arch
        vec = (ctypes.c_int * len(w.arch.vector()))(*w.arch.vector())
        flat = np.ascontiguousarray(w.flat, dtype=np.float64)
        h = ctypes.c_void_p()
        _lib.check(self.lib.sv_trainer_create(vec, len(w.arch.vector()),
                                              flat.ctypes.data_as(ctypes.c_void_p), flat.size,
                                              ctypes.byref(h)), "sv_trainer_create")
        self.handle = h
        self.n = int(flat.size)
        self.lr = lr
        self._ws = None
        self._ws_key = None

    def __del__(self):
        try:
            if self.handle:
                self.lib.sv_trainer_destroy(self.handle)
        except Exception:
            pass

    # ---------------------------------------------------------- state
    def params(self) -> np.ndarray:
        out = np.zeros(self.n)
        _lib.check(self.lib.sv_trainer_get_params(self.handle, out.ctypes.data_as(ctypes.c_void_p),
                                                  self.n), "get_params")
        return out

    def grads(self) -> np.ndarray:
        out = np.zeros(self.n)
        _lib.check(self.lib.sv_trainer_get_grads(self.handle, out.ctypes.data_as(ctypes.c_void_p),
                                                 self.n), "get_grads")
        return out

    def set_params(self, flat) -> None:
        a = np.ascontiguousarray(np.asarray(flat, dtype=np.float64).ravel())
        _lib.check(self.lib.sv_trainer_set_params(self.handle, a.ctypes.data_as(ctypes.c_void_p),
                                                  a.size), "set_params")

    def reset_adam(self) -> None:
        _lib.check(self.lib.sv_trainer_reset_adam(self.handle), "reset_adam")

    def blocks(self):
        """The parameters split into all_params() blocks (FP64)."""
        flat = self.params()
        out, k = [], 0
        for n in self.arch.block_sizes():
            out.append(flat[k:k + n])
            k += n
        return out

    # ---------------------------------------------------------- steps
    def _workspace(self, B, W, H):
        key = (B, W, H)
        if self._ws_key != key:
            need = self.lib.sv_train_workspace_size(self.handle, B, W, H)
            if need == 0:
                _lib.raise_last("train workspace")
            self._ws = torch.empty(need, dtype=torch.uint8, device=_device())
            self._ws_key = key
        return self._ws

    def compute_grads(self, left, right, disp, valid, pred: bool = False):
        """train_grads over a batch: tensors (or arrays) [B][H][W]; returns
        the per-sample losses (device FP64 [B]) and, if asked, the
        full-resolution predictions (device FP32 [B][H][W])."""
        dev = _device()
        l = torch.as_tensor(left, dtype=torch.float32).to(dev).contiguous()
        r = torch.as_tensor(right, dtype=torch.float32).to(dev).contiguous()
        d = torch.as_tensor(disp, dtype=torch.float32).to(dev).contiguous()
        v = torch.as_tensor(valid).to(dev).to(torch.uint8).contiguous()
        if l.dim() == 2:
            l, r, d, v = l[None], r[None], d[None], v[None]
        B, H, W = l.shape
        for t in (r, d, v):
            if tuple(t.shape) != (B, H, W):
                raise ValueError("left, right, disp and valid must all be [B][H][W]")
        ws = self._workspace(B, W, H)
        loss = torch.empty(B, dtype=torch.float64, device=dev)
        out = torch.empty((B, H, W), dtype=torch.float32, device=dev) if pred else None
        _lib.check(self.lib.sv_train_grads(self.handle, _ptr(l), _ptr(r), _ptr(d), _ptr(v), B, W,
                                           H, _ptr(loss), _ptr(out), _ptr(ws), ws.numel(),
                                           ctypes.c_void_p(_stream())), "train_grads")
        return (loss, out) if pred else loss

    def adam(self, lr: float | None = None, clip: float = 5.0) -> None:
        _lib.check(self.lib.sv_train_adam(self.handle, float(self.lr if lr is None else lr),
                                          float(clip), ctypes.c_void_p(_stream())), "adam")

    def step(self, left, right, disp, valid, lr: float | None = None):
        """One optimiser step on a batch (train_step, with the harness's
        batch averaging); returns the per-sample losses (device)."""
        loss = self.compute_grads(left, right, disp, valid)
        self.adam(lr)
        return loss


# ------------------------------------------------------------ drop-ins
_trainers: dict = {}


def _trainer_for(net) -> Trainer:
    w = _weights_of(net)
    key = (id(net), torch.cuda.current_device())
    t = _trainers.get(key)
    if t is None or t.arch != w.arch:
        t = Trainer(w)
        _trainers[key] = t
    else:
        t.set_params(w.flat)
    return t


def build_targets(sample):
    """stereonet.py:1595-1611 (pool_disp 1572, pool_valid 1579, avgpool2
    979) with the reference's FP64 arithmetic, as its lists."""
    W, H = sample["W"], sample["H"]

    def pool(img, w, h):
        a = np.asarray(img, dtype=np.float64).reshape(h, w)[: h // 2 * 2, : w // 2 * 2]
        return 0.25 * (((a[0::2, 0::2] + a[0::2, 1::2]) + a[1::2, 0::2]) + a[1::2, 1::2])

    def pool_valid(v, w, h):
        a = np.asarray(v, dtype=bool).reshape(h, w)[: h // 2 * 2, : w // 2 * 2]
        return a[0::2, 0::2] & a[0::2, 1::2] & a[1::2, 0::2] & a[1::2, 1::2]

    d_full, v_full, g_full = sample["disp"], sample["valid"], sample["left"]
    W2, H2 = W // 2, H // 2
    W4, H4 = W2 // 2, H2 // 2
    d_half = pool(d_full, W, H) * 0.5
    v_half = pool_valid(v_full, W, H)
    g_half = pool(g_full, W, H)
    d_qtr = pool(d_half, W2, H2) * 0.5
    v_qtr = pool_valid(v_half, W2, H2)
    return {"d": [d_qtr.ravel().tolist(), d_half.ravel().tolist(), list(d_full)],
            "v": [v_qtr.ravel().tolist(), v_half.ravel().tolist(), list(v_full)],
            "guide_half": g_half.ravel().tolist(), "guide_full": list(g_full),
            "dims": [(W4, H4), (W2, H2), (W, H)]}


def train_grads(net, sample):
    """stereonet.py:1619-1653 on the GPU: gradients into the network's own
    gradient lists; returns (total loss, full-resolution prediction,
    targets)."""
    W, H = int(sample["W"]), int(sample["H"])
    t = _trainer_for(net)
    loss, pred = t.compute_grads(np.asarray(sample["left"], dtype=np.float32).reshape(H, W),
                                 np.asarray(sample["right"], dtype=np.float32).reshape(H, W),
                                 np.asarray(sample["disp"], dtype=np.float32).reshape(H, W),
                                 np.asarray(sample["valid"], dtype=bool).reshape(H, W),
                                 pred=True)
    g = t.grads()
    if hasattr(net, "all_params"):
        k = 0
        for _, gl in net.all_params():
            n = len(gl)
            gl[:] = g[k:k + n].tolist()
            k += n
    return float(loss[0]), pred[0].double().reshape(-1).cpu().tolist(), build_targets(sample)


def train_step(net, opt, sample):
    """stereonet.py:1656-1659: train_grads, then the caller's optimiser."""
    total, pred, tgt = train_grads(net, sample)
    opt.step()
    return total, pred, tgt
