"""lr_refine over many pairs of uneven sizes at once (sv_batch_lr_refine).

``lr_refine_batch(pairs, tol=1.0, **kw)`` takes a list of
``(left, right, disp0, W, H)`` tuples with the reference's argument meaning
(stereonet.py:5343-5391) and returns a list of ``(disparity, status)``, each
bit-identical to ``refine.lr_refine`` on that pair alone.  ``BatchRefiner``
is the device-resident form: the images, disparities and outputs stay in
HBM and one call enqueues the whole batch (seven launches; the SGM stage is
a persistent kernel over a device-side queue of scanline tasks).

``BatchRefiner.autotune()`` picks the batch's scheduling (pixels per CTA of
the per-pixel stages, the persistent SGM kernel's CTA size, CTAs per SM and
tasks per queue fetch) by timing the batch itself, one knob at a time from
the defaults, and remembers the choice per device, band and batch shape in
a small JSON file (``$SV_B200_CACHE`` or ``~/.cache/sv_b200``).  Every
configuration gives the same bits; only the time changes.

``NetBatch`` puts the network in front: predict_auto (stereonet.py:
3872-3929) for every pair, with the work-width decisions taken on the
device, then the same batched lr_refine, as one launch sequence that a CUDA
graph replays (sv_netbatch_*).  Each pair's network disparity, work-width
trace and refined output equal predict_auto + lr_refine on that pair alone.
"""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import torch

from . import _lib
from .refine import _device, _image, _kind, _params, _ptr, _ret, _stream, _to_dev, _finite_disp


class PairDesc(ctypes.Structure):
    _fields_ = [("left", ctypes.c_void_p), ("right", ctypes.c_void_p),
                ("disp0", ctypes.c_void_p), ("out", ctypes.c_void_p),
                ("status", ctypes.c_void_p), ("W", ctypes.c_int), ("H", ctypes.c_int)]


class BatchConfig(ctypes.Structure):
    """sv_batch_config: the batched refinement's scheduling."""
    _fields_ = [("px_per_block", ctypes.c_int), ("sgm_threads", ctypes.c_int),
                ("sgm_ctas_per_sm", ctypes.c_int), ("sgm_fetch", ctypes.c_int)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}

    @classmethod
    def from_dict(cls, d):
        return cls(*(int(d[k]) for k, _ in cls._fields_))


def default_config() -> BatchConfig:
    c = BatchConfig()
    _lib.load().sv_batch_config_default(ctypes.byref(c))
    return c


# candidate values per knob, tried one knob at a time
TUNE_SPACE = {"px_per_block": (512, 1024, 2048, 4096),
              "sgm_threads": (64, 128, 256),
              "sgm_ctas_per_sm": (4, 8, 16),
              "sgm_fetch": (32, 64)}


def _cache_path() -> str:
    root = os.environ.get("SV_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache",
                                                            "sv_b200")
    return os.path.join(root, "batch_tune.json")


class BatchRefiner:
    """lr_refine for a fixed list of (W, H) sizes; buffers allocated once."""

    def __init__(self, sizes, dtype=torch.uint8, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                 paths=8, uniq=0.0, config: BatchConfig | None = None):
        self.lib = _lib.load()
        self.config = config if config is not None else default_config()
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
        _lib.check(self.lib.sv_batch_lr_refine_ex(self.descs, len(self.sizes), self.code,
                                                  self.tol, ctypes.byref(self.p),
                                                  ctypes.byref(self.config), _ptr(self.ws),
                                                  self.need,
                                                  _stream() if stream is None else stream),
                   "lr_refine_batch")

    def _key(self) -> str:
        props = torch.cuda.get_device_properties(torch.cuda.current_device())
        mpix = self.pixels / 1e6
        bucket = 1 << max(0, int(np.ceil(np.log2(max(mpix, 1e-6)))) + 20)   # pixels, next 2^k
        return "%s|sm%d|R%d|paths%d|n%d|px%d" % (props.name, props.multi_processor_count,
                                                 self.p.R, self.p.paths, len(self.sizes), bucket)

    def time_config(self, cfg: BatchConfig, reps: int = 3) -> float:
        """Median device milliseconds of one batched call with `cfg`."""
        old = self.config
        self.config = cfg
        try:
            self.run()
            times = []
            for _ in range(reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                self.run()
                e1.record()
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            return float(np.median(times))
        finally:
            self.config = old

    def autotune(self, reps: int = 3, use_cache: bool = True) -> dict:
        """Pick the scheduling by timing this batch (the buffers' current
        contents are used as they are); returns the choice and its times."""
        key = self._key()
        path = _cache_path()
        cache = {}
        if use_cache and os.path.exists(path):
            try:
                with open(path) as f:
                    cache = json.load(f)
            except (OSError, ValueError):
                cache = {}
        if use_cache and key in cache:
            self.config = BatchConfig.from_dict(cache[key]["config"])
            return dict(cache[key], cached=True)
        best = default_config()
        best_ms = self.time_config(best, reps)
        base_ms = best_ms
        tried = {json.dumps(best.as_dict(), sort_keys=True): best_ms}
        for knob, values in TUNE_SPACE.items():
            for v in values:
                cand = BatchConfig.from_dict(dict(best.as_dict(), **{knob: v}))
                k = json.dumps(cand.as_dict(), sort_keys=True)
                if k not in tried:
                    tried[k] = self.time_config(cand, reps)
                if tried[k] < best_ms:
                    best, best_ms = cand, tried[k]
        self.config = best
        entry = {"config": best.as_dict(), "ms": best_ms, "default_ms": base_ms,
                 "candidates": len(tried)}
        if use_cache:
            try:
                os.makedirs(os.path.dirname(path), exist_ok=True)
                cache[key] = entry
                with open(path, "w") as f:
                    json.dump(cache, f, indent=1, sort_keys=True)
            except OSError:
                pass
        return dict(entry, cached=False)

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


class NetBatch:
    """predict_auto + lr_refine for a fixed list of (W, H) sizes, on the
    device end to end.  ``left``/``right`` (images) and ``out``/``status``
    (refined disparity and left-right status) are per-pair device buffers
    allocated once; ``run()`` enqueues the whole batch on the current stream
    (the first run records a CUDA graph, later runs replay it)."""

    def __init__(self, sizes, net, dtype=torch.uint8, target_peak=None, probe_width=64,
                 max_width=320, passes=3, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                 paths=8, uniq=0.0):
        from . import network
        self.lib = _lib.load()
        self.g = network.gpu_net(net)
        self.sizes = [(int(W), int(H)) for W, H in sizes]
        self.passes = int(passes)
        self.p = _params(R=R, P1=P1, P2=P2, rx=rx, ry=ry, paths=paths, uniq=uniq)
        self.code = {torch.uint8: _lib.SV_U8, torch.float32: _lib.SV_F32,
                     torch.float64: _lib.SV_F64}[dtype]
        n = len(self.sizes)
        Ws = (ctypes.c_int * n)(*[W for W, _ in self.sizes])
        Hs = (ctypes.c_int * n)(*[H for _, H in self.sizes])
        tp = float(self.g.target_peak if target_peak is None else target_peak)
        h = ctypes.c_void_p()
        _lib.check(self.lib.sv_netbatch_create(self.g.handle, Ws, Hs, n, self.code, tp,
                                               int(probe_width), int(max_width), self.passes,
                                               _lib.SV_FP32, float(tol), ctypes.byref(self.p),
                                               ctypes.byref(h)), "sv_netbatch_create")
        self.handle = h
        dev = _device()
        self.left = [torch.empty(W * H, dtype=dtype, device=dev) for W, H in self.sizes]
        self.right = [torch.empty(W * H, dtype=dtype, device=dev) for W, H in self.sizes]
        self.out = [torch.empty(W * H, dtype=torch.float64, device=dev) for W, H in self.sizes]
        self.status = [torch.empty(W * H, dtype=torch.uint8, device=dev) for W, H in self.sizes]
        self.descs = (PairDesc * n)()
        for i, (W, H) in enumerate(self.sizes):
            self.descs[i] = PairDesc(self.left[i].data_ptr(), self.right[i].data_ptr(), None,
                                     self.out[i].data_ptr(), self.status[i].data_ptr(), W, H)
        self.need = self.lib.sv_netbatch_workspace_size(self.handle)
        self.ws = torch.empty(self.need, dtype=torch.uint8, device=dev)
        _lib.check(self.lib.sv_netbatch_bind(self.handle, self.descs, _ptr(self.ws), self.need,
                                             _stream()), "sv_netbatch_bind")

    def __del__(self):
        try:
            if self.handle:
                self.lib.sv_netbatch_destroy(self.handle)
        except Exception:
            pass

    @property
    def pixels(self) -> int:
        return sum(W * H for W, H in self.sizes)

    def run(self, stream=None) -> None:
        """predict_auto + lr_refine of every pair (enqueued only)."""
        _lib.check(self.lib.sv_netbatch_run(self.handle, _stream() if stream is None else stream),
                   "sv_netbatch_run")

    def predict(self, stream=None) -> None:
        """predict_auto of every pair (enqueued only)."""
        _lib.check(self.lib.sv_netbatch_predict(self.handle,
                                                _stream() if stream is None else stream),
                   "sv_netbatch_predict")

    def disparity(self, i: int) -> torch.Tensor:
        """Pair i's network disparity (FP64, W*H), a view into the workspace."""
        ptr = ctypes.c_void_p()
        _lib.check(self.lib.sv_netbatch_disparity(self.handle, i, ctypes.byref(ptr)),
                   "sv_netbatch_disparity")
        W, H = self.sizes[i]
        off = ptr.value - self.ws.data_ptr()
        return self.ws[off:off + 8 * W * H].view(torch.float64)

    def traces(self):
        """[(widths chosen, (Ww, Hw)), ...] per pair (synchronises)."""
        n = len(self.sizes)
        tl = self.passes + 2
        tr = (ctypes.c_int * (n * tl))()
        ws = (ctypes.c_int * (2 * n))()
        _lib.check(self.lib.sv_netbatch_trace(self.handle, tr, tl, ws, _stream()),
                   "sv_netbatch_trace")
        res = []
        for i in range(n):
            t = [int(v) for v in tr[i * tl:(i + 1) * tl]]
            res.append(([v for v in t if v > 0], (int(ws[2 * i]), int(ws[2 * i + 1]))))
        return res

    def data_status(self) -> None:
        _lib.check(self.lib.sv_netbatch_data_status(self.handle, ctypes.c_void_p(_stream())),
                   "sv_netbatch_run")
