"""Drop-ins for the StereoNet forward and resolution selection of stereonet.py.

    resize_gray(img, W, H, W2, H2)                                 (3843-3845)
    avgpool2(img, C, H, W)                                         (979-995)
    forward(net, left, right, H, W, guide_half, guide_full)        (1203-1233)
    predict(net, left, right, W, H)                                (5891-5897)
    predict_at_scale(net, left, right, W, H, work_width=96, verbose=True)
    predict_auto(net, left, right, W, H, target_peak=None, probe_width=64,
                 max_width=320, passes=3, verbose=True)             (3872-3929)

``net`` is either a checkpoint from ``weights.load_model`` or the
reference's own ``StereoNet`` object (its parameters are read through
``all_params()``).  The weights are uploaded once per object and reused.
The network runs in FP32 on the GPU (convolutions accumulate in FP32,
soft-argmin in FP32 with max subtraction); resampling runs in FP64 like the
reference.  Outputs follow the reference's return types: lists for list
inputs, numpy for numpy, CUDA tensors for tensors.
"""

from __future__ import annotations

import ctypes
import weakref

import numpy as np
import torch

from . import _lib
from .refine import _device, _image, _kind, _ptr, _ret, _stream, _to_dev
from .weights import NetArch, StereoNetWeights


class GpuNet:
    """One checkpoint uploaded to the current device (sv_net)."""

    def __init__(self, w: StereoNetWeights):
        self.lib = _lib.load()
        self.weights = w
        arch = (ctypes.c_int * len(w.arch.vector()))(*w.arch.vector())
        flat = np.ascontiguousarray(w.flat, dtype=np.float64)
        h = ctypes.c_void_p()
        _lib.check(self.lib.sv_net_create(arch, len(w.arch.vector()),
                                          flat.ctypes.data_as(ctypes.c_void_p), flat.size,
                                          ctypes.byref(h)), "sv_net_create")
        self.handle = h
        self.target_peak = w.target_peak
        self.D = w.arch.D

    def __del__(self):
        try:
            if self.handle:
                self.lib.sv_net_destroy(self.handle)
        except Exception:
            pass


_cache: "weakref.WeakKeyDictionary" = weakref.WeakKeyDictionary()
_cache_by_id: dict = {}


def _weights_of(net) -> StereoNetWeights:
    if isinstance(net, StereoNetWeights):
        return net
    if hasattr(net, "all_params"):          # the reference's StereoNet
        arch = NetArch(feat_C=int(net.feat_C), cost_C=int(net.filt.c1.oc), D=int(net.D),
                       max_disp=int(getattr(net, "max_disp", 32)),
                       refine_C=int(net.ref1.convs[0].oc),
                       refine_dil=tuple(int(d) for d in net.ref1.dilations),
                       target_peak=int(getattr(net, "target_peak", 20)))
        blocks = [np.asarray(p, dtype=np.float64) for p, _ in net.all_params()]
        return StereoNetWeights(arch, blocks)
    raise TypeError("net must be a StereoNetWeights or a reference StereoNet")


def gpu_net(net) -> GpuNet:
    """The uploaded copy of ``net`` (re-uploaded if its parameters changed)."""
    if isinstance(net, GpuNet):
        return net
    w = _weights_of(net)
    key = (id(net), torch.cuda.current_device())
    fp = hash(w.flat.tobytes())
    hit = _cache_by_id.get(key)
    if hit is not None and hit[0] == fp:
        return hit[1]
    g = GpuNet(w)
    _cache_by_id[key] = (fp, g)
    return g


# ------------------------------------------------------------ resampling
def resize_gray(img, W, H, W2, H2):
    """stereonet.py:3843-3845 (FP64 on the GPU, bit-identical)."""
    lib = _lib.load()
    t = _to_dev(img, W * H, torch.float64, name="img")
    out = torch.empty(W2 * H2, dtype=torch.float64, device=t.device)
    _lib.check(lib.sv_resize(_ptr(t), W, H, W2, H2, _ptr(out), _stream()), "resize_gray")
    return _ret(out, img)


def avgpool2(img, C, H, W):
    """stereonet.py:979-995 -> (pooled, H//2, W//2), FP64, bit-identical."""
    lib = _lib.load()
    t = _to_dev(img, C * H * W, torch.float64, name="img")
    out = torch.empty(C * (H // 2) * (W // 2), dtype=torch.float64, device=t.device)
    _lib.check(lib.sv_avgpool2(_ptr(t), C, H, W, _ptr(out), _stream()), "avgpool2")
    return _ret(out, img), H // 2, W // 2


# --------------------------------------------------------------- forward
def _f32(x, n, name):
    return _to_dev(x, n, torch.float32, name=name)


def _precision(precision) -> int:
    """"fp32" (default) or "bf16": FeatureNet and CostFilter c1/c2 as BF16
    tensor-core GEMMs with FP32 accumulation (soft-argmin and Refinement stay
    FP32).  In predict_auto BF16 applies to the last permitted pass only --
    the one no work-width decision follows -- so the widths are FP32's."""
    codes = {"fp32": _lib.SV_FP32, "bf16": _lib.SV_BF16, _lib.SV_FP32: _lib.SV_FP32,
             _lib.SV_BF16: _lib.SV_BF16}
    if precision not in codes:
        raise ValueError("precision must be 'fp32' or 'bf16', not %r" % (precision,))
    return codes[precision]


def _flag_check(lib, ws, code, what):
    """BF16 kernels report a stalled tensor-core wait through the workspace flag."""
    if code == _lib.SV_BF16:
        _lib.check(lib.sv_workspace_status(_ptr(ws), ctypes.c_void_p(_stream())), what)


def forward(net, left, right, H, W, guide_half, guide_full, *, precision="fp32"):
    """StereoNet.forward (stereonet.py:1203-1233): (d_quarter, d_half, d_full)."""
    code = _precision(precision)
    g = gpu_net(net)
    lib = g.lib
    h1, w1 = (H - 1) // 2 + 1, (W - 1) // 2 + 1
    h, w = (h1 - 1) // 2 + 1, (w1 - 1) // 2 + 1
    tl, tr = _f32(left, H * W, "left"), _f32(right, H * W, "right")
    gh = _f32(guide_half, (H // 2) * (W // 2), "guide_half")
    gf = _f32(guide_full, H * W, "guide_full")
    dev = tl.device
    d0 = torch.empty(h * w, dtype=torch.float32, device=dev)
    d1 = torch.empty((H // 2) * (W // 2), dtype=torch.float32, device=dev)
    d2 = torch.empty(H * W, dtype=torch.float32, device=dev)
    need = lib.sv_forward_workspace_size(g.handle, H, W)
    ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    _lib.check(lib.sv_stereonet_forward(g.handle, _ptr(tl), _ptr(tr), H, W, _ptr(gh), _ptr(gf),
                                        _ptr(d0), _ptr(d1), _ptr(d2), code, _ptr(ws),
                                        need, _stream()), "forward")
    _flag_check(lib, ws, code, "forward")
    return tuple(_ret(d.to(torch.float64), left) for d in (d0, d1, d2))


def predict(net, left, right, W, H, *, precision="fp32"):
    """stereonet.py:5891-5897: full-resolution disparity of the network
    (guide_half = avgpool2(left), guide_full = left)."""
    return predict_at_scale(net, left, right, W, H, work_width=W, verbose=False,
                            precision=precision)[0]


# ------------------------------------------------- resolution selection
def _pair_inputs(left, right, W, H):
    tl, code = _image(left, W * H, "left")
    tr, code_r = _image(right, W * H, "right")
    if code_r != code:
        tr = tr.to(tl.dtype)
    return tl, tr, code


def predict_at_scale(net, left, right, W, H, work_width=96, verbose=True, *, precision="fp32"):
    """stereonet.py:3932-3960 -> (disp_full, disp_work, W_work, H_work)."""
    code_p = _precision(precision)
    g = gpu_net(net)
    lib = g.lib
    tl, tr, code = _pair_inputs(left, right, W, H)
    dev = tl.device
    df = torch.empty(W * H, dtype=torch.float64, device=dev)
    dw = torch.empty(max(W * H, 64 * 64), dtype=torch.float64, device=dev)
    need = lib.sv_predict_workspace_size(g.handle, W, H, max(int(work_width), 48))
    ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    Ww, Hw = ctypes.c_int(), ctypes.c_int()
    _lib.check(lib.sv_predict_at_scale(g.handle, _ptr(tl), _ptr(tr), code, W, H, int(work_width),
                                       code_p, _ptr(df), _ptr(dw), ctypes.byref(Ww),
                                       ctypes.byref(Hw), _ptr(ws), need, _stream()),
               "predict_at_scale")
    _flag_check(lib, ws, code_p, "predict_at_scale")
    if verbose and work_width < W:
        print("  running at %dx%d (input %dx%d, scale %.3f)"
              % (Ww.value, Hw.value, W, H, work_width / float(W)))
    dwv = dw[:Ww.value * Hw.value]
    return _ret(df, left), _ret(dwv, left), Ww.value, Hw.value


def _peak(disp, q=0.95):
    """stereonet.py:3866-3869: sorted(disp)[int(len(disp) * q)], at least
    0.5 -- an exact radix select on the GPU."""
    lib = _lib.load()
    d = disp if isinstance(disp, torch.Tensor) else np.asarray(disp, dtype=np.float64)
    n = int(d.numel() if isinstance(d, torch.Tensor) else d.size)
    t = _to_dev(d, n, torch.float64, name="disp")
    out = torch.empty(1, dtype=torch.float64, device=t.device)
    need = lib.sv_peak_workspace_size()
    ws = torch.empty(need, dtype=torch.uint8, device=t.device)
    _lib.check(lib.sv_peak(_ptr(t), n, float(q), _ptr(out), _ptr(ws), need, _stream()), "_peak")
    return float(out.item())


def work_width(disp, W, target_peak, max_width=320, scale=1.0):
    """The work width predict_auto takes from a map (stereonet.py:3866-3869
    and 3915-3919): int(W * target_peak / max(p, 1e-6) + 0.5) clamped to
    [48, min(W, max_width)], p = max(sorted(disp)[int(n * 0.95)], 0.5) *
    scale -- decided on the GPU from a histogram of the rule's per-value
    widths, as predict_auto decides it."""
    lib = _lib.load()
    d = disp if isinstance(disp, torch.Tensor) else np.asarray(disp, dtype=np.float64)
    n = int(d.numel() if isinstance(d, torch.Tensor) else d.size)
    t = _to_dev(d, n, torch.float64, name="disp")
    need = lib.sv_peak_workspace_size()
    ws = torch.empty(need, dtype=torch.uint8, device=t.device)
    w = ctypes.c_int()
    _lib.check(lib.sv_work_width(_ptr(t), n, int(W), float(target_peak), int(max_width),
                                 float(scale), ctypes.byref(w), _ptr(ws), need, _stream()),
               "work_width")
    return w.value


def predict_auto(net, left, right, W, H, target_peak=None, probe_width=64, max_width=320,
                 passes=3, verbose=True, return_trace=False, *, precision="fp32"):
    """stereonet.py:3872-3929 -> (disp_full, disp_work, W_work, H_work).

    The work width depends on each pass's 95% disparity quantile, so the
    call reads one number back from the GPU per pass."""
    code_p = _precision(precision)
    g = gpu_net(net)
    lib = g.lib
    tp = float(g.target_peak if target_peak is None else target_peak)
    tl, tr, code = _pair_inputs(left, right, W, H)
    dev = tl.device
    df = torch.empty(W * H, dtype=torch.float64, device=dev)
    dw = torch.empty(max(W * H, 64 * 64), dtype=torch.float64, device=dev)
    need = lib.sv_predict_workspace_size(g.handle, W, H, int(max_width))
    ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    Ww, Hw = ctypes.c_int(), ctypes.c_int()
    trace = (ctypes.c_int * (passes + 2))()
    _lib.check(lib.sv_predict_auto(g.handle, _ptr(tl), _ptr(tr), code, W, H, tp,
                                   int(probe_width), int(max_width), int(passes), code_p,
                                   _ptr(df), _ptr(dw), ctypes.byref(Ww), ctypes.byref(Hw), trace,
                                   _ptr(ws), need, _stream()), "predict_auto")
    _flag_check(lib, ws, code_p, "predict_auto")
    widths = [int(t) for t in trace if t > 0]
    if verbose:
        for i, wd in enumerate(widths):
            print("  %s work width %d" % ("probe chose" if i == 0 else "rescaled to", wd))
    res = (_ret(df, left), _ret(dw[:Ww.value * Hw.value], left), Ww.value, Hw.value)
    if return_trace:
        return res, widths
    return res


# ----------------------------------------- network-level LR consistency
def predict_consistent(net, left, right, W, H, work_width=None, tol=1.5, verbose=True, *,
                       precision="fp32"):
    """stereonet.py:5048-5076 -> (disparity, valid fraction): the network on
    the pair and on the mirrored pair at the same work width, the left-right
    check and the row fill of the rejected pixels."""
    code_p = _precision(precision)
    g = gpu_net(net)
    lib = g.lib
    tl, tr, code = _pair_inputs(left, right, W, H)
    dev = tl.device
    mw = 320 if work_width is None else max(int(work_width), 48)
    need = lib.sv_predict_consistent_workspace_size(g.handle, W, H, code, mw)
    if need == 0:
        raise ValueError("predict_consistent: bad shape")
    ws = torch.empty(need, dtype=torch.uint8, device=dev)
    out = torch.empty(W * H, dtype=torch.float64, device=dev)
    kept = ctypes.c_longlong()
    _lib.check(lib.sv_predict_consistent(g.handle, _ptr(tl), _ptr(tr), code, W, H,
                                         0 if work_width is None else int(work_width),
                                         float(g.target_peak), 64, 320, 3, float(tol), code_p,
                                         _ptr(out), ctypes.byref(kept), _ptr(ws), need,
                                         _stream()), "predict_consistent")
    frac = kept.value / float(W * H)
    if verbose:
        print("  left-right consistency: %.1f%% of pixels agree within %.1f px"
              % (100.0 * frac, tol))
    return _ret(out, left), frac
