"""Drop-ins for the full-resolution refinement of stereonet.py (5115-5391).

Every function keeps the reference's name, signature, argument meaning and
return shape, and runs on the GPU through libsv_b200.so:

    census(img, W, H, rx=2, ry=2)                       -> list[int]
    band_costs(cl, cr, gl, gr, base, W, H, R, ad_weight, ad_trunc, invalid,
               prior=None, prior_w=0.0, prior_t=4.0)     -> list[float]
    _aggregate_path(C, base, W, H, K, P1, P2, dx, dy, S) -> None (S += L)
    refine_fullres(left, right, disp0, W, H, R=3, P1=1.0, P2=12.0, ...)
    left_to_right(dl, W, H)                              -> list[float]
    lr_refine(left, right, disp0, W, H, tol=1.0, **kw)   -> (list, list[int])

Inputs may be the reference's flat Python lists, numpy arrays or torch
tensors (CPU or CUDA).  Lists come back as lists, numpy as numpy, tensors as
tensors on the input's device.  Images are compared exactly as given: float
grays in FP64 (the reference's values), uint8 images as integers (the same
order as u/255.0).  Parameters the exact integer path cannot honour
(ad_weight != 0, a prior, non-integer P1/P2) raise ValueError rather than
fall back to anything; so do NaN or infinite disparities, as the reference's
int() does.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

_TORCH_CODE = {torch.uint8: _lib.SV_U8, torch.float32: _lib.SV_F32,
               torch.float64: _lib.SV_F64}
_NP_CODE = {np.dtype(np.uint8): _lib.SV_U8, np.dtype(np.float32): _lib.SV_F32,
            np.dtype(np.float64): _lib.SV_F64}


def sgm_kernel_name(K: int = 21) -> str:
    """Name of the single-pair SGM kernel the library runs for a band of K
    (the library reads SV_SGM_KERNEL = group8 | group4 | thread once)."""
    import os
    Kp = next((k for k in (8, 16, 24, 32) if k >= K + 2), None)
    if Kp is None:
        return "k_sgm_packed"
    v = os.environ.get("SV_SGM_KERNEL", "group8")
    if v == "thread":
        return "k_sgm_thread"
    sl = 4 if v == "group4" else 8
    return "k_sgm_group<%d slots x %d lanes>" % (sl, Kp // sl)


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("the refinement runs on a CUDA device; none is available")
    return torch.device("cuda", torch.cuda.current_device())


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _kind(x):
    if isinstance(x, torch.Tensor):
        return "torch"
    if isinstance(x, np.ndarray):
        return "numpy"
    return "list"


def _to_dev(x, n, dtype=None, name="array"):
    """Flat contiguous device tensor of n elements (dtype kept unless given)."""
    dev = _device()
    if isinstance(x, torch.Tensor):
        t = x.reshape(-1)
        if dtype is not None:
            t = t.to(dtype)
        t = t.to(dev).contiguous()
    else:
        a = np.asarray(x)
        if dtype is not None:
            a = a.astype(torch.empty(0, dtype=dtype).numpy().dtype, copy=False)
        elif a.dtype == np.uint64:
            a = a.view(np.int64)                   # census words: keep the bits
        elif a.dtype.kind not in "uif":
            a = a.astype(np.float64)
        t = torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to(dev)
    if t.numel() != n:
        raise ValueError("%s has %d elements, expected %d" % (name, t.numel(), n))
    return t


def _image(x, n, name):
    t = _to_dev(x, n, name=name)
    if t.dtype not in _TORCH_CODE:
        t = t.to(torch.float64)
    return t, _TORCH_CODE[t.dtype]


def _ret(t: torch.Tensor, like, as_int=False):
    k = _kind(like)
    if k == "torch":
        return t if like.device.type == "cuda" else t.cpu()
    a = t.cpu().numpy()
    if k == "numpy":
        return a
    return [int(v) for v in a] if as_int else a.tolist()


def _finite_disp(disp0, name="disp0"):
    d = disp0 if isinstance(disp0, torch.Tensor) else np.asarray(disp0, dtype=np.float64)
    ok = bool(torch.isfinite(d).all()) if isinstance(d, torch.Tensor) else bool(np.isfinite(d).all())
    if not ok:
        raise ValueError("%s contains NaN or infinite values (the reference's int() raises)" % name)


def _params(R=3, P1=1.0, P2=12.0, ad_weight=0.0, ad_trunc=20.0, paths=8, uniq=0.0,
            rx=2, ry=2, prior_w=0.0, prior_t=4.0) -> _lib.RefineParams:
    p = _lib.RefineParams()
    p.R, p.P1, p.P2 = int(R), float(P1), float(P2)
    p.rx, p.ry, p.paths = int(rx), int(ry), int(paths)
    p.uniq, p.ad_weight, p.ad_trunc = float(uniq), float(ad_weight), float(ad_trunc)
    # refine_fullres applies the prior only when prior_w > 0 (stereonet.py:5181),
    # but a negative weight still shifts the invalid cost (5261-5262).
    p.prior_w, p.prior_t = float(prior_w), float(prior_t)
    return p


def _workspace(nbytes: int) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=_device())


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _data_status(ws: torch.Tensor, what: str) -> None:
    rc = _lib.load().sv_workspace_status(_ptr(ws), ctypes.c_void_p(_stream()))
    _lib.check(rc, what)


# ------------------------------------------------------------------ census
def census(img, W, H, rx=2, ry=2):
    """stereonet.py:5115-5142 on the GPU; bit-identical signatures."""
    lib = _lib.load()
    t, code = _image(img, W * H, "img")
    out = torch.empty(W * H, dtype=torch.int64, device=t.device)
    _lib.check(lib.sv_census(_ptr(t), code, W, H, rx, ry, _ptr(out), _stream()), "census")
    if _kind(img) == "torch":
        return out
    a = out.cpu().numpy().view(np.uint64)
    return a if _kind(img) == "numpy" else [int(v) for v in a]


def _census_words(c, n, name):
    """Census descriptors (Python ints, uint64 or int64) as a device int64
    tensor holding the same 64 bits."""
    if isinstance(c, torch.Tensor):
        t = c.reshape(-1).to(_device())
        if t.dtype != torch.int64:
            raise ValueError("%s must be an int64 tensor of census words" % name)
        if t.numel() != n:
            raise ValueError("%s has %d elements, expected %d" % (name, t.numel(), n))
        return t.contiguous()
    return _to_dev(np.asarray(c, dtype=np.uint64).view(np.int64), n, name=name)


# -------------------------------------------------------------- band_costs
def band_costs(cl, cr, gl, gr, base, W, H, R, ad_weight, ad_trunc, invalid,
               prior=None, prior_w=0.0, prior_t=4.0):
    """stereonet.py:5156-5189 for ad_weight == 0 and no prior term."""
    if ad_weight != 0.0 or prior_w > 0.0:
        raise ValueError("band_costs on the GPU supports ad_weight == 0 and prior_w <= 0")
    inv = float(invalid)
    if inv != int(inv) or not 0 <= inv <= 255:
        raise ValueError("invalid cost %r must be an integer in 0..255" % invalid)
    lib = _lib.load()
    N, K = W * H, 2 * R + 1
    tl = _census_words(cl, N, "cl")
    tr = _census_words(cr, N, "cr")
    tb = _to_dev(base, N, torch.int32, name="base")
    C = torch.empty(N * K, dtype=torch.uint8, device=tl.device)
    _lib.check(lib.sv_band_costs(_ptr(tl), _ptr(tr), _ptr(tb), W, H, R, int(inv), _ptr(C),
                                 _stream()), "band_costs")
    Cf = C.to(torch.float64)
    if _kind(cl) == "torch":
        return Cf
    a = Cf.cpu().numpy()
    return a if _kind(cl) == "numpy" else a.tolist()


# ---------------------------------------------------------- _aggregate_path
def _aggregate_path(C, base, W, H, K, P1, P2, dx, dy, S):
    """stereonet.py:5192-5241: adds one SGM path into S in place."""
    lib = _lib.load()
    N = W * H
    for name, v in (("P1", P1), ("P2", P2)):
        if float(v) != int(v) or not 0 <= v <= 4096:
            raise ValueError("%s=%r must be an integer in 0..4096 on the GPU" % (name, v))
    Cd = _to_dev(C, N * K, torch.float64, name="C")
    if bool((Cd != torch.round(Cd)).any()) or bool((Cd < 0).any()) or bool((Cd > 255).any()):
        raise ValueError("costs must be integers in 0..255 on the GPU")
    Sd = _to_dev(S, N * K, torch.float64, name="S")
    if bool((Sd != torch.round(Sd)).any()) or bool((Sd < 0).any()) or \
            float(Sd.max()) + float(Cd.max()) + float(P2) > 65535:
        raise ValueError("S must hold integers small enough for 16-bit accumulation")
    Cu = Cd.to(torch.uint8)
    Su = Sd.to(torch.int32).to(torch.int16)        # bit pattern of uint16
    tb = _to_dev(base, N, torch.int32, name="base")
    _lib.check(lib.sv_aggregate_path(_ptr(Cu), _ptr(tb), W, H, K, int(P1), int(P2), int(dx),
                                     int(dy), _ptr(Su), _stream()), "_aggregate_path")
    res = Su.to(torch.int32) & 0xFFFF
    if isinstance(S, torch.Tensor):
        S.copy_(res.to(S.dtype).view(S.shape))
    elif isinstance(S, np.ndarray):
        S[...] = res.cpu().numpy().reshape(S.shape)
    else:
        S[:] = [float(v) for v in res.cpu().numpy()]
    return None


# ---------------------------------------------------------- refine_fullres
def refine_fullres(left, right, disp0, W, H, R=3, P1=1.0, P2=12.0, ad_weight=0.0,
                   ad_trunc=20.0, paths=8, uniq=0.0, rx=2, ry=2, prior_w=0.0,
                   prior_t=4.0, return_conf=False):
    """stereonet.py:5244-5305 on the GPU, bit-identical output."""
    lib = _lib.load()
    N = W * H
    _finite_disp(disp0)
    p = _params(R, P1, P2, ad_weight, ad_trunc, paths, uniq, rx, ry, prior_w, prior_t)
    tl, code = _image(left, N, "left")
    tr, code_r = _image(right, N, "right")
    if code_r != code:
        tr = tr.to(tl.dtype)
    td = _to_dev(disp0, N, torch.float64, name="disp0")
    need = lib.sv_refine_workspace_size(W, H, ctypes.byref(p))
    if need == 0:
        _lib.raise_last("refine_fullres")
    ws = _workspace(need)
    out = torch.empty(N, dtype=torch.float64, device=td.device)
    conf = torch.empty(N, dtype=torch.float64, device=td.device) if return_conf else None
    _lib.check(lib.sv_refine_fullres(_ptr(tl), _ptr(tr), code, _ptr(td), W, H,
                                     ctypes.byref(p), _ptr(out), _ptr(conf), _ptr(ws), need,
                                     _stream()), "refine_fullres")
    _data_status(ws, "refine_fullres")
    if return_conf:
        return _ret(out, left), _ret(conf, left)
    return _ret(out, left)


# ------------------------------------------------------------ left_to_right
def left_to_right(dl, W, H):
    """stereonet.py:5317-5340 on the GPU, bit-identical output."""
    lib = _lib.load()
    _finite_disp(dl, "dl")
    td = _to_dev(dl, W * H, torch.float64, name="dl")
    dr = torch.empty_like(td)
    _lib.check(lib.sv_left_to_right(_ptr(td), W, H, _ptr(dr), _stream()), "left_to_right")
    return _ret(dr, dl)


# ---------------------------------------------------------------- lr_refine
def lr_refine(left, right, disp0, W, H, tol=1.0, **kw):
    """stereonet.py:5343-5391 on the GPU: (disparity, status), bit-identical."""
    lib = _lib.load()
    N = W * H
    _finite_disp(disp0)
    p = _params(**kw)
    tl, code = _image(left, N, "left")
    tr, code_r = _image(right, N, "right")
    if code_r != code:
        tr = tr.to(tl.dtype)
    td = _to_dev(disp0, N, torch.float64, name="disp0")
    need = lib.sv_lr_refine_workspace_size(W, H, ctypes.byref(p))
    if need == 0:
        _lib.raise_last("lr_refine")
    ws = _workspace(need)
    out = torch.empty(N, dtype=torch.float64, device=td.device)
    st = torch.empty(N, dtype=torch.uint8, device=td.device)
    _lib.check(lib.sv_lr_refine(_ptr(tl), _ptr(tr), code, _ptr(td), W, H, float(tol),
                                ctypes.byref(p), _ptr(out), _ptr(st), _ptr(ws), need,
                                _stream()), "lr_refine")
    _data_status(ws, "lr_refine")
    return _ret(out, left), _ret(st, left, as_int=True)


class LRRefiner:
    """Device-resident lr_refine for one image size: the workspace is
    allocated once and ``run`` only enqueues kernels on the current stream
    (no host synchronisation).  Parameters default to refine_disparity's
    (R=10, P1=12, P2=150, rx=4, ry=3, tol=2.0; stereonet.py:5865-5866)."""

    def __init__(self, W, H, R=10, P1=12.0, P2=150.0, rx=4, ry=3, tol=2.0, paths=8, uniq=0.0):
        self.lib = _lib.load()
        self.W, self.H, self.tol = W, H, float(tol)
        self.p = _params(R=R, P1=P1, P2=P2, rx=rx, ry=ry, paths=paths, uniq=uniq)
        self.need = self.lib.sv_lr_refine_workspace_size(W, H, ctypes.byref(self.p))
        if self.need == 0:
            raise ValueError("unsupported refinement parameters for %dx%d" % (W, H))
        self.ws = _workspace(self.need)

    def run(self, left: torch.Tensor, right: torch.Tensor, disp0: torch.Tensor,
            out: torch.Tensor, status: torch.Tensor, stream: int | None = None) -> None:
        code = _TORCH_CODE[left.dtype]
        _lib.check(self.lib.sv_lr_refine(_ptr(left), _ptr(right), code, _ptr(disp0), self.W,
                                         self.H, self.tol, ctypes.byref(self.p), _ptr(out),
                                         _ptr(status), _ptr(self.ws), self.need,
                                         _stream() if stream is None else stream),
                   "lr_refine")

    def run_timed(self, left, right, disp0, out, status, events, stream=None) -> None:
        """``run`` that also records ``events`` (STAGES + 1 torch.cuda.Event
        with timing enabled) around its stages: base + left_to_right, census,
        band costs, SGM, WTA, left-right check."""
        code = _TORCH_CODE[left.dtype]
        for e in events:
            if e.cuda_event == 0:          # torch creates events lazily
                e.record()
        arr = (ctypes.c_void_p * len(events))(*[e.cuda_event for e in events])
        _lib.check(self.lib.sv_lr_refine_timed(
            _ptr(left), _ptr(right), code, _ptr(disp0), self.W, self.H, self.tol,
            ctypes.byref(self.p), _ptr(out), _ptr(status), _ptr(self.ws), self.need,
            _stream() if stream is None else stream, arr, len(events)), "lr_refine")

    STAGES = ("base+left_to_right", "census", "band_costs", "sgm", "wta", "lr_check")

    def data_status(self) -> None:
        _data_status(self.ws, "lr_refine")
