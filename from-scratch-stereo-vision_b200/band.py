"""Learned adaptive band for lr_refine (no counterpart in the reference).

The reference refines the network disparity inside a fixed +-R band
(lr_refine, stereonet.py:5343-5391 with refine_disparity's R=10).  Where the
network is more than R px off -- thin foreground structures, boundaries --
the true disparity is outside the band and cannot be recovered.  The band
net (4 convolutions, 6098 parameters, BF16 tensor-core kernels) reads eight
per-pixel features (network disparity, a wide 9-row census search, costs at
the network disparity and inside its band, gray level, and how sure the
network was: the spread and peak probability of its soft-argmin
distribution, stereonet.py:858-885).  The band is built around a rule
centre -- the network disparity moved to the wide search's argmin wherever
that argmin's cost is below rule_tau (chosen on validation pairs) -- and
the net predicts a shift from that centre with a Laplace scale b.  Where
b <= b_thr the band moves to centre + shift and narrows to ceil(rad_k * b)
(at least rad_min); elsewhere it stays at the rule centre with the full
+-R width.  It is trained on the method's own
full-range SGM disparities (refine_fullres with disp0 = R, R = (dmax+2)//2+1
as in eval_real.py:143-146) with Adam (stereonet.py:1354-1387).

Entry points: ``features``, ``rule_centre``, ``BandNet`` (forward / grads /
train_step), ``targets``, ``apply``, ``lr_refine_band`` and
``LearnedBandRefiner``.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from .refine import _data_status, _device, _finite_disp, _image, _params, _ptr, _ret, _stream, \
    _to_dev, _workspace

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "band_weights.npz")

N_FEATURES = 8
N_OUTPUTS = 2
LAYERS = ((8, 16, 1), (16, 16, 2), (16, 16, 4), (16, 2, 1))    # (in, out, dilation)
# band application defaults (a trained checkpoint may carry its own)
APPLY = dict(b_thr=3.0, rad_k=3.0, rad_min=3, R=10, shift_max=160.0,
             rule_tau=0.1)           # rule_tau: the no-net ablation's threshold (band_train)


def param_count() -> int:
    return int(_lib.load().sv_band_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """He initialisation as the reference's Conv2d (stereonet.py:466-481):
    w ~ N(0, 2 / fan_in), b = 0; the last layer is scaled by 0.1 so the
    first predictions are a zero shift with b = e px."""
    rng = np.random.default_rng(seed)
    blocks = []
    for i, (ic, oc, _d) in enumerate(LAYERS):
        w = rng.normal(0.0, np.sqrt(2.0 / (ic * 9)), oc * ic * 9)
        if i == len(LAYERS) - 1:
            w *= 0.1
        blocks += [w, np.zeros(oc)]
    return np.concatenate(blocks)


def _f32_dev(x, n, name):
    return _to_dev(x, n, torch.float32, name=name)


def features(left, right, disp0, W, H, dmax=255, spread=None, pmax=None):
    """[8][H][W] FP32 device tensor (see the module docstring); spread and
    pmax are the network's confidence maps of the pass that gave disp0
    (network.confidence); without them planes 6 and 7 are 0."""
    lib = _lib.load()
    N = W * H
    _finite_disp(disp0)
    tl, code = _image(left, N, "left")
    tr, code_r = _image(right, N, "right")
    if code_r != code:
        tr = tr.to(tl.dtype)
    td = _to_dev(disp0, N, torch.float64, name="disp0")
    need = lib.sv_band_features_workspace_size(W, H)
    ws = _workspace(need)
    feat = torch.empty(N_FEATURES * N, dtype=torch.float32, device=td.device)
    _lib.check(lib.sv_band_features(_ptr(tl), _ptr(tr), code, _ptr(td), W, H, int(dmax),
                                    _ptr(feat), _ptr(ws), need, _stream()), "band_features")
    _data_status(ws, "band_features")
    sp = torch.zeros(N, dtype=torch.float64, device=td.device) if spread is None else \
        _to_dev(spread, N, torch.float64, name="spread")
    pm = torch.full((N,), 0.5, dtype=torch.float64, device=td.device) if pmax is None else \
        _to_dev(pmax, N, torch.float64, name="pmax")
    _lib.check(lib.sv_band_conf_features(_ptr(sp), _ptr(pm), W, H, _ptr(feat), _stream()),
               "band_conf_features")
    return feat


def rule_centre(feat, disp0, W, H, tau):
    """The rule centre (FP64 device tensor) from the features and disp0."""
    lib = _lib.load()
    N = W * H
    f = _f32_dev(feat, N_FEATURES * N, "feat")
    td = _to_dev(disp0, N, torch.float64, name="disp0")
    out = torch.empty(N, dtype=torch.float64, device=td.device)
    _lib.check(lib.sv_band_rule_centre(_ptr(f), _ptr(td), W, H, float(tau), _ptr(out),
                                       _stream()), "band_rule_centre")
    return out


class BandNet:
    """One band net on the current device (sv_band): FP32 master parameters,
    Adam moments and the packed BF16 tensor-core operands."""

    def __init__(self, params=None, seed: int = 0, meta=None):
        self.lib = _lib.load()
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float64).ravel()
        if p.size != param_count():
            raise ValueError("band net has %d parameters, got %d" % (param_count(), p.size))
        h = ctypes.c_void_p()
        flat = np.ascontiguousarray(p)
        _lib.check(self.lib.sv_band_create(flat.ctypes.data_as(ctypes.c_void_p), flat.size,
                                           ctypes.byref(h)), "band_create")
        self.handle = h
        self.n = flat.size
        self.meta = dict(APPLY if meta is None else meta)
        self._ws = {}
        self.loss = torch.zeros(1, dtype=torch.float64, device=_device())

    def __del__(self):
        try:
            if self.handle:
                self.lib.sv_band_destroy(self.handle)
        except Exception:
            pass

    @classmethod
    def load(cls, path: str | None = None) -> "BandNet":
        z = np.load(DEFAULT_WEIGHTS if path is None else path)
        meta = dict(APPLY)
        for k in APPLY:
            if k in z.files:
                meta[k] = type(APPLY[k])(z[k])
        return cls(z["params"], meta=meta)

    def params(self) -> np.ndarray:
        out = np.zeros(self.n)
        _lib.check(self.lib.sv_band_get_params(self.handle, out.ctypes.data_as(ctypes.c_void_p),
                                               self.n), "band_get_params")
        return out

    def save(self, path: str, **extra) -> None:
        np.savez(path, params=self.params(), **{k: np.asarray(v) for k, v in self.meta.items()},
                 **{k: np.asarray(v) for k, v in extra.items()})

    def _workspace(self, nb, W, H):
        key = (nb, W, H)
        if key not in self._ws:
            need = self.lib.sv_band_workspace_size(nb, W, H)
            self._ws[key] = (_workspace(need), need)
        return self._ws[key]

    def forward(self, feat, nb, W, H, out=None, stream=None):
        """feat [nb][6][H][W] (device) -> out [nb][2][H][W] FP32."""
        ws, need = self._workspace(nb, W, H)
        f = _f32_dev(feat, nb * N_FEATURES * W * H, "feat")
        if out is None:
            out = torch.empty(nb * N_OUTPUTS * W * H, dtype=torch.float32, device=f.device)
        _lib.check(self.lib.sv_band_forward(self.handle, _ptr(f), nb, W, H, _ptr(out), _ptr(ws),
                                            need, _stream() if stream is None else stream),
                   "band_forward")
        return out

    def grads(self, feat, target, mask, nb, W, H):
        """-> (FP32 gradients in parameter order, loss) on the device."""
        ws, need = self._workspace(nb, W, H)
        n = nb * W * H
        f = _f32_dev(feat, n * N_FEATURES, "feat")
        t = _f32_dev(target, n, "target")
        m = _to_dev(mask, n, torch.uint8, name="mask")
        g = torch.empty(self.n, dtype=torch.float32, device=f.device)
        _lib.check(self.lib.sv_band_grads(self.handle, _ptr(f), _ptr(t), _ptr(m), nb, W, H,
                                          _ptr(g), _ptr(self.loss), _ptr(ws), need, _stream()),
                   "band_grads")
        _data_status(ws, "band_grads")
        return g, self.loss

    def train_step(self, feat, target, mask, nb, W, H, lr=5e-4, stream=None):
        """One Adam step on a batch of device tensors (no host sync); the
        batch's loss (before the step) is left in a device scalar that
        ``last_loss`` reads."""
        ws, need = self._workspace(nb, W, H)
        _lib.check(self.lib.sv_band_train_step(self.handle, _ptr(feat), _ptr(target), _ptr(mask),
                                               nb, W, H, float(lr), _ptr(self._step_loss()),
                                               _ptr(ws), need,
                                               _stream() if stream is None else stream),
                   "band_train_step")

    def _step_loss(self):
        if not hasattr(self, "_sl"):
            self._sl = torch.zeros(1, dtype=torch.float64, device=_device())
        return self._sl

    @property
    def last_loss(self) -> float:
        return float(self._step_loss().item())


def targets(label, status, disp0, shift_max=160.0):
    """(target shift FP32, mask u8) device tensors from full-range labels."""
    lib = _lib.load()
    n = int(np.asarray(label).size if not isinstance(label, torch.Tensor) else label.numel())
    tl = _to_dev(label, n, torch.float64, name="label")
    ts = _to_dev(status, n, torch.uint8, name="status")
    td = _to_dev(disp0, n, torch.float64, name="disp0")
    t = torch.empty(n, dtype=torch.float32, device=tl.device)
    m = torch.empty(n, dtype=torch.uint8, device=tl.device)
    _lib.check(lib.sv_band_targets(_ptr(tl), _ptr(ts), _ptr(td), n, float(shift_max), _ptr(t),
                                   _ptr(m), _stream()), "band_targets")
    return t, m


def apply(out, disp0, W, H, b_thr=3.0, rad_k=3.0, rad_min=3, R=10, shift_max=160.0):
    """Band net output of one pair -> (centre FP64, half-width u8) device tensors."""
    lib = _lib.load()
    N = W * H
    o = _f32_dev(out, N_OUTPUTS * N, "out")
    td = _to_dev(disp0, N, torch.float64, name="disp0")
    centre = torch.empty(N, dtype=torch.float64, device=td.device)
    rad = torch.empty(N, dtype=torch.uint8, device=td.device)
    _lib.check(lib.sv_band_apply(_ptr(o), _ptr(td), W, H, float(b_thr), float(rad_k),
                                 int(rad_min), int(R), float(shift_max), _ptr(centre), _ptr(rad),
                                 _stream()), "band_apply")
    return centre, rad


def lr_refine_band(left, right, centre, rad, W, H, tol=2.0, **kw):
    """lr_refine around per-pixel centres with per-pixel left-view half-widths."""
    lib = _lib.load()
    N = W * H
    _finite_disp(centre, "centre")
    p = _params(**kw)
    tl, code = _image(left, N, "left")
    tr, code_r = _image(right, N, "right")
    if code_r != code:
        tr = tr.to(tl.dtype)
    tc = _to_dev(centre, N, torch.float64, name="centre")
    trad = _to_dev(rad, N, torch.uint8, name="rad")
    need = lib.sv_lr_refine_workspace_size(W, H, ctypes.byref(p))
    if need == 0:
        _lib.raise_last("lr_refine_band")
    ws = _workspace(need)
    out = torch.empty(N, dtype=torch.float64, device=tc.device)
    st = torch.empty(N, dtype=torch.uint8, device=tc.device)
    _lib.check(lib.sv_lr_refine_band(_ptr(tl), _ptr(tr), code, _ptr(tc), _ptr(trad), W, H,
                                     float(tol), ctypes.byref(p), _ptr(out), _ptr(st), _ptr(ws),
                                     need, _stream()), "lr_refine_band")
    _data_status(ws, "lr_refine_band")
    return _ret(out, left), _ret(st, left, as_int=True)


class LearnedBandRefiner:
    """Device-resident learned-band refinement of one W x H size: features,
    band net, band application and the masked lr_refine enqueued on a
    stream with buffers allocated once (refine_disparity's R=10, P1=12,
    P2=150, 9x7 census, tol=2)."""

    def __init__(self, W, H, band: BandNet, dmax=255, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                 tol=2.0):
        self.lib = _lib.load()
        self.W, self.H, self.band, self.dmax, self.tol = W, H, band, int(dmax), float(tol)
        self.p = _params(R=R, P1=P1, P2=P2, rx=rx, ry=ry)
        dev = _device()
        N = W * H
        self.feat = torch.empty(N_FEATURES * N, dtype=torch.float32, device=dev)
        self.out = torch.empty(N_OUTPUTS * N, dtype=torch.float32, device=dev)
        self.base = torch.empty(N, dtype=torch.float64, device=dev)     # the rule centre
        self.centre = torch.empty(N, dtype=torch.float64, device=dev)
        self.rad = torch.empty(N, dtype=torch.uint8, device=dev)
        self.fneed = self.lib.sv_band_features_workspace_size(W, H)
        self.fws = _workspace(self.fneed)
        self.rneed = self.lib.sv_lr_refine_workspace_size(W, H, ctypes.byref(self.p))
        self.rws = _workspace(self.rneed)
        self.bws, self.bneed = band._workspace(1, W, H)

    def run(self, left, right, code, disp0, out, status, stream, spread, pmax):
        """spread / pmax: the network's confidence maps of the pass that gave
        disp0 (PairPipeline.confidence)."""
        W, H, m = self.W, self.H, self.band.meta
        _lib.check(self.lib.sv_band_features(_ptr(left), _ptr(right), code, _ptr(disp0), W, H,
                                             self.dmax, _ptr(self.feat), _ptr(self.fws),
                                             self.fneed, stream), "band_features")
        _lib.check(self.lib.sv_band_conf_features(_ptr(spread), _ptr(pmax), W, H,
                                                  _ptr(self.feat), stream), "band_conf_features")
        _lib.check(self.lib.sv_band_rule_centre(_ptr(self.feat), _ptr(disp0), W, H,
                                                float(m["rule_tau"]), _ptr(self.base), stream),
                   "band_rule_centre")
        _lib.check(self.lib.sv_band_forward(self.band.handle, _ptr(self.feat), 1, W, H,
                                            _ptr(self.out), _ptr(self.bws), self.bneed, stream),
                   "band_forward")
        _lib.check(self.lib.sv_band_apply(_ptr(self.out), _ptr(self.base), W, H, float(m["b_thr"]),
                                          float(m["rad_k"]), int(m["rad_min"]), int(m["R"]),
                                          float(m["shift_max"]), _ptr(self.centre),
                                          _ptr(self.rad), stream), "band_apply")
        _lib.check(self.lib.sv_lr_refine_band(_ptr(left), _ptr(right), code, _ptr(self.centre),
                                              _ptr(self.rad), W, H, self.tol,
                                              ctypes.byref(self.p), _ptr(out), _ptr(status),
                                              _ptr(self.rws), self.rneed, stream),
                   "lr_refine_band")
