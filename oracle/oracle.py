"""TEST INFRASTRUCTURE ONLY -- ctypes wrapper over the FP64 C oracle.

``sv_oracle.c`` restates the reference's disparity hot path (stereonet.py) in
plain C with the reference's own operation order; the golden fixtures in
tests/golden/ (made by running the reference itself) pin it bit-for-bit.
Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.  Function names and argument meanings follow the
reference (flat row-major FP64 arrays, ``W, H`` order except
``stereonet_forward`` which keeps the reference's ``H, W``).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libsv_oracle.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_u64 = ctypes.POINTER(ctypes.c_uint64)
_i64 = ctypes.POINTER(ctypes.c_int64)
_i32 = ctypes.POINTER(ctypes.c_int32)
_int = ctypes.c_int
_dbl = ctypes.c_double


def build() -> str:
    subprocess.check_call(["make", "-s", "-C", _HERE])
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO) or os.path.getmtime(_SO) < max(
                os.path.getmtime(os.path.join(_HERE, f))
                for f in ("sv_oracle.c", "sv_band_oracle.c", "sv_train_oracle.c")):
            build()
        L = ctypes.CDLL(_SO)
        L.orc_fexp.restype = _dbl
        L.orc_fexp.argtypes = [_dbl]
        L.orc_peak.restype = _dbl
        L.orc_peak.argtypes = [_d, ctypes.c_long, _dbl]
        L.orc_param_count.restype = ctypes.c_long
        L.orc_band_param_count.restype = ctypes.c_long
        L.orc_band_loss.restype = _dbl
        L.orc_fsqrt.restype = _dbl
        L.orc_fsqrt.argtypes = [_dbl]
        L.orc_flog.restype = _dbl
        L.orc_flog.argtypes = [_dbl]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def _check(rc, what):
    if rc != 0:
        raise ValueError("oracle %s failed with code %d" % (what, rc))


# ---------------------------------------------------------------- refinement
def census(img, W, H, rx=2, ry=2) -> np.ndarray:
    img = _f64(img)
    out = np.zeros(W * H, dtype=np.uint64)
    _check(lib().orc_census(_p(img), W, H, rx, ry, _p(out, _u64)), "census")
    return out


def band_costs(cl, cr, gl, gr, base, W, H, R, ad_weight, ad_trunc, invalid,
               prior=None, prior_w=0.0, prior_t=4.0) -> np.ndarray:
    K = 2 * R + 1
    cl = np.ascontiguousarray(cl, dtype=np.uint64)
    cr = np.ascontiguousarray(cr, dtype=np.uint64)
    gl, gr = _f64(gl), _f64(gr)
    base = np.ascontiguousarray(base, dtype=np.int64)
    pr = _f64(prior) if prior is not None else np.zeros(W * H)
    C = np.zeros(W * H * K)
    lib().orc_band_costs(_p(cl, _u64), _p(cr, _u64), _p(gl), _p(gr), _p(base, _i64),
                         W, H, R, _dbl(ad_weight), _dbl(ad_trunc), _dbl(invalid),
                         _p(pr), _dbl(prior_w), _dbl(prior_t), _p(C))
    return C


def aggregate_path(C, base, W, H, K, P1, P2, dx, dy, S: np.ndarray) -> None:
    """Adds one path into ``S`` (a float64 array, modified in place)."""
    C = _f64(C)
    base = np.ascontiguousarray(base, dtype=np.int64)
    assert S.dtype == np.float64 and S.flags.c_contiguous
    lib().orc_aggregate_path(_p(C), _p(base, _i64), W, H, K, _dbl(P1), _dbl(P2),
                             dx, dy, _p(S))


def refine_fullres(left, right, disp0, W, H, R=3, P1=1.0, P2=12.0,
                   ad_weight=0.0, ad_trunc=20.0, paths=8, uniq=0.0,
                   rx=2, ry=2, prior_w=0.0, prior_t=4.0, return_conf=False):
    left, right, disp0 = _f64(left), _f64(right), _f64(disp0)
    out = np.zeros(W * H)
    conf = np.zeros(W * H)
    _check(lib().orc_refine_fullres(_p(left), _p(right), _p(disp0), W, H, R,
                                    _dbl(P1), _dbl(P2), _dbl(ad_weight), _dbl(ad_trunc),
                                    paths, _dbl(uniq), rx, ry, _dbl(prior_w),
                                    _dbl(prior_t), _p(out), _p(conf)), "refine_fullres")
    return (out, conf) if return_conf else out


def left_to_right(dl, W, H) -> np.ndarray:
    dl = _f64(dl)
    dr = np.zeros(W * H)
    _check(lib().orc_left_to_right(_p(dl), W, H, _p(dr)), "left_to_right")
    return dr


def lr_refine(left, right, disp0, W, H, tol=1.0, R=3, P1=1.0, P2=12.0,
              ad_weight=0.0, ad_trunc=20.0, paths=8, uniq=0.0, rx=2, ry=2,
              prior_w=0.0, prior_t=4.0):
    left, right, disp0 = _f64(left), _f64(right), _f64(disp0)
    out = np.zeros(W * H)
    st = np.zeros(W * H, dtype=np.int32)
    _check(lib().orc_lr_refine(_p(left), _p(right), _p(disp0), W, H, _dbl(tol), R,
                               _dbl(P1), _dbl(P2), _dbl(ad_weight), _dbl(ad_trunc),
                               paths, _dbl(uniq), rx, ry, _dbl(prior_w), _dbl(prior_t),
                               _p(out), _p(st, _i32)), "lr_refine")
    return out, st


def refine_pipeline(left, right, disp0, W, H, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                    tol=2.0):
    """``lr_refine`` with ``refine_disparity``'s defaults (stereonet.py:5865-5872)."""
    return lr_refine(left, right, disp0, W, H, tol=tol, R=R, P1=P1, P2=P2, rx=rx, ry=ry)


# ------------------------------------------------------------------- network
def fexp(x: float) -> float:
    return float(lib().orc_fexp(_dbl(x)))


def resize_gray(img, W, H, W2, H2) -> np.ndarray:
    img = _f64(img)
    out = np.zeros(W2 * H2)
    lib().orc_resize(_p(img), W, H, W2, H2, _p(out))
    return out


def avgpool2(img, C, H, W):
    img = _f64(img)
    out = np.zeros(C * (H // 2) * (W // 2))
    lib().orc_avgpool2(_p(img), C, H, W, _p(out))
    return out, H // 2, W // 2


def peak(disp, q=0.95) -> float:
    d = _f64(disp)
    return float(lib().orc_peak(_p(d), len(d), _dbl(q)))


def _net_args(net):
    arch = np.array(net.arch.vector(), dtype=np.int32)
    params = net.flat
    return arch, params


def stereonet_forward(net, left, right, H, W, guide_half, guide_full):
    arch, params = _net_args(net)
    left, right = _f64(left), _f64(right)
    gh, gf = _f64(guide_half), _f64(guide_full)
    h = (((H - 1) // 2 + 1) - 1) // 2 + 1
    w = (((W - 1) // 2 + 1) - 1) // 2 + 1
    d0 = np.zeros(h * w)
    d1 = np.zeros((H // 2) * (W // 2))
    d2 = np.zeros(H * W)
    oh, ow = _int(), _int()
    _check(lib().orc_stereonet_forward(_p(arch, _i32), _p(params), _p(left), _p(right),
                                       H, W, _p(gh), _p(gf), _p(d0), _p(d1), _p(d2),
                                       ctypes.byref(oh), ctypes.byref(ow)), "forward")
    return d0, d1, d2


def predict(net, left, right, W, H) -> np.ndarray:
    arch, params = _net_args(net)
    left, right = _f64(left), _f64(right)
    out = np.zeros(W * H)
    _check(lib().orc_predict(_p(arch, _i32), _p(params), _p(left), _p(right), W, H,
                             _p(out)), "predict")
    return out


def predict_at_scale(net, left, right, W, H, work_width=96):
    arch, params = _net_args(net)
    left, right = _f64(left), _f64(right)
    df = np.zeros(W * H)
    dw = np.zeros(W * H)
    Ww, Hw = _int(), _int()
    _check(lib().orc_predict_at_scale(_p(arch, _i32), _p(params), _p(left), _p(right),
                                      W, H, work_width, _p(df), _p(dw), ctypes.byref(Ww),
                                      ctypes.byref(Hw)), "predict_at_scale")
    return df, dw[:Ww.value * Hw.value].copy(), Ww.value, Hw.value


def predict_auto(net, left, right, W, H, target_peak=None, probe_width=64,
                 max_width=320, passes=3, return_trace=False):
    arch, params = _net_args(net)
    left, right = _f64(left), _f64(right)
    tp = float(net.target_peak if target_peak is None else target_peak)
    df = np.zeros(W * H)
    dw = np.zeros(W * H)
    Ww, Hw = _int(), _int()
    trace = np.zeros(passes + 2, dtype=np.int32)
    _check(lib().orc_predict_auto(_p(arch, _i32), _p(params), _p(left), _p(right), W, H,
                                  _dbl(tp), probe_width, max_width, passes, _p(df), _p(dw),
                                  ctypes.byref(Ww), ctypes.byref(Hw), _p(trace, _i32)),
           "predict_auto")
    res = (df, dw[:Ww.value * Hw.value].copy(), Ww.value, Hw.value)
    if return_trace:
        return res, [int(t) for t in trace if t > 0]
    return res


# ------------------------------------------------------------ learned band
# FP64 definition of the band predictor (sv_band_oracle.c): features, the
# 4-layer net's forward / loss / gradients, Adam, band application and the
# masked lr_refine.
_u8 = ctypes.POINTER(ctypes.c_uint8)


def band_param_count() -> int:
    return int(lib().orc_band_param_count())


def band_features(left, right, disp0, W, H, dmax, spread=None, pmax=None) -> np.ndarray:
    """[8][H][W] band-net inputs: six features (census 9x7 of both views,
    disparity, gray) and the network's spread / 16 and peak probability - 0.5
    (given; zero spread and 0.5 probability when absent)."""
    gl, gr = _f64(left), _f64(right)
    cl, cr = census(gl, W, H, 4, 3), census(gr, W, H, 4, 3)
    d0 = _f64(disp0)
    N = W * H
    out = np.zeros(8 * N)
    _check(lib().orc_band_features(_p(cl, _u64), _p(cr, _u64), _p(d0), _p(gl), W, H,
                                   int(dmax), _p(out)), "band_features")
    if spread is not None:
        out[6 * N:7 * N] = (_f64(spread) / 16.0).astype(np.float32)
    if pmax is not None:
        out[7 * N:] = (_f64(pmax) - 0.5).astype(np.float32)
    return out


def band_rule_centre(feat, disp0, W, H, tau) -> np.ndarray:
    """disp0 + 64 * f1 where f2 < tau, else disp0 (the learned band's base)."""
    N = W * H
    f = np.asarray(feat, dtype=np.float32).astype(np.float64).reshape(-1, N)
    d0 = _f64(disp0)
    return np.where(f[2] < tau, d0 + 64.0 * f[1], d0)


def band_forward(params, feat, nb, W, H) -> np.ndarray:
    params, feat = _f64(params), _f64(feat)
    out = np.zeros(nb * 2 * W * H)
    _check(lib().orc_band_forward(_p(params), _p(feat), nb, W, H, _p(out)), "band_forward")
    return out


def band_grads(params, feat, target, mask, nb, W, H):
    """-> (gradients in parameter order, loss)."""
    params, feat, target = _f64(params), _f64(feat), _f64(target)
    mask = np.ascontiguousarray(mask, dtype=np.uint8)
    g = np.zeros(band_param_count())
    loss = _dbl()
    _check(lib().orc_band_grads(_p(params), _p(feat), _p(target), _p(mask, _u8), nb, W, H,
                                _p(g), ctypes.byref(loss)), "band_grads")
    return g, loss.value


def band_loss(out, target, mask, nb, W, H) -> float:
    out, target = _f64(out), _f64(target)
    mask = np.ascontiguousarray(mask, dtype=np.uint8)
    return float(lib().orc_band_loss(_p(out), _p(target), _p(mask, _u8), nb, W, H, None))


class Adam:
    """Adam.step of stereonet.py:1354-1387 over one flat parameter vector."""

    def __init__(self, params, lr=5e-4, b1=0.9, b2=0.999, eps=1e-8, clip=5.0):
        self.p = np.array(params, dtype=np.float64)
        self.m = np.zeros_like(self.p)
        self.v = np.zeros_like(self.p)
        self.lr, self.b1, self.b2, self.eps, self.clip = lr, b1, b2, eps, clip
        self.b1t, self.b2t = _dbl(1.0), _dbl(1.0)

    def step(self, g):
        g = _f64(g)
        lib().orc_adam_step(_p(self.p), _p(g), _p(self.m), _p(self.v),
                            ctypes.c_long(self.p.size), _dbl(self.lr), _dbl(self.b1),
                            _dbl(self.b2), _dbl(self.eps), _dbl(self.clip),
                            ctypes.byref(self.b1t), ctypes.byref(self.b2t))
        return self.p


def band_apply(out, disp0, W, H, b_thr=3.0, rad_k=3.0, rad_min=3, R=10, shift_max=160.0):
    out, d0 = _f64(out), _f64(disp0)
    centre = np.zeros(W * H)
    rad = np.zeros(W * H, dtype=np.uint8)
    lib().orc_band_apply(_p(out), _p(d0), W, H, _dbl(b_thr), _dbl(rad_k), int(rad_min), int(R),
                         _dbl(shift_max), _p(centre), _p(rad, _u8))
    return centre, rad


def band_targets(label, status, disp0, shift_max=160.0):
    label, d0 = _f64(label), _f64(disp0)
    status = np.ascontiguousarray(status, dtype=np.int32)
    t = np.zeros(label.size)
    m = np.zeros(label.size, dtype=np.uint8)
    lib().orc_band_targets(_p(label), _p(status, _i32), _p(d0), ctypes.c_long(label.size),
                           _dbl(shift_max), _p(t), _p(m, _u8))
    return t, m


def lr_refine_band(left, right, centre, rad, W, H, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4,
                   ry=3):
    gl, gr, c = _f64(left), _f64(right), _f64(centre)
    rad = None if rad is None else np.ascontiguousarray(rad, dtype=np.uint8)
    out = np.zeros(W * H)
    st = np.zeros(W * H, dtype=np.int32)
    _check(lib().orc_lr_refine_band(_p(gl), _p(gr), _p(c), None if rad is None else _p(rad, _u8),
                                    W, H, _dbl(tol), R, _dbl(P1), _dbl(P2), rx, ry, _p(out),
                                    _p(st, _i32)), "lr_refine_band")
    return out, st


# --------------------------------------------- rest of refine_disparity
def _m2(compactness, step):
    # the reference computes (compactness / step) ** 2 with CPython's float
    # power, which calls the C library's pow()
    return (float(compactness) / step) ** 2


def slic(rgb, W, H, step=12, compactness=10.0, iters=5):
    rgb = _f64(rgb)
    lab = np.zeros(W * H, dtype=np.int32)
    nseg = _int()
    _check(lib().orc_slic(_p(rgb), W, H, int(step), _dbl(_m2(compactness, step)), int(iters),
                          _p(lab, _i32), ctypes.byref(nseg)), "slic")
    return lab, nseg.value


def plane_snap(disp, rgb, W, H, valid=None, step=12, thr=1.0, min_inl=0.6, trials=40,
               seed=12345):
    disp, rgb = _f64(disp), _f64(rgb)
    v = None if valid is None else np.ascontiguousarray(np.asarray(valid, dtype=bool), np.uint8)
    out = np.zeros(W * H)
    _check(lib().orc_plane_snap(_p(disp), _p(rgb), W, H,
                                None if v is None else _p(v, ctypes.POINTER(ctypes.c_uint8)),
                                int(step), _dbl(_m2(10.0, step)), _dbl(thr), _dbl(min_inl),
                                int(trials), ctypes.c_uint32(seed), _p(out)), "plane_snap")
    return out


def median_filter(disp, W, H, radius=1, passes=1):
    disp = _f64(disp)
    out = np.zeros(W * H)
    _check(lib().orc_median_filter(_p(disp), W, H, int(radius), int(passes), _p(out)),
           "median_filter")
    return out


def refine_disparity(left, right, rgb, disp0, W, H, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                     tol=2.0, planes=True, plane_step=12, plane_thr=1.0, plane_min_inl=0.4):
    left, right, d0 = _f64(left), _f64(right), _f64(disp0)
    rgbv = None if rgb is None else _f64(rgb)
    out = np.zeros(W * H)
    st = np.zeros(W * H, dtype=np.int32)
    _check(lib().orc_refine_disparity(_p(left), _p(right), None if rgbv is None else _p(rgbv),
                                      _p(d0), W, H, R, _dbl(P1), _dbl(P2), rx, ry, _dbl(tol),
                                      int(bool(planes)), int(plane_step),
                                      _dbl(_m2(10.0, plane_step)), _dbl(plane_thr),
                                      _dbl(plane_min_inl), _p(out), _p(st, _i32)),
           "refine_disparity")
    return out, st


# ------------------------------------------- network-level LR consistency
def lr_consistency(disp_l, disp_r, W, H, tol=1.5):
    dl, dr = _f64(disp_l), _f64(disp_r)
    v = np.zeros(W * H, dtype=np.uint8)
    lib().orc_lr_consistency(_p(dl), _p(dr), W, H, _dbl(tol), _p(v, ctypes.POINTER(ctypes.c_uint8)))
    return v.astype(bool)


def fill_invalid(disp, valid, W, H):
    d = _f64(disp)
    v = np.ascontiguousarray(np.asarray(valid, dtype=bool), dtype=np.uint8)
    out = np.zeros(W * H)
    lib().orc_fill_invalid(_p(d), _p(v, ctypes.POINTER(ctypes.c_uint8)), W, H, _p(out))
    return out


def predict_consistent(net, left, right, W, H, work_width=None, tol=1.5, target_peak=None,
                       probe_width=64, max_width=320, passes=3):
    arch, params = _net_args(net)
    left, right = _f64(left), _f64(right)
    tp = float(net.target_peak if target_peak is None else target_peak)
    out = np.zeros(W * H)
    kept = ctypes.c_long()
    _check(lib().orc_predict_consistent(_p(arch, _i32), _p(params), _p(left), _p(right), W, H,
                                        0 if work_width is None else int(work_width), _dbl(tp),
                                        probe_width, max_width, passes, _dbl(tol), _p(out),
                                        ctypes.byref(kept)), "predict_consistent")
    return out, kept.value / float(W * H)


# ------------------------------------------------------------------ training
def train_grads(net, left, right, disp, valid, W, H, params=None):
    """train_grads (stereonet.py:1619-1653) on one sample: returns (loss,
    gradient in all_params() order, full-resolution prediction).  `params`
    (flat, all_params() order) overrides the network's own."""
    arch, p0 = _net_args(net)
    params = _f64(p0 if params is None else params)
    n = int(lib().orc_param_count(_p(arch, _i32)))
    g = np.zeros(n)
    d2 = np.zeros(W * H)
    loss = ctypes.c_double()
    l_, r_, d_ = _f64(left), _f64(right), _f64(disp)
    v_ = np.ascontiguousarray(np.asarray(valid).ravel().astype(np.uint8))
    _check(lib().orc_train_grads(_p(arch, _i32), _p(params), _p(l_), _p(r_), _p(d_),
                                 v_.ctypes.data_as(ctypes.c_void_p), W, H, _p(g),
                                 ctypes.byref(loss), _p(d2)), "train_grads")
    return loss.value, g, d2


class AdamState:
    """Adam (stereonet.py:1354-1387) over a flat parameter vector, with the
    reference's own fsqrt (bit-identical steps)."""

    def __init__(self, params, lr=1.0e-3):
        self.p = _f64(params).copy()
        self.m = np.zeros_like(self.p)
        self.v = np.zeros_like(self.p)
        self.lr = lr
        self.b1t = ctypes.c_double(1.0)
        self.b2t = ctypes.c_double(1.0)

    def step(self, grads, clip=5.0):
        g = _f64(grads)
        lib().orc_train_adam_step(_p(self.p), _p(g), _p(self.m), _p(self.v),
                                  ctypes.c_long(self.p.size), ctypes.c_double(self.lr),
                                  ctypes.byref(self.b1t), ctypes.byref(self.b2t),
                                  ctypes.c_double(clip))
        return self.p
