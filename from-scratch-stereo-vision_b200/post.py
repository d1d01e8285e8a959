"""The rest of refine_disparity on the GPU: median_filter, slic, plane_snap
and refine_disparity itself (stereonet.py:2231-2259, 5394-5563, 5865-5883),
bit-identical to the reference, with its signatures.

``rgb`` is the interleaved RGB image in [0, 1] (as the reference's
read_image returns it); disparities are FP64.  Lists come back as lists,
numpy arrays as arrays, CUDA tensors as CUDA tensors.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .refine import _data_status, _finite_disp, _image, _params, _ptr, _ret, _stream, _to_dev, \
    _workspace


def _f64(x, n, name):
    return _to_dev(x, n, torch.float64, name=name)


def median_filter(disp, W, H, radius=1, passes=1):
    """stereonet.py:2231-2259 (radius <= 3)."""
    lib = _lib.load()
    d = _f64(disp, W * H, "disp")
    out = torch.empty_like(d)
    need = lib.sv_median_workspace_size(W, H)
    ws = _workspace(need)
    _lib.check(lib.sv_median_filter(_ptr(d), W, H, int(radius), int(passes), _ptr(out), _ptr(ws),
                                    need, _stream()), "median_filter")
    return _ret(out, disp)


def slic(rgb, W, H, step=12, compactness=10.0, iters=5):
    """stereonet.py:5394-5455 -> (labels, number of clusters)."""
    lib = _lib.load()
    r = _f64(rgb, 3 * W * H, "rgb")
    lab = torch.empty(W * H, dtype=torch.int32, device=r.device)
    need = lib.sv_postproc_workspace_size(W, H, int(step))
    if need == 0:
        raise ValueError("slic: bad shape or step")
    ws = _workspace(need)
    _lib.check(lib.sv_slic(_ptr(r), W, H, int(step), float(compactness), int(iters), _ptr(lab),
                           _ptr(ws), need, _stream()), "slic")
    return _ret(lab, rgb, as_int=True), int(lib.sv_slic_count(W, H, int(step)))


def plane_snap(disp, rgb, W, H, valid=None, step=12, thr=1.0, min_inl=0.6, trials=40,
               seed=12345):
    """stereonet.py:5505-5563."""
    lib = _lib.load()
    N = W * H
    d = _f64(disp, N, "disp")
    r = _f64(rgb, 3 * N, "rgb")
    v = None if valid is None else _to_dev([bool(x) for x in valid] if isinstance(valid, list)
                                           else valid, N, torch.uint8, name="valid")
    out = torch.empty_like(d)
    need = lib.sv_postproc_workspace_size(W, H, int(step))
    if need == 0:
        raise ValueError("plane_snap: bad shape or step")
    ws = _workspace(need)
    _lib.check(lib.sv_plane_snap(_ptr(d), _ptr(r), W, H, _ptr(v), int(step), float(thr),
                                 float(min_inl), int(trials), ctypes.c_uint32(int(seed) & 0xFFFFFFFF),
                                 _ptr(out), _ptr(ws), need, _stream()), "plane_snap")
    return _ret(out, disp)


def refine_disparity(left, right, rgb, disp0, W, H, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                     tol=2.0, planes=True, plane_step=12, plane_thr=1.0, plane_min_inl=0.4,
                     verbose=False):
    """stereonet.py:5865-5883 -> (disparity, status)."""
    lib = _lib.load()
    N = W * H
    _finite_disp(disp0)
    p = _params(R=R, P1=P1, P2=P2, rx=rx, ry=ry)
    tl, code = _image(left, N, "left")
    tr, code_r = _image(right, N, "right")
    if code_r != code:
        tr = tr.to(tl.dtype)
    td = _f64(disp0, N, "disp0")
    r = None if rgb is None else _f64(rgb, 3 * N, "rgb")
    need = lib.sv_refine_disparity_workspace_size(W, H, ctypes.byref(p), int(plane_step))
    if need == 0:
        _lib.raise_last("refine_disparity")
    ws = _workspace(need)
    out = torch.empty(N, dtype=torch.float64, device=td.device)
    st = torch.empty(N, dtype=torch.uint8, device=td.device)
    _lib.check(lib.sv_refine_disparity(_ptr(tl), _ptr(tr), code, _ptr(r), _ptr(td), W, H,
                                       float(tol), ctypes.byref(p), int(bool(planes)),
                                       int(plane_step), float(plane_thr), float(plane_min_inl),
                                       _ptr(out), _ptr(st), _ptr(ws), need, _stream()),
               "refine_disparity")
    _data_status(ws, "refine_disparity")
    if verbose:
        s = st.cpu().numpy()
        print("  full-res refinement: %.1f%% occluded, %.1f%% mismatched"
              % (100.0 * (s == 1).mean(), 100.0 * (s == 2).mean()))
    return _ret(out, left), _ret(st, left, as_int=True)


def lr_consistency(disp_l, disp_r, W, H, tol=1.5):
    """stereonet.py:4986-5009 -> list of bools (or a bool array / tensor)."""
    lib = _lib.load()
    N = W * H
    dl, dr = _f64(disp_l, N, "disp_l"), _f64(disp_r, N, "disp_r")
    v = torch.empty(N, dtype=torch.uint8, device=dl.device)
    kept = torch.zeros(1, dtype=torch.int64, device=dl.device)
    _lib.check(lib.sv_lr_consistency(_ptr(dl), _ptr(dr), W, H, float(tol), _ptr(v), _ptr(kept),
                                     _stream()), "lr_consistency")
    vb = v.bool()
    if isinstance(disp_l, list):
        return [bool(x) for x in vb.cpu().numpy()]
    return _ret(vb, disp_l)


def fill_invalid(disp, valid, W, H):
    """stereonet.py:5012-5045."""
    lib = _lib.load()
    N = W * H
    d = _f64(disp, N, "disp")
    v = _to_dev([bool(x) for x in valid] if isinstance(valid, list) else valid, N, torch.uint8,
                name="valid")
    out = torch.empty_like(d)
    need = lib.sv_fill_invalid_workspace_size(W, H)
    ws = _workspace(need)
    _lib.check(lib.sv_fill_invalid(_ptr(d), _ptr(v), W, H, _ptr(out), _ptr(ws), need, _stream()),
               "fill_invalid")
    return _ret(out, disp)
