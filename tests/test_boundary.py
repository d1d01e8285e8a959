"""The C-ABI library: it loads, exports every declared symbol, and rejects
bad arguments before touching a GPU (host-only checks, no compute)."""

import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(REPO, "include", "sv_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sv_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree(svb):
    assert header_functions() == svb._lib.exported_symbols()


def test_library_exports_every_declared_symbol(svb):
    lib = ctypes.CDLL(svb._lib.LIB_PATH)
    for name in header_functions():
        assert hasattr(lib, name), name


def test_status_strings(svb):
    lib = svb._lib.load()
    for code in range(9):
        assert lib.sv_status_string(code) != b"unknown status"
    assert lib.sv_version() >= 1


def test_default_params_match_reference(svb):
    p = svb._lib.default_params()
    # refine_fullres defaults, stereonet.py:5244-5246
    assert (p.R, p.P1, p.P2, p.rx, p.ry, p.paths, p.uniq) == (3, 1.0, 12.0, 2, 2, 8, 0.0)
    assert (p.ad_weight, p.ad_trunc, p.prior_w, p.prior_t) == (0.0, 20.0, 0.0, 4.0)


def _params(svb, **kw):
    p = svb._lib.default_params()
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("kw,W,H", [
    (dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3), 450, 375),
    (dict(), 160, 120),
])
def test_workspace_sizes(svb, kw, W, H):
    lib = svb._lib.load()
    p = _params(svb, **kw)
    one = lib.sv_refine_workspace_size(W, H, ctypes.byref(p))
    two = lib.sv_lr_refine_workspace_size(W, H, ctypes.byref(p))
    K = 2 * p.R + 1
    assert one >= W * H * K * (1 + 8)         # costs + 8 uint8 path arrays
    assert two >= 2 * one - 4096
    assert one % 256 == 0 and two % 256 == 0


@pytest.mark.parametrize("kw,W", [
    (dict(R=127), 64), (dict(rx=5, ry=5), 64), (dict(P1=1.5), 64), (dict(P2=5000.0), 64),
    (dict(ad_weight=0.5), 64), (dict(prior_w=1.0), 64), (dict(uniq=float("nan")), 64),
    (dict(), 0), (dict(), 20000),
])
def test_bad_params_rejected_on_host(svb, kw, W):
    lib = svb._lib.load()
    p = _params(svb, **kw)
    assert lib.sv_lr_refine_workspace_size(W, 8, ctypes.byref(p)) == 0
    assert lib.sv_last_error()


def test_null_and_workspace_checks(svb):
    lib = svb._lib.load()
    p = _params(svb)
    assert lib.sv_census(None, 0, 8, 8, 2, 2, None, None) == svb._lib.SV_ERR_NULL
    assert lib.sv_census(ctypes.c_void_p(256), 0, 8, 8, 5, 5, ctypes.c_void_p(256),
                         None) == svb._lib.SV_ERR_SHAPE
    rc = lib.sv_lr_refine(ctypes.c_void_p(256), ctypes.c_void_p(256), 0, ctypes.c_void_p(256),
                          8, 8, 1.0, ctypes.byref(p), ctypes.c_void_p(256),
                          ctypes.c_void_p(256), ctypes.c_void_p(0), 0, None)
    assert rc == svb._lib.SV_ERR_WORKSPACE
    rc = lib.sv_lr_refine(ctypes.c_void_p(256), ctypes.c_void_p(256), 0, ctypes.c_void_p(256),
                          8, 8, 1.0, ctypes.byref(p), ctypes.c_void_p(256),
                          ctypes.c_void_p(256), ctypes.c_void_p(256 + 8), 1 << 30, None)
    assert rc == svb._lib.SV_ERR_WORKSPACE     # misaligned
    assert lib.sv_aggregate_path(ctypes.c_void_p(256), ctypes.c_void_p(256), 8, 8, 21, 1, 2, 2,
                                 0, ctypes.c_void_p(256), None) == svb._lib.SV_ERR_PARAM
    # predict_auto + lr_refine in one call: argument errors surface before any device work
    v = ctypes.c_void_p(256)
    Ww, Hw = ctypes.c_int(), ctypes.c_int()
    rc = lib.sv_predict_refine(None, v, v, 0, 64, 48, 2.0, 64, 320, 3, 0, v, v,
                               ctypes.byref(Ww), ctypes.byref(Hw), None, v, 1 << 20, 2.0,
                               ctypes.byref(p), v, v, v, 1 << 20, None)
    assert rc == svb._lib.SV_ERR_NULL


def test_batch_schedule_defaults_and_validation(svb):
    """sv_batch_config_default and the argument check of
    sv_batch_lr_refine_ex (rejected before any device work)."""
    import ctypes
    c = svb.batch.default_config()
    assert c.as_dict() == {"px_per_block": 2048, "sgm_threads": 128, "sgm_ctas_per_sm": 8,
                           "sgm_fetch": 32}
    lib = svb._lib.load()
    d = (svb.batch.PairDesc * 1)()
    d[0] = svb.batch.PairDesc(1, 1, 1, 1, 1, 8, 8)
    p = svb._lib.default_params()
    for bad in ((3000, 128, 8, 32), (2048, 96, 8, 32), (2048, 128, 0, 32), (2048, 128, 8, 48)):
        cfg = svb.batch.BatchConfig(*bad)
        rc = lib.sv_batch_lr_refine_ex(d, 1, 0, 2.0, ctypes.byref(p), ctypes.byref(cfg), None, 0,
                                       None)
        assert rc == svb._lib.SV_ERR_PARAM, bad
