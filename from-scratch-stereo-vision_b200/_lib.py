"""ctypes binding of libsv_b200.so (declared in include/sv_b200.h).

There is no fallback: if the library is missing or cannot be loaded the
import of any calling module raises, and every entry point turns a nonzero
status into an exception (ValueError for argument and data errors, as the
reference raises; RuntimeError for CUDA failures).
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsv_b200.so")

SV_OK, SV_ERR_SHAPE, SV_ERR_PARAM, SV_ERR_DISP, SV_ERR_WORKSPACE, SV_ERR_CUDA, \
    SV_ERR_NULL, SV_ERR_NET, SV_ERR_TIMEOUT = range(9)
SV_U8, SV_F32, SV_F64 = 0, 1, 2
SV_FP32, SV_BF16 = 0, 1


class RefineParams(ctypes.Structure):
    """sv_refine_params (refine_fullres keyword arguments)."""
    _fields_ = [("R", ctypes.c_int), ("P1", ctypes.c_double), ("P2", ctypes.c_double),
                ("rx", ctypes.c_int), ("ry", ctypes.c_int), ("paths", ctypes.c_int),
                ("uniq", ctypes.c_double), ("ad_weight", ctypes.c_double),
                ("ad_trunc", ctypes.c_double), ("prior_w", ctypes.c_double),
                ("prior_t", ctypes.c_double)]


SV_IMAGE_PNG, SV_IMAGE_PNM = 1, 2


class RawImage(ctypes.Structure):
    """sv_raw_image (a decoded file's raw samples)."""
    _fields_ = [("kind", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("depth", ctypes.c_int), ("colortype", ctypes.c_int), ("channels", ctypes.c_int),
                ("stride", ctypes.c_int), ("interlace", ctypes.c_int), ("maxval", ctypes.c_int),
                ("ascii", ctypes.c_int), ("palette_len", ctypes.c_int), ("inv", ctypes.c_double),
                ("palette", ctypes.c_uint8 * 768)]


# name -> (restype, argtypes)
_VP = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_SZ = ctypes.c_size_t
_PRM = ctypes.POINTER(RefineParams)
_IP = ctypes.POINTER(ctypes.c_int)

SIGNATURES = {
    "sv_status_string": (ctypes.c_char_p, [_I]),
    "sv_last_error": (ctypes.c_char_p, []),
    "sv_version": (_I, []),
    "sv_launch_count": (ctypes.c_ulonglong, []),
    "sv_refine_params_default": (None, [_PRM]),
    "sv_workspace_status": (_I, [_VP, _VP]),
    "sv_census": (_I, [_VP, _I, _I, _I, _I, _I, _VP, _VP]),
    "sv_band_costs": (_I, [_VP, _VP, _VP, _I, _I, _I, _I, _VP, _VP]),
    "sv_aggregate_path": (_I, [_VP, _VP, _I, _I, _I, _I, _I, _I, _I, _VP, _VP]),
    "sv_left_to_right": (_I, [_VP, _I, _I, _VP, _VP]),
    "sv_refine_workspace_size": (_SZ, [_I, _I, _PRM]),
    "sv_refine_fullres": (_I, [_VP, _VP, _I, _VP, _I, _I, _PRM, _VP, _VP, _VP, _SZ, _VP]),
    "sv_lr_refine_workspace_size": (_SZ, [_I, _I, _PRM]),
    "sv_lr_refine": (_I, [_VP, _VP, _I, _VP, _I, _I, _D, _PRM, _VP, _VP, _VP, _SZ, _VP]),
    "sv_lr_refine_timed": (_I, [_VP, _VP, _I, _VP, _I, _I, _D, _PRM, _VP, _VP, _VP, _SZ, _VP,
                                ctypes.POINTER(_VP), _I]),
    "sv_refine_fullres_noalloc": (_I, [_VP, _VP, _I, _VP, _I, _I, _PRM, _VP, _VP, _VP]),
    "sv_selftest_wait_timeout": (_I, [ctypes.c_uint, _VP, _VP]),
    "sv_selftest_slot_wait": (_I, [_VP]),
    "sv_batch_lr_refine_workspace_size": (_SZ, [_VP, _I, _PRM]),
    "sv_batch_lr_refine": (_I, [_VP, _I, _I, _D, _PRM, _VP, _SZ, _VP]),
    "sv_batch_config_default": (None, [_VP]),
    "sv_batch_lr_refine_ex": (_I, [_VP, _I, _I, _D, _PRM, _VP, _VP, _SZ, _VP]),
    "sv_netbatch_create": (_I, [_VP, _IP, _IP, _I, _I, _D, _I, _I, _I, _I, _D, _PRM,
                                ctypes.POINTER(_VP)]),
    "sv_netbatch_workspace_size": (_SZ, [_VP]),
    "sv_netbatch_bind": (_I, [_VP, _VP, _VP, _SZ, _VP]),
    "sv_netbatch_run": (_I, [_VP, _VP]),
    "sv_netbatch_predict": (_I, [_VP, _VP]),
    "sv_netbatch_disparity": (_I, [_VP, _I, ctypes.POINTER(_VP)]),
    "sv_netbatch_trace": (_I, [_VP, _IP, _I, _IP, _VP]),
    "sv_netbatch_data_status": (_I, [_VP, _VP]),
    "sv_netbatch_destroy": (None, [_VP]),
    "sv_predict_consistent_workspace_size": (_SZ, [_VP, _I, _I, _I, _I]),
    "sv_predict_consistent": (_I, [_VP, _VP, _VP, _I, _I, _I, _I, _D, _I, _I, _I, _D, _I, _VP,
                                   ctypes.POINTER(ctypes.c_longlong), _VP, _SZ, _VP]),
    "sv_lr_consistency": (_I, [_VP, _VP, _I, _I, _D, _VP, _VP, _VP]),
    "sv_fill_invalid_workspace_size": (_SZ, [_I, _I]),
    "sv_fill_invalid": (_I, [_VP, _VP, _I, _I, _VP, _VP, _SZ, _VP]),
    "sv_peak_workspace_size": (_SZ, []),
    "sv_peak": (_I, [_VP, ctypes.c_long, _D, _VP, _VP, _SZ, _VP]),
    "sv_work_width": (_I, [_VP, ctypes.c_long, _I, _D, _I, _D, _VP, _VP, _SZ, _VP]),
    "sv_image_info": (_I, [ctypes.c_char_p, _SZ, ctypes.POINTER(RawImage)]),
    "sv_image_decode_raw": (_I, [ctypes.c_char_p, _SZ, _VP, _SZ, ctypes.POINTER(RawImage)]),
    "sv_image_decode_batch": (_I, [_I, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(_SZ),
                                   ctypes.POINTER(_VP), ctypes.POINTER(_SZ),
                                   ctypes.POINTER(RawImage), _IP, _I]),
    "sv_raw_to_float": (_I, [_VP, ctypes.POINTER(RawImage), _VP, _VP, _VP]),
    "sv_median_workspace_size": (_SZ, [_I, _I]),
    "sv_median_filter": (_I, [_VP, _I, _I, _I, _I, _VP, _VP, _SZ, _VP]),
    "sv_postproc_workspace_size": (_SZ, [_I, _I, _I]),
    "sv_slic_count": (_I, [_I, _I, _I]),
    "sv_slic": (_I, [_VP, _I, _I, _I, _D, _I, _VP, _VP, _SZ, _VP]),
    "sv_plane_snap": (_I, [_VP, _VP, _I, _I, _VP, _I, _D, _D, _I, ctypes.c_uint32, _VP, _VP, _SZ,
                           _VP]),
    "sv_refine_disparity_workspace_size": (_SZ, [_I, _I, _PRM, _I]),
    "sv_refine_disparity": (_I, [_VP, _VP, _I, _VP, _VP, _I, _I, _D, _PRM, _I, _I, _D, _D, _VP,
                                 _VP, _VP, _SZ, _VP]),
    "sv_lr_refine_band": (_I, [_VP, _VP, _I, _VP, _VP, _I, _I, _D, _PRM, _VP, _VP, _VP, _SZ,
                               _VP]),
    "sv_band_param_count": (ctypes.c_long, []),
    "sv_band_create": (_I, [_VP, ctypes.c_long, ctypes.POINTER(_VP)]),
    "sv_band_destroy": (None, [_VP]),
    "sv_band_get_params": (_I, [_VP, _VP, ctypes.c_long]),
    "sv_band_features_workspace_size": (_SZ, [_I, _I]),
    "sv_band_conf_features": (_I, [_VP, _VP, _I, _I, _VP, _VP]),
    "sv_band_rule_centre": (_I, [_VP, _VP, _I, _I, _D, _VP, _VP]),
    "sv_predict_confidence": (_I, [_VP, _I, _I, _I, _I, _I, _I, _VP, _SZ, _VP, _VP, _VP]),
    "sv_band_features": (_I, [_VP, _VP, _I, _VP, _I, _I, _I, _VP, _VP, _SZ, _VP]),
    "sv_band_workspace_size": (_SZ, [_I, _I, _I]),
    "sv_band_forward": (_I, [_VP, _VP, _I, _I, _I, _VP, _VP, _SZ, _VP]),
    "sv_band_grads": (_I, [_VP, _VP, _VP, _VP, _I, _I, _I, _VP, _VP, _VP, _SZ, _VP]),
    "sv_band_train_step": (_I, [_VP, _VP, _VP, _VP, _I, _I, _I, _D, _VP, _VP, _SZ, _VP]),
    "sv_band_targets": (_I, [_VP, _VP, _VP, ctypes.c_long, _D, _VP, _VP, _VP]),
    "sv_band_apply": (_I, [_VP, _VP, _I, _I, _D, _D, _I, _I, _D, _VP, _VP, _VP]),
    "sv_trainer_create": (_I, [_VP, _I, _VP, ctypes.c_long, ctypes.POINTER(_VP)]),
    "sv_trainer_destroy": (None, [_VP]),
    "sv_trainer_param_count": (ctypes.c_long, [_VP]),
    "sv_trainer_get_params": (_I, [_VP, _VP, ctypes.c_long]),
    "sv_trainer_get_grads": (_I, [_VP, _VP, ctypes.c_long]),
    "sv_trainer_set_params": (_I, [_VP, _VP, ctypes.c_long]),
    "sv_trainer_set_grads": (_I, [_VP, _VP, ctypes.c_long]),
    "sv_train_workspace_size": (_SZ, [_VP, _I, _I, _I]),
    "sv_train_grads": (_I, [_VP, _VP, _VP, _VP, _VP, _I, _I, _I, _VP, _VP, _VP, _SZ, _VP]),
    "sv_train_adam": (_I, [_VP, _D, _D, _VP]),
    "sv_trainer_reset_adam": (_I, [_VP]),
    "sv_net_create": (_I, [_VP, _I, _VP, ctypes.c_long, ctypes.POINTER(_VP)]),
    "sv_net_destroy": (None, [_VP]),
    "sv_resize": (_I, [_VP, _I, _I, _I, _I, _VP, _VP]),
    "sv_avgpool2": (_I, [_VP, _I, _I, _I, _VP, _VP]),
    "sv_forward_workspace_size": (_SZ, [_VP, _I, _I]),
    "sv_stereonet_forward": (_I, [_VP, _VP, _VP, _I, _I, _VP, _VP, _VP, _VP, _VP, _I, _VP,
                                  _SZ, _VP]),
    "sv_predict_workspace_size": (_SZ, [_VP, _I, _I, _I]),
    "sv_predict_auto": (_I, [_VP, _VP, _VP, _I, _I, _I, _D, _I, _I, _I, _I, _VP, _VP, _IP,
                             _IP, _IP, _VP, _SZ, _VP]),
    "sv_predict_at_scale": (_I, [_VP, _VP, _VP, _I, _I, _I, _I, _I, _VP, _VP, _IP, _IP,
                                 _VP, _SZ, _VP]),
    "sv_predict_refine": (_I, [_VP, _VP, _VP, _I, _I, _I, _D, _I, _I, _I, _I, _VP, _VP, _IP,
                               _IP, _IP, _VP, _SZ, _D, _PRM, _VP, _VP, _VP, _SZ, _VP]),
}

_lib = None


def load():
    """Load the library once; raise if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libsv_b200.so is not built (%s); run __graft_entry__.build() or "
            "python from-scratch-stereo-vision_b200/build.py" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name, None)
        if f is None:          # tests/test_boundary.py requires every symbol
            continue
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return sorted(SIGNATURES)


def check(rc: int, what: str) -> None:
    if rc == SV_OK:
        return
    lib = load()
    detail = lib.sv_last_error().decode(errors="replace")
    msg = "%s: %s (%s)" % (what, lib.sv_status_string(rc).decode(), detail)
    if rc in (SV_ERR_CUDA, SV_ERR_TIMEOUT):
        raise RuntimeError(msg)
    raise ValueError(msg)


def raise_last(what: str) -> None:
    """Raise the argument error a *_workspace_size() call recorded (it
    returns 0 for parameters the library rejects)."""
    raise ValueError("%s: %s" % (what, load().sv_last_error().decode(errors="replace")))


def default_params() -> RefineParams:
    p = RefineParams()
    load().sv_refine_params_default(ctypes.byref(p))
    return p
