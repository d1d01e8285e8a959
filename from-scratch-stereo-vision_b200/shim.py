"""Install the GPU drop-ins into an exec'd reference namespace.

The reference has no import system: every caller runs ``exec`` of
stereonet.py into a dict and looks functions up there (eval_real.py:41-44,
serve.py:34-37, test_stereonet.py:18-22).  Inside that dict the reference's
functions call each other through the same dict, so rebinding a name
redirects every caller, e.g. ``lr_refine`` -> ``refine_fullres`` and
``reconstruct_from_pair`` -> ``refine_disparity``:

    SN = {}
    exec(open("stereonet.py").read(), SN)
    sv_b200.shim.install(SN)          # census ... predict_auto now run on the GPU
    d, status = SN["refine_disparity"](left, right, rgb, disp0, W, H)

``StereoNet.forward`` is replaced on the class for inference (the GPU
forward keeps no caches for ``backward``; training stays on the
reference's own path).  ``uninstall(SN)`` restores the originals.
"""

from __future__ import annotations

from . import image, network, post, refine, train

# reference name -> drop-in
DROP_INS = {
    "census": refine.census,
    "band_costs": refine.band_costs,
    "_aggregate_path": refine._aggregate_path,
    "refine_fullres": refine.refine_fullres,
    "left_to_right": refine.left_to_right,
    "lr_refine": refine.lr_refine,
    "resize_gray": network.resize_gray,
    "avgpool2": network.avgpool2,
    "predict": network.predict,
    "predict_at_scale": network.predict_at_scale,
    "predict_auto": network.predict_auto,
    "_peak": network._peak,
    "median_filter": post.median_filter,
    "slic": post.slic,
    "plane_snap": post.plane_snap,
    "refine_disparity": post.refine_disparity,
    "predict_consistent": network.predict_consistent,
    "lr_consistency": post.lr_consistency,
    "fill_invalid": post.fill_invalid,
    "read_png": image.read_png,
    "read_pnm": image.read_pnm,
    "read_image": image.read_image,
    "train_grads": train.train_grads,
    "train_step": train.train_step,
}

_SAVED = "__sv_b200_saved__"


def _forward(self, left, right, H, W, guide_half, guide_full):
    return network.forward(self, left, right, H, W, guide_half, guide_full)


def install(SN: dict, names=None) -> dict:
    """Rebind the hot-path names in ``SN``; returns the originals."""
    saved = SN.setdefault(_SAVED, {})
    for name in (names or DROP_INS):
        if name in SN and name not in saved:
            saved[name] = SN[name]
        SN[name] = DROP_INS[name]
    cls = SN.get("StereoNet")
    if cls is not None and (names is None or "StereoNet.forward" in names):
        if "StereoNet.forward" not in saved:
            saved["StereoNet.forward"] = cls.forward
        cls.forward = _forward
    return saved


def uninstall(SN: dict) -> None:
    saved = SN.pop(_SAVED, {})
    for name, fn in saved.items():
        if name == "StereoNet.forward":
            SN["StereoNet"].forward = fn
        else:
            SN[name] = fn
