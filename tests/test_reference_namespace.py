"""The drop-ins inside the reference's own exec'd namespace.

Every caller of the reference runs ``exec`` of stereonet.py into a dict and
looks functions up there (eval_real.py:41-44, serve.py:34-37).  These tests
do exactly that with the real reference, when its checkout is available
(SV_REFERENCE_DIR, or a ``reference`` directory beside this repository), and
skip with that reason otherwise:

* on the host: the reference's own ``load_model`` (stereonet.py:1810-1854)
  builds its ``StereoNet``; the drop-ins read its architecture from
  ``net.filt.c1.oc``, ``net.ref1.convs[0].oc`` and ``net.ref1.dilations``
  and its parameters from ``all_params()``, and must get the checkpoint this
  package ships; ``install(SN)`` rebinds the real names and the real class;
* on the GPU: the reference's ``predict_auto`` name, now the drop-in, runs
  with that reference ``StereoNet`` object, and the reference's own Python
  ``lr_refine`` (left in place) reaches the GPU ``refine_fullres`` through
  the namespace; both match the fixtures the reference produced.
"""

import os

import numpy as np
import pytest

from conftest import REPO, bits, golden


def _ref_dir():
    for d in (os.environ.get("SV_REFERENCE_DIR"), os.path.join(REPO, os.pardir, "reference")):
        if d and os.path.isfile(os.path.join(d, "stereonet.py")):
            return os.path.abspath(d)
    return None


def _load_ns():
    d = _ref_dir()
    if d is None:
        pytest.skip("reference checkout not available (set SV_REFERENCE_DIR)")
    src = open(os.path.join(d, "stereonet.py")).read().replace(
        "if __name__ == '__main__':\n    run_demo()\n", "")
    SN = {"__name__": "stereonet_ns"}
    exec(src, SN)
    return SN, SN["load_model"](os.path.join(d, "stereonet_weights.txt"))


@pytest.fixture(scope="module")
def ref_ns():
    return _load_ns()


def test_weights_read_from_reference_object(svb, ref_ns):
    SN, rnet = ref_ns
    w = svb.network._weights_of(rnet)
    ours = svb.weights.load_model()
    assert w.arch.feat_C == ours.arch.feat_C and w.arch.cost_C == ours.arch.cost_C
    assert w.arch.D == ours.arch.D and w.arch.refine_C == ours.arch.refine_C
    assert tuple(w.arch.refine_dil) == tuple(ours.arch.refine_dil)
    assert np.array_equal(bits(w.flat), bits(ours.flat))


def test_install_into_reference_namespace(svb, ref_ns):
    SN, _ = ref_ns
    orig_forward = SN["StereoNet"].forward
    saved = svb.shim.install(SN)
    try:
        for name, fn in svb.shim.DROP_INS.items():
            assert SN[name] is fn, name
            assert name in saved, name            # every name exists in the reference
        assert SN["StereoNet"].forward is svb.shim._forward
    finally:
        svb.shim.uninstall(SN)
    assert SN["StereoNet"].forward is orig_forward
    assert SN["lr_refine"] is saved["lr_refine"]


@pytest.mark.gpu
def test_reference_namespace_runs_on_gpu(svb, ref_ns):
    SN, rnet = ref_ns
    g = golden("config_small.npz")
    H, W = g["left"].shape
    L = (g["left"].astype(np.float64) / 255.0).ravel().tolist()
    R = (g["right"].astype(np.float64) / 255.0).ravel().tolist()
    svb.shim.install(SN)
    SN["lr_refine"] = SN["__sv_b200_saved__"]["lr_refine"]   # the reference's own Python
    try:
        df, _, Ww, Hw = SN["predict_auto"](rnet, L, R, W, H, verbose=False)
        assert [Ww, Hw] == list(g["dims"])
        assert np.max(np.abs(np.asarray(df) - g["disp0"])) < 2e-3
        out, status = SN["lr_refine"](L, R, g["disp0"].tolist(), W, H, tol=2.0, R=10, P1=12.0,
                                      P2=150.0, rx=4, ry=3)
        assert np.array_equal(bits(out), bits(g["out"]))
        assert np.array_equal(np.asarray(status, dtype=np.int64), g["status"].astype(np.int64))
    finally:
        svb.shim.uninstall(SN)
