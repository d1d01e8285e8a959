"""The drop-ins keep the reference's signatures, and install(SN) rebinds
them in an exec'd namespace (host-only checks)."""

import inspect
import json
import os

import pytest

from conftest import GOLDEN

with open(os.path.join(GOLDEN, "signatures.json")) as f:
    REF_SIGS = json.load(f)


def _params(sig_str):
    # "(a, b=1, **kw)" -> [(name, default-or-None, kind)]
    ns = {}
    exec("def f%s: pass" % sig_str, ns)
    return [(p.name, p.default, p.kind) for p in inspect.signature(ns["f"]).parameters.values()]


@pytest.mark.parametrize("name", sorted(n for n in REF_SIGS if n != "StereoNet.forward"))
def test_signature_kept(svb, name):
    fn = svb.shim.DROP_INS[name]
    ref = _params(REF_SIGS[name])
    ours = [(p.name, p.default, p.kind) for p in inspect.signature(fn).parameters.values()]
    assert ours[:len(ref)] == ref, (name, ours, ref)
    # anything extra is an optional trailing keyword
    for n, d, k in ours[len(ref):]:
        assert d is not inspect.Parameter.empty


def test_forward_signature_kept(svb):
    ref = _params(REF_SIGS["StereoNet.forward"])
    ours = [(p.name, p.default, p.kind)
            for p in inspect.signature(svb.shim._forward).parameters.values()]
    assert ours == ref


def test_install_and_uninstall(svb):
    class StereoNet:
        def forward(self, left, right, H, W, guide_half, guide_full):
            return "reference"

    orig = {n: (lambda *a, **k: n) for n in svb.shim.DROP_INS}
    SN = dict(orig)
    SN["StereoNet"] = StereoNet
    svb.shim.install(SN)
    for n, fn in svb.shim.DROP_INS.items():
        assert SN[n] is fn
    assert StereoNet.forward is svb.shim._forward
    svb.shim.uninstall(SN)
    for n in svb.shim.DROP_INS:
        assert SN[n] is orig[n]
    assert StereoNet.forward(None, 0, 0, 0, 0, 0, 0) == "reference"
