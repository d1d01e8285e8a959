"""GPU StereoNet forward and resolution selection against the FP64 oracle.

The network runs in FP32 on the GPU; the reference (and the oracle, pinned
to it bit-for-bit) in FP64.  Tolerance: 2e-3 px max abs on every disparity
output (the observed FP32 error is ~1e-5 px).  Resampling is FP64 on both
sides and must be bit-identical.
"""

import numpy as np
import pytest

from conftest import bits, golden

pytestmark = pytest.mark.gpu

TOL_PX = 2e-3


def test_resize_and_avgpool_bit_exact(svb):
    g = golden("primitives.npz")
    img = g["img"]
    for key in g.files:
        if key.startswith("resize_"):
            W2, H2 = map(int, key[7:].split("x"))
            got = svb.network.resize_gray(img, 13, 9, W2, H2)
            assert np.array_equal(bits(got), bits(g[key])), key
    ap, H2, W2 = svb.network.avgpool2(img, 1, 9, 13)
    assert (H2, W2) == (4, 6)
    assert np.array_equal(bits(ap), bits(g["avgpool"]))


def test_resize_list_io(svb):
    g = golden("primitives.npz")
    out = svb.network.resize_gray(list(g["img"]), 13, 9, 29, 17)
    assert isinstance(out, list) and np.array_equal(bits(out), bits(g["resize_29x17"]))


def test_forward_vs_golden(svb, net):
    g = golden("network_small.npz")
    H, W = g["left"].shape
    L = g["left"].astype(np.float64).ravel() / 255.0
    R = g["right"].astype(np.float64).ravel() / 255.0
    gh, _, _ = svb.network.avgpool2(L, 1, H, W)
    d0, d1, d2 = svb.network.forward(net, L, R, H, W, gh, L)
    for got, key in ((d0, "d0"), (d1, "d1"), (d2, "d2")):
        assert got.shape == g[key].shape
        assert np.max(np.abs(got - g[key])) < TOL_PX, key


def test_predict_at_scale_vs_golden(svb, net):
    g = golden("network_small.npz")
    H, W = g["left"].shape
    L = g["left"].astype(np.float64).ravel() / 255.0
    R = g["right"].astype(np.float64).ravel() / 255.0
    df, dw, Ww, Hw = svb.network.predict_at_scale(net, L, R, W, H, 48, verbose=False)
    assert [Ww, Hw] == list(g["pas_dims"])
    assert np.max(np.abs(df - g["pas_full"])) < TOL_PX
    assert np.max(np.abs(dw - g["pas_work"])) < TOL_PX


@pytest.mark.parametrize("W,H", [(64, 48), (97, 61), (160, 120)])
def test_predict_vs_oracle_u8_and_f64(svb, orc, net, W, H):
    pair = svb.synth.make_pair(W + H, W, H, 2.0, 30.0)
    L, R = pair.gray("left").ravel(), pair.gray("right").ravel()
    ref = orc.predict(net, L, R, W, H)
    assert np.max(np.abs(svb.network.predict(net, L, R, W, H) - ref)) < TOL_PX
    # uint8 images give the same u/255.0 grays
    got = svb.network.predict(net, pair.left, pair.right, W, H)
    assert np.max(np.abs(got - ref)) < TOL_PX


def test_predict_auto_config_small(svb, orc, net):
    g = golden("config_small.npz")
    H, W = g["left"].shape
    (df, dw, Ww, Hw), trace = svb.network.predict_auto(net, g["left"], g["right"], W, H,
                                                       verbose=False, return_trace=True)
    assert [Ww, Hw] == list(g["dims"])
    err = np.abs(df - g["disp0"])
    assert err.max() < TOL_PX
    # downstream: refinement from the GPU disparity vs from the FP64 one
    kw = dict(tol=2.0, R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    out, st = svb.refine.lr_refine(g["left"], g["right"], df, W, H, **kw)
    same = np.mean((bits(out) == bits(g["out"])) & (st.astype(np.int8) == g["status"]))
    # Pixels whose refined value is the network's own disparity (edge winners,
    # mismatches) carry its FP32 error, so bit-identity is not expected there;
    # a pixel counts as changed when it moved by more than that error.
    moved = np.mean(np.abs(out - g["out"]) > 10 * TOL_PX)
    st_same = np.mean(st.astype(np.int8) == g["status"])
    print("config 160x120: max err %.2e px, mean %.2e px, refined bit-identical %.4f, "
          "status identical %.4f, moved %.4f" % (err.max(), err.mean(), same, st_same, moved))
    assert st_same > 0.99 and moved < 0.01


def test_predict_auto_config_full(svb, orc, net, golden_meta):
    p = svb.synth.config_full()
    L, R = p.gray("left").ravel(), p.gray("right").ravel()
    ref, rtrace = orc.predict_auto(net, L, R, p.W, p.H, return_trace=True)
    (df, dw, Ww, Hw), trace = svb.network.predict_auto(net, p.left, p.right, p.W, p.H,
                                                       verbose=False, return_trace=True)
    assert [Ww, Hw] == golden_meta["config_full"]["work"] == [ref[2], ref[3]]
    assert trace == rtrace
    err = np.abs(df - ref[0])
    assert err.max() < TOL_PX
    print("config 450x375: max err %.2e px, mean %.2e px" % (err.max(), err.mean()))


def test_pipeline_matches_drop_ins(svb, net):
    import torch
    p = svb.synth.config_full()
    pipe = svb.pipeline.PairPipeline(p.W, p.H, net)
    hl, hr = torch.from_numpy(p.left.ravel()), torch.from_numpy(p.right.ravel())
    # first run records the passes as CUDA graphs, the second replays them
    out, st = (t.clone() for t in pipe.run_host(hl, hr))
    out2, st2 = pipe.run_host(hl, hr)
    assert np.array_equal(bits(out.numpy()), bits(out2.numpy()))
    assert np.array_equal(st.numpy(), st2.numpy())
    # drop-ins on the default stream (no graphs) give the same bits
    df, _, _, _ = svb.network.predict_auto(net, p.left, p.right, p.W, p.H, verbose=False)
    o2, s2 = svb.refine.lr_refine(p.left, p.right, df, p.W, p.H, tol=2.0, R=10, P1=12.0,
                                  P2=150.0, rx=4, ry=3)
    assert np.array_equal(bits(out.numpy()), bits(o2))
    assert np.array_equal(st.numpy(), s2)


def test_narrow_input_raises(svb, net):
    L = np.zeros(40 * 30)
    with pytest.raises(ValueError):
        svb.network.predict(net, L, L, 40, 30)
