"""The rest of refine_disparity on the GPU -- median_filter, slic,
plane_snap, refine_disparity (stereonet.py:2231-2259, 5394-5563,
5865-5883) -- bit-identical to the reference's fixtures and to the FP64
oracle."""

import numpy as np
import pytest

from conftest import bits, golden

pytestmark = pytest.mark.gpu

KW = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_postproc_vs_reference_fixtures(svb, tag):
    g = golden("postproc.npz")
    W, H, step = map(int, g[tag + "_dims"])
    rgb, d, st = g[tag + "_rgb"], g[tag + "_lr"], g[tag + "_status"]
    lab, n = svb.post.slic(rgb, W, H, step)
    assert np.array_equal(lab, g[tag + "_slic"]) and n == lab.max() + 1
    assert np.array_equal(svb.post.slic(rgb, W, H, step, 20.0, 3)[0], g[tag + "_slic_c20_it3"])
    snap = svb.post.plane_snap(d, rgb, W, H, valid=st == 0, step=step, thr=1.0, min_inl=0.4)
    assert np.array_equal(bits(snap), bits(g[tag + "_snap"]))
    assert np.array_equal(bits(svb.post.plane_snap(d, rgb, W, H, step=step)),
                          bits(g[tag + "_snap_novalid"]))
    assert np.array_equal(bits(svb.post.median_filter(d, W, H)), bits(g[tag + "_median"]))
    assert np.array_equal(bits(svb.post.median_filter(d, W, H, radius=2, passes=2)),
                          bits(g[tag + "_median_r2p2"]))
    rd, rs = svb.post.refine_disparity(g[tag + "_left"], g[tag + "_right"], rgb, g[tag + "_disp0"],
                                       W, H, plane_step=step)
    assert np.array_equal(bits(rd), bits(g[tag + "_refine_disparity"]))
    assert np.array_equal(np.asarray(rs), g[tag + "_refine_disparity_status"])
    rd2, _ = svb.post.refine_disparity(g[tag + "_left"], g[tag + "_right"], rgb, g[tag + "_disp0"],
                                       W, H, planes=False)
    assert np.array_equal(bits(rd2), bits(g[tag + "_refine_disparity_noplanes"]))


def test_slic_uncovered_pixels(svb):
    g = golden("postproc.npz")
    W, H, step = map(int, g["u_dims"])
    assert np.array_equal(svb.post.slic(g["u_rgb"], W, H, step, float(g["u_comp"]))[0], g["u_slic"])
    snap = svb.post.plane_snap(g["u_disp"], g["u_rgb"], W, H, step=step, thr=5.0, min_inl=0.3)
    assert np.array_equal(bits(snap), bits(g["u_snap"]))


def _rgb(p):
    gl = p.left.astype(np.float64) / 255.0
    h, w = gl.shape
    yy, xx = np.mgrid[0:h, 0:w]
    rgb = np.stack([gl, 0.5 * gl + 0.5 * xx / (w - 1), 1.0 - 0.7 * gl * yy / (h - 1)], axis=-1)
    return (np.round(rgb * 255.0) / 255.0).ravel()


@pytest.mark.parametrize("W,H,step", [(320, 240, 12), (173, 91, 9), (450, 375, 16)])
def test_refine_disparity_vs_oracle(svb, orc, W, H, step):
    p = svb.synth.make_pair(W * 7 + H, W, H, 2.0, 40.0, n_planes=(4, 8), lowtex_frac=0.1)
    rgb = _rgb(p)
    d0 = p.disp.ravel() + np.random.default_rng(W).uniform(-3, 3, W * H)
    ref, rst = orc.refine_disparity(p.gray("left").ravel(), p.gray("right").ravel(), rgb, d0, W, H,
                                    plane_step=step)
    got, st = svb.post.refine_disparity(p.left, p.right, rgb, d0, W, H, plane_step=step)
    assert np.array_equal(bits(got), bits(ref))
    assert np.array_equal(np.asarray(st), rst)
    lab_ref, _ = orc.slic(rgb, W, H, step)
    assert np.array_equal(svb.post.slic(rgb, W, H, step)[0], lab_ref)


def test_edge_cases(svb, orc):
    rng = np.random.default_rng(5)
    for W, H, step in [(5, 4, 12), (1, 1, 1), (30, 2, 3), (2, 40, 4), (24, 24, 24)]:
        rgb = np.round(rng.random(3 * W * H) * 255) / 255
        d = rng.uniform(0, 30, W * H)
        d[::7] = -0.0
        assert np.array_equal(svb.post.slic(rgb, W, H, step)[0], orc.slic(rgb, W, H, step)[0])
        for valid in (None, rng.random(W * H) < 0.5, np.zeros(W * H, bool)):
            got = svb.post.plane_snap(d, rgb, W, H, valid=valid, step=step, thr=4.0, min_inl=0.2)
            ref = orc.plane_snap(d, rgb, W, H, valid=valid, step=step, thr=4.0, min_inl=0.2)
            assert np.array_equal(bits(got), bits(ref)), (W, H, step)
        for r, n in ((0, 1), (1, 3), (3, 1)):
            assert np.array_equal(bits(svb.post.median_filter(d, W, H, r, n)),
                                  bits(orc.median_filter(d, W, H, r, n)))


def test_rejects(svb):
    with pytest.raises(ValueError):
        svb.post.median_filter(np.zeros(12), 4, 3, radius=4)
    with pytest.raises(ValueError):
        svb.post.plane_snap(np.zeros(12), np.zeros(36), 4, 3, trials=65)


@pytest.mark.parametrize("tag", ["c", "d"])
def test_predict_consistent_vs_reference(svb, net, tag):
    """stereonet.py:5048-5076; the network is FP32 here, FP64 in the
    reference, so the disparity is compared within the network tolerance
    (2e-3 px) and the valid fraction exactly."""
    g = golden("postproc.npz")
    W, H, ww = map(int, g[tag + "_dims"])
    d, frac = svb.network.predict_consistent(net, g[tag + "_left"], g[tag + "_right"], W, H,
                                             work_width=None if ww == 0 else ww, verbose=False)
    assert frac == float(g[tag + "_frac"])
    assert np.max(np.abs(np.asarray(d) - g[tag + "_consistent"])) < 2e-3


def test_predict_consistent_vs_oracle_large(svb, orc, net):
    p = svb.synth.make_pair(77, 450, 375, 0.0, 80.0, n_planes=(8, 15), lowtex_frac=0.2)
    W, H = p.W, p.H
    ref, rf = orc.predict_consistent(net, p.gray("left").ravel(), p.gray("right").ravel(), W, H)
    got, gf = svb.network.predict_consistent(net, p.left, p.right, W, H, verbose=False)
    # a pixel whose left-right difference sits within FP32 noise of tol may flip
    assert abs(gf - rf) < 1e-3
    close = np.abs(np.asarray(got) - ref) < 2e-3
    assert close.mean() > 0.995


def test_lr_consistency_and_fill_vs_reference(svb):
    """lr_consistency and fill_invalid (stereonet.py:4986-5045) bit-exact."""
    g = golden("postproc.npz")
    for tag in "cd":
        W, H, _ = map(int, g[tag + "_dims"])
        dl, dr = g[tag + "_lrc_in"]
        v = svb.post.lr_consistency(dl, dr, W, H, 1.5)
        assert np.array_equal(np.asarray(v), g[tag + "_lrc"])
        f = svb.post.fill_invalid(dl, g[tag + "_lrc"], W, H)
        assert np.array_equal(bits(f), bits(g[tag + "_fill"]))
    # rows without any valid pixel keep their values; single-pixel rows
    rng = np.random.default_rng(3)
    for W, H in ((1, 5), (7, 1), (2000, 3)):
        d = rng.uniform(0, 9, W * H)
        v = rng.random(W * H) < 0.3
        v[:W] = False
        assert np.array_equal(bits(svb.post.fill_invalid(d, v, W, H)),
                              bits(_fill_ref(d, v, W, H)))


def _fill_ref(d, v, W, H):
    out = d.copy()
    for y in range(H):
        x = 0
        while x < W:
            if v[y * W + x]:
                x += 1
                continue
            s = x
            while x < W and not v[y * W + x]:
                x += 1
            lv = d[y * W + s - 1] if s > 0 else None
            rv = d[y * W + x] if x < W else None
            if lv is None and rv is None:
                continue
            f = rv if lv is None else lv if rv is None else (lv if lv < rv else rv)
            out[y * W + s:y * W + x] = f
    return out
