"""The C oracle against the golden fixtures made by running the reference.

These are CPU tests: they pin the FP64 restatement (oracle/sv_oracle.c)
bit-for-bit to the reference's own outputs, which is what lets the GPU tests
use the oracle as their checker at sizes the Python reference cannot reach.
"""

import hashlib

import numpy as np
import pytest

from conftest import bits, golden


def sha(a, dtype=np.float64):
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=dtype)).tobytes()).hexdigest()


def test_weights_pack_matches_reference(net, golden_meta):
    assert net.n_params() == golden_meta["n_params"] == 9921
    assert sha(net.flat) == golden_meta["weights_sha256"]
    assert net.target_peak == golden_meta["target_peak"] == 34


def test_primitives(orc):
    g = golden("primitives.npz")
    got = np.array([orc.fexp(float(x)) for x in g["fexp_x"]])
    assert np.array_equal(bits(got), bits(g["fexp"]))
    img = g["img"]
    for key in g.files:
        if key.startswith("resize_"):
            W2, H2 = map(int, key[7:].split("x"))
            assert np.array_equal(bits(orc.resize_gray(img, 13, 9, W2, H2)), bits(g[key])), key
    ap, _, _ = orc.avgpool2(img, 1, 9, 13)
    assert np.array_equal(bits(ap), bits(g["avgpool"]))
    assert orc.peak(g["peak_in"]) == g["peak"][0]


@pytest.fixture(scope="module")
def small():
    g = golden("refine_small.npz")
    W, H = g["left"].shape[1], g["left"].shape[0]
    L = g["left"].astype(np.float64).ravel() / 255.0
    R = g["right"].astype(np.float64).ravel() / 255.0
    return g, W, H, L, R


def test_census_exact(orc, small):
    g, W, H, L, R = small
    assert np.array_equal(orc.census(L, W, H, 4, 3), g["census_l_4x3"])
    assert np.array_equal(orc.census(R, W, H, 4, 3), g["census_r_4x3"])
    assert np.array_equal(orc.census(L, W, H, 2, 2), g["census_l_2x2"])
    assert np.array_equal(orc.census(R, W, H, 1, 1), g["census_r_1x1"])


def test_band_costs_and_paths_exact(orc, small):
    g, W, H, L, R = small
    base = g["base"]
    C = orc.band_costs(g["census_l_4x3"], g["census_r_4x3"], L, R, base, W, H, 10, 0.0, 20.0,
                       66.0, g["disp0"], 0.0, 4.0)
    assert np.array_equal(C, g["costs_R10"].astype(np.float64))
    dirs = [(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, 1), (1, -1), (-1, -1)]
    S = np.zeros(W * H * 21)
    for i, (dx, dy) in enumerate(dirs):
        S1 = np.zeros(W * H * 21)
        orc.aggregate_path(C, base, W, H, 21, 12.0, 150.0, dx, dy, S1)
        assert np.array_equal(S1, g["path%d_R10" % i].astype(np.float64)), (dx, dy)
        orc.aggregate_path(C, base, W, H, 21, 12.0, 150.0, dx, dy, S)
    assert np.array_equal(S, g["S_R10"].astype(np.float64))


def test_refine_fullres_exact(orc, small):
    g, W, H, L, R = small
    d0 = g["disp0"]
    out, conf = orc.refine_fullres(L, R, d0, W, H, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                                   return_conf=True)
    assert np.array_equal(bits(out), bits(g["refine_R10"]))
    assert np.array_equal(bits(conf), bits(g["conf_R10"]))
    assert np.array_equal(bits(orc.refine_fullres(L, R, d0, W, H)), bits(g["refine_default"]))
    assert np.array_equal(bits(orc.refine_fullres(L, R, d0, W, H, R=4, P1=12.0, P2=150.0,
                                                  paths=4, rx=4, ry=3)),
                          bits(g["refine_R4_paths4"]))
    assert np.array_equal(bits(orc.refine_fullres(L, R, d0, W, H, R=6, P1=8.0, P2=96.0, rx=3,
                                                  ry=3, uniq=0.15)), bits(g["refine_uniq"]))
    Rf = int(g["fullrange_R"][0])
    assert np.array_equal(bits(orc.refine_fullres(L, R, np.full(W * H, float(Rf)), W, H, R=Rf,
                                                  P1=12.0, P2=150.0, rx=4, ry=3)),
                          bits(g["fullrange"]))


def test_left_to_right_exact(orc, small):
    g, W, H, L, R = small
    assert np.array_equal(bits(orc.left_to_right(g["disp0"], W, H)), bits(g["l2r"]))


def test_lr_refine_exact(orc, small):
    g, W, H, L, R = small
    out, st = orc.lr_refine(L, R, g["disp0"], W, H, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4,
                            ry=3)
    assert np.array_equal(bits(out), bits(g["lr_out"]))
    assert np.array_equal(st, g["lr_status"].astype(np.int32))
    out, st = orc.lr_refine(L, R, g["disp0"], W, H)
    assert np.array_equal(bits(out), bits(g["lr_default_out"]))
    assert np.array_equal(st, g["lr_default_status"].astype(np.int32))


def test_network_exact(orc, net):
    g = golden("network_small.npz")
    H, W = g["left"].shape
    L = g["left"].astype(np.float64).ravel() / 255.0
    R = g["right"].astype(np.float64).ravel() / 255.0
    gh, _, _ = orc.avgpool2(L, 1, H, W)
    d0, d1, d2 = orc.stereonet_forward(net, L, R, H, W, gh, L)
    assert np.array_equal(bits(d0), bits(g["d0"]))
    assert np.array_equal(bits(d1), bits(g["d1"]))
    assert np.array_equal(bits(d2), bits(g["d2"]))
    df, dw, Ww, Hw = orc.predict_at_scale(net, L, R, W, H, 48)
    assert [Ww, Hw] == list(g["pas_dims"])
    assert np.array_equal(bits(df), bits(g["pas_full"]))
    assert np.array_equal(bits(dw), bits(g["pas_work"]))


def test_network_rejects_narrow_input(orc, net):
    # the reference's invalid_mask raises IndexError when the quarter width <= D-2
    L = np.zeros(40 * 30)
    with pytest.raises(ValueError):
        orc.predict(net, L, L, 40, 30)


def test_config_small_end_to_end(orc, net):
    g = golden("config_small.npz")
    H, W = g["left"].shape
    L = g["left"].astype(np.float64).ravel() / 255.0
    R = g["right"].astype(np.float64).ravel() / 255.0
    df, dw, Ww, Hw = orc.predict_auto(net, L, R, W, H)
    assert [Ww, Hw] == list(g["dims"])
    assert np.array_equal(bits(df), bits(g["disp0"]))
    assert np.array_equal(bits(dw), bits(g["disp_work"]))
    out, st = orc.lr_refine(L, R, df, W, H, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    assert np.array_equal(bits(out), bits(g["out"]))
    assert np.array_equal(st, g["status"].astype(np.int32))


def test_config_full_digests(orc, net, svb, golden_meta):
    m = golden_meta["config_full"]
    p = svb.synth.config_full()
    assert sha(np.concatenate([p.left.ravel(), p.right.ravel()]), np.uint8) == m["images_sha256"]
    L, R = p.gray("left").ravel(), p.gray("right").ravel()
    df, dw, Ww, Hw = orc.predict_auto(net, L, R, p.W, p.H)
    assert [Ww, Hw] == m["work"]
    assert sha(df) == m["disp0_sha256"]
    assert sha(dw) == m["disp_work_sha256"]
    out, st = orc.lr_refine(L, R, df, p.W, p.H, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    assert sha(out) == m["out_sha256"]
    assert sha(st, np.int8) == m["status_sha256"]


# ------------------------------------------- rest of refine_disparity
@pytest.mark.parametrize("tag", ["a", "b"])
def test_postproc_oracle_vs_reference(orc, tag):
    """slic, plane_snap, median_filter and refine_disparity (stereonet.py:
    2231-2259, 5394-5563, 5865-5883) bit-for-bit against the reference."""
    g = golden("postproc.npz")
    W, H, step = map(int, g[tag + "_dims"])
    rgb, d, st = g[tag + "_rgb"], g[tag + "_lr"], g[tag + "_status"]
    assert np.array_equal(orc.slic(rgb, W, H, step)[0], g[tag + "_slic"])
    assert np.array_equal(orc.slic(rgb, W, H, step, 20.0, 3)[0], g[tag + "_slic_c20_it3"])
    snap = orc.plane_snap(d, rgb, W, H, valid=st == 0, step=step, thr=1.0, min_inl=0.4)
    assert np.array_equal(bits(snap), bits(g[tag + "_snap"]))
    assert np.array_equal(bits(orc.plane_snap(d, rgb, W, H, step=step)),
                          bits(g[tag + "_snap_novalid"]))
    assert np.array_equal(bits(orc.median_filter(d, W, H)), bits(g[tag + "_median"]))
    assert np.array_equal(bits(orc.median_filter(d, W, H, 2, 2)), bits(g[tag + "_median_r2p2"]))
    L, R = g[tag + "_left"].ravel() / 255.0, g[tag + "_right"].ravel() / 255.0
    rd, rs = orc.refine_disparity(L, R, rgb, g[tag + "_disp0"], W, H, plane_step=step)
    assert np.array_equal(bits(rd), bits(g[tag + "_refine_disparity"]))
    assert np.array_equal(rs, g[tag + "_refine_disparity_status"])
    rd2, _ = orc.refine_disparity(L, R, rgb, g[tag + "_disp0"], W, H, planes=False)
    assert np.array_equal(bits(rd2), bits(g[tag + "_refine_disparity_noplanes"]))


def test_slic_uncovered_pixels_oracle_vs_reference(orc):
    """Pixels no cluster window covers keep their labels (stereonet.py:
    5409-5432); on this image that happens in SLIC iterations 3 and 4."""
    g = golden("postproc.npz")
    W, H, step = map(int, g["u_dims"])
    assert np.array_equal(orc.slic(g["u_rgb"], W, H, step, float(g["u_comp"]))[0], g["u_slic"])
    snap = orc.plane_snap(g["u_disp"], g["u_rgb"], W, H, step=step, thr=5.0, min_inl=0.3)
    assert np.array_equal(bits(snap), bits(g["u_snap"]))


@pytest.mark.parametrize("tag", ["c", "d"])
def test_predict_consistent_oracle_vs_reference(orc, net, tag):
    """predict_consistent, lr_consistency, fill_invalid (stereonet.py:4974-5076)."""
    g = golden("postproc.npz")
    W, H, ww = map(int, g[tag + "_dims"])
    dl, dr = g[tag + "_lrc_in"]
    v = orc.lr_consistency(dl, dr, W, H, 1.5)
    assert np.array_equal(v, g[tag + "_lrc"])
    assert np.array_equal(bits(orc.fill_invalid(dl, v, W, H)), bits(g[tag + "_fill"]))
    d, frac = orc.predict_consistent(net, g[tag + "_left"].ravel() / 255.0,
                                     g[tag + "_right"].ravel() / 255.0, W, H,
                                     work_width=None if ww == 0 else ww)
    assert np.array_equal(bits(d), bits(g[tag + "_consistent"])) and frac == float(g[tag + "_frac"])
