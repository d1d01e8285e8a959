"""GPU parity of the refinement drop-ins (bit-exact against the reference).

Each test calls the reference-named function (through libsv_b200.so) and
compares it with the golden fixtures made by the reference itself, or with
the C oracle (pinned to those fixtures) on seeded inputs at sizes the oracle
finishes in seconds.  Bit-exact means FP64 bit patterns and integer statuses.
"""

import numpy as np
import pytest

from conftest import bits, golden

pytestmark = pytest.mark.gpu

DIRS = [(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, 1), (1, -1), (-1, -1)]
PIPE = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)   # refine_disparity's defaults


@pytest.fixture(scope="module")
def small():
    g = golden("refine_small.npz")
    H, W = g["left"].shape
    L = g["left"].astype(np.float64).ravel() / 255.0
    R = g["right"].astype(np.float64).ravel() / 255.0
    return g, W, H, L, R


def noisy_disp(pair, seed, noise=3.0):
    rng = np.random.default_rng(seed)
    d = pair.disp.ravel() + rng.uniform(-noise, noise, pair.W * pair.H)
    idx = rng.choice(d.size, d.size // 50, replace=False)
    d[idx[0::3]] = -0.0
    d[idx[1::3]] = np.floor(d[idx[1::3]]) + 0.5
    d[idx[2::3]] = -rng.uniform(0, 1, len(idx[2::3]))
    return d


# ------------------------------------------------------------------ census
def test_census_golden_lists(svb, small):
    g, W, H, L, R = small
    # reference-style call: flat Python lists in, list of ints out
    out = svb.refine.census(list(L), W, H, 4, 3)
    assert isinstance(out, list) and out == [int(v) for v in g["census_l_4x3"]]
    assert np.array_equal(svb.refine.census(R, W, H, 4, 3), g["census_r_4x3"])
    assert np.array_equal(svb.refine.census(L, W, H, 2, 2), g["census_l_2x2"])
    assert np.array_equal(svb.refine.census(R, W, H, 1, 1), g["census_r_1x1"])


@pytest.mark.parametrize("dtype", [np.uint8, np.float32, np.float64])
@pytest.mark.parametrize("shape,win", [((37, 23), (4, 3)), ((5, 3), (4, 3)), ((130, 67), (3, 2)),
                                       ((1, 9), (1, 1)), ((64, 1), (2, 2))])
def test_census_dtypes_and_edges(svb, orc, dtype, shape, win):
    W, H = shape
    rng = np.random.default_rng(W * 131 + H)
    u8 = rng.integers(0, 256, W * H).astype(np.uint8)
    u8[::7] = u8[0]                                  # equal neighbours: strict < matters
    img = u8 if dtype == np.uint8 else (u8.astype(np.float64) / 255.0).astype(dtype)
    ref = orc.census(img.astype(np.float64), W, H, *win)
    assert np.array_equal(svb.refine.census(img, W, H, *win), ref)


def test_census_identical_images_zero_hamming(svb, small):
    # the reference's own check (test_stereonet.py:492-495)
    g, W, H, L, R = small
    c = svb.refine.census(L, W, H, 4, 3)
    assert all(bin(int(a) ^ int(a)).count("1") == 0 for a in c)


# --------------------------------------------------------- costs and paths
def test_band_costs_golden(svb, small):
    g, W, H, L, R = small
    C = svb.refine.band_costs(g["census_l_4x3"], g["census_r_4x3"], L, R, g["base"], W, H, 10,
                              0.0, 20.0, 66.0, g["disp0"], 0.0, 4.0)
    assert np.array_equal(C, g["costs_R10"].astype(np.float64))


@pytest.mark.parametrize("i", range(8))
def test_aggregate_path_golden(svb, small, i):
    g, W, H, L, R = small
    dx, dy = DIRS[i]
    S = np.zeros(W * H * 21)
    svb.refine._aggregate_path(g["costs_R10"].astype(np.float64), g["base"], W, H, 21, 12.0,
                               150.0, dx, dy, S)
    assert np.array_equal(S, g["path%d_R10" % i].astype(np.float64))


def test_aggregate_all_paths_sum_golden(svb, small):
    g, W, H, L, R = small
    S = [0.0] * (W * H * 21)
    for dx, dy in DIRS:
        svb.refine._aggregate_path(list(g["costs_R10"].astype(np.float64)), list(g["base"]),
                                   W, H, 21, 12.0, 150.0, dx, dy, S)
    assert np.array_equal(np.array(S), g["S_R10"].astype(np.float64))


# ----------------------------------------------------------- refine_fullres
def test_refine_fullres_golden(svb, small):
    g, W, H, L, R = small
    d0 = g["disp0"]
    out, conf = svb.refine.refine_fullres(L, R, d0, W, H, return_conf=True, **PIPE)
    assert np.array_equal(bits(out), bits(g["refine_R10"]))
    assert np.array_equal(bits(conf), bits(g["conf_R10"]))
    assert np.array_equal(bits(svb.refine.refine_fullres(L, R, d0, W, H)), bits(g["refine_default"]))
    assert np.array_equal(bits(svb.refine.refine_fullres(L, R, d0, W, H, R=4, P1=12.0, P2=150.0,
                                                         paths=4, rx=4, ry=3)),
                          bits(g["refine_R4_paths4"]))
    assert np.array_equal(bits(svb.refine.refine_fullres(L, R, d0, W, H, R=6, P1=8.0, P2=96.0,
                                                         rx=3, ry=3, uniq=0.15)),
                          bits(g["refine_uniq"]))
    Rf = int(g["fullrange_R"][0])
    out = svb.refine.refine_fullres(L, R, np.full(W * H, float(Rf)), W, H, R=Rf, P1=12.0,
                                    P2=150.0, rx=4, ry=3)
    assert np.array_equal(bits(out), bits(g["fullrange"]))


def test_refine_fullres_list_io(svb, small):
    g, W, H, L, R = small
    out = svb.refine.refine_fullres(list(L), list(R), list(g["disp0"]), W, H, **PIPE)
    assert isinstance(out, list)
    assert np.array_equal(bits(out), bits(g["refine_R10"]))


@pytest.mark.parametrize("case", [
    dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3),            # pipeline: K=21, uint8 path costs
    dict(R=10, P1=12.0, P2=400.0, rx=4, ry=3),            # uint16 path costs
    dict(R=3, P1=1.0, P2=12.0, rx=2, ry=2),               # refine_fullres defaults
    dict(R=20, P1=10.0, P2=120.0, rx=4, ry=3),            # K=41: two band values per lane
    dict(R=50, P1=12.0, P2=150.0, rx=4, ry=3, paths=4),   # K=101: four per lane
    dict(R=100, P1=12.0, P2=150.0, rx=3, ry=2),           # K=201: eight per lane
    dict(R=0, P1=5.0, P2=9.0, rx=1, ry=1),                # K=1: every winner is an edge
    dict(R=6, P1=0.0, P2=0.0, rx=4, ry=3, uniq=0.05),     # zero penalties, uniqueness test
])
def test_refine_fullres_vs_oracle(svb, orc, case):
    pair = svb.synth.make_pair(77, 97, 61, 2.0, 40.0, n_planes=(2, 4))
    W, H = pair.W, pair.H
    d0 = noisy_disp(pair, 5)
    d0[: W * 3] += 60.0          # a band far off, and jumps between rows
    ref = orc.refine_fullres(pair.gray("left").ravel(), pair.gray("right").ravel(), d0, W, H,
                             **case)
    got = svb.refine.refine_fullres(pair.left, pair.right, d0, W, H, **case)
    assert np.array_equal(bits(got), bits(ref))


def test_fullrange_mode_vs_oracle(svb, orc):
    # eval_real.py:143-146: disp0 == R everywhere, band 0..2R
    pair = svb.synth.make_pair(78, 160, 120, 2.0, 60.0, n_planes=(3, 5))
    W, H = pair.W, pair.H
    Rf = int(np.max(pair.disp) + 2) // 2 + 1
    d0 = np.full(W * H, float(Rf))
    kw = dict(R=Rf, P1=12.0, P2=150.0, rx=4, ry=3)
    ref = orc.refine_fullres(pair.gray("left").ravel(), pair.gray("right").ravel(), d0, W, H, **kw)
    got = svb.refine.refine_fullres(pair.left, pair.right, d0, W, H, **kw)
    assert np.array_equal(bits(got), bits(ref))


# --------------------------------------------------------- left_to_right
def test_left_to_right_golden(svb, small):
    g, W, H, L, R = small
    assert np.array_equal(bits(svb.refine.left_to_right(g["disp0"], W, H)), bits(g["l2r"]))


@pytest.mark.parametrize("W,H", [(1, 1), (7, 3), (300, 5), (2049, 2)])
def test_left_to_right_vs_oracle(svb, orc, W, H):
    rng = np.random.default_rng(W + H)
    d = rng.uniform(-3.0, min(40.0, W), W * H)
    d[::5] = -0.0
    d[1::5] = 0.0
    d[2::9] = np.round(d[2::9])                 # many ties
    d[3::11] = 1e8 + 5.0                        # above the 1e8 fill threshold
    assert np.array_equal(bits(svb.refine.left_to_right(d, W, H)),
                          bits(orc.left_to_right(d, W, H)))


# -------------------------------------------------------------- lr_refine
def test_lr_refine_golden(svb, small):
    g, W, H, L, R = small
    out, st = svb.refine.lr_refine(L, R, g["disp0"], W, H, tol=2.0, **PIPE)
    assert np.array_equal(bits(out), bits(g["lr_out"]))
    assert np.array_equal(st.astype(np.int8), g["lr_status"])
    out, st = svb.refine.lr_refine(list(L), list(R), list(g["disp0"]), W, H)
    assert isinstance(st, list)
    assert np.array_equal(bits(out), bits(g["lr_default_out"]))
    assert np.array_equal(np.array(st, dtype=np.int8), g["lr_default_status"])


def test_lr_refine_config_small_golden(svb):
    g = golden("config_small.npz")
    H, W = g["left"].shape
    out, st = svb.refine.lr_refine(g["left"], g["right"], g["disp0"], W, H, tol=2.0, **PIPE)
    assert np.array_equal(bits(out), bits(g["out"]))
    assert np.array_equal(st.astype(np.int8), g["status"])


def test_lr_refine_config_full_vs_oracle(svb, orc, net, golden_meta):
    """450x375: the oracle's network disparity (pinned by digest) refined on
    the GPU must hash to the reference's own lr_refine output."""
    import hashlib
    p = svb.synth.config_full()
    L, R = p.gray("left").ravel(), p.gray("right").ravel()
    df, _, _, _ = orc.predict_auto(net, L, R, p.W, p.H)
    m = golden_meta["config_full"]
    assert hashlib.sha256(df.tobytes()).hexdigest() == m["disp0_sha256"]
    out, st = svb.refine.lr_refine(p.left, p.right, df, p.W, p.H, tol=2.0, **PIPE)
    assert hashlib.sha256(np.ascontiguousarray(out).tobytes()).hexdigest() == m["out_sha256"]
    assert hashlib.sha256(st.astype(np.int8).tobytes()).hexdigest() == m["status_sha256"]


@pytest.mark.parametrize("W,H,seed", [(333, 201, 1), (41, 300, 2), (1000, 31, 3)])
def test_lr_refine_vs_oracle_odd_shapes(svb, orc, W, H, seed):
    pair = svb.synth.make_pair(seed, W, H, 1.0, min(60.0, W / 3), n_planes=(2, 5))
    d0 = noisy_disp(pair, seed)
    ref_out, ref_st = orc.lr_refine(pair.gray("left").ravel(), pair.gray("right").ravel(), d0, W,
                                    H, tol=2.0, **PIPE)
    out, st = svb.refine.lr_refine(pair.left, pair.right, d0, W, H, tol=2.0, **PIPE)
    assert np.array_equal(bits(out), bits(ref_out))
    assert np.array_equal(st.astype(np.int32), ref_st)


def test_lr_refine_deterministic(svb):
    pair = svb.synth.make_pair(9, 200, 150, 2.0, 40.0)
    d0 = noisy_disp(pair, 9)
    a = svb.refine.lr_refine(pair.left, pair.right, d0, 200, 150, tol=2.0, **PIPE)
    b = svb.refine.lr_refine(pair.left, pair.right, d0, 200, 150, tol=2.0, **PIPE)
    assert np.array_equal(bits(a[0]), bits(b[0])) and np.array_equal(a[1], b[1])


# ------------------------------------------------ the reference's properties
def test_band_sgm_halves_error(svb):
    # test_stereonet.py:497-514, on this package's generator
    pair = svb.synth.make_pair(5, 96, 64, 2.0, 12.0, n_planes=(3, 3))
    W, H = pair.W, pair.H
    gt = pair.disp.ravel()
    d0 = gt + np.random.default_rng(9).uniform(-2.0, 2.0, W * H)
    mask = (np.arange(W * H) % W >= 14) & pair.valid.ravel()
    e0 = np.mean(np.abs(d0 - gt)[mask])
    d1 = svb.refine.refine_fullres(pair.left, pair.right, d0, W, H, R=4, P1=12.0, P2=150.0)
    e1 = np.mean(np.abs(d1 - gt)[mask])
    assert e1 < 0.5 * e0


def test_lr_marks_left_margin_occluded(svb):
    # test_stereonet.py:515-517
    pair = svb.synth.make_pair(5, 96, 64, 2.0, 12.0, n_planes=(3, 3))
    W, H = pair.W, pair.H
    gt = pair.disp.ravel()
    d0 = gt + np.random.default_rng(9).uniform(-2.0, 2.0, W * H)
    _, st = svb.refine.lr_refine(pair.left, pair.right, d0, W, H, tol=2.0, R=4, P1=12.0, P2=150.0)
    assert all(st[y * W] == 1 for y in range(H) if gt[y * W] >= 1.5)


# ------------------------------------------------------------------ errors
def test_nan_disparity_raises(svb):
    W, H = 32, 16
    img = np.zeros(W * H, dtype=np.uint8)
    d = np.ones(W * H)
    d[5] = np.nan
    with pytest.raises(ValueError):
        svb.refine.refine_fullres(img, img, d, W, H)
    with pytest.raises(ValueError):
        svb.refine.lr_refine(img, img, d, W, H)


def test_out_of_range_disparity_flagged_on_device(svb):
    W, H = 32, 16
    img = np.zeros(W * H, dtype=np.uint8)
    d = np.ones(W * H)
    d[7] = 3.0e9                      # finite, but beyond the int32 band centre
    with pytest.raises(ValueError, match="disparity"):
        svb.refine.lr_refine(img, img, d, W, H)


@pytest.mark.parametrize("kw", [dict(ad_weight=1.0), dict(prior_w=0.5), dict(P1=1.5),
                                dict(P2=-1.0), dict(R=127), dict(rx=5, ry=5)])
def test_unsupported_params_raise(svb, kw):
    W, H = 32, 16
    img = np.zeros(W * H, dtype=np.uint8)
    with pytest.raises(ValueError):
        svb.refine.refine_fullres(img, img, np.ones(W * H), W, H, **kw)


def test_size_mismatch_raises(svb):
    with pytest.raises(ValueError):
        svb.refine.lr_refine(np.zeros(10, np.uint8), np.zeros(10, np.uint8), np.ones(10), 4, 4)
