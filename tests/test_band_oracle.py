"""The learned band's FP64 oracle (CPU): gradients against central
differences (the reference's own gradient-check method, test_stereonet.py:
99-215), Adam against a transcription of stereonet.py:1368-1387, the masked
lr_refine against the plain lr_refine restatement, features against numpy."""

import numpy as np
import pytest


def _case(orc, nb=2, W=9, H=7, seed=0):
    rng = np.random.default_rng(seed)
    n = orc.band_param_count()
    params = rng.normal(0, 0.3, n)
    feat = rng.normal(0, 1, nb * 8 * W * H)
    target = rng.normal(0, 20, nb * W * H)
    mask = (rng.random(nb * W * H) < 0.8).astype(np.uint8)
    return params, feat, target, mask


def test_param_count(orc):
    assert orc.band_param_count() == 6098 <= 20000


def test_band_gradients_central_differences(orc):
    nb, W, H = 2, 9, 7
    params, feat, target, mask = _case(orc, nb, W, H)
    g, loss = orc.band_grads(params, feat, target, mask, nb, W, H)
    out = orc.band_forward(params, feat, nb, W, H)
    assert abs(orc.band_loss(out, target, mask, nb, W, H) - loss) < 1e-12
    rng = np.random.default_rng(5)
    idx = rng.choice(params.size, 60, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = params.copy(), params.copy()
        pp[i] += h
        pm[i] -= h
        lp = orc.band_loss(orc.band_forward(pp, feat, nb, W, H), target, mask, nb, W, H)
        lm = orc.band_loss(orc.band_forward(pm, feat, nb, W, H), target, mask, nb, W, H)
        num = (lp - lm) / (2 * h)
        assert abs(num - g[i]) <= 1e-5 * max(1.0, abs(num)), (i, num, g[i])


def test_adam_matches_reference_semantics(orc):
    rng = np.random.default_rng(1)
    p0 = rng.normal(0, 1, 50)
    opt = orc.Adam(p0, lr=5e-4)
    p, m, v = p0.copy(), np.zeros(50), np.zeros(50)
    b1t = b2t = 1.0
    for step in range(5):
        g = rng.normal(0, 4, 50)
        got = opt.step(g)
        b1t *= 0.9
        b2t *= 0.999
        c1, c2 = 1.0 / (1.0 - b1t), 1.0 / (1.0 - b2t)
        gc = np.clip(g, -5.0, 5.0)
        m = 0.9 * m + (1.0 - 0.9) * gc
        v = 0.999 * v + (1.0 - 0.999) * gc * gc
        p = p - 5e-4 * (m * c1) / (np.sqrt(v * c2) + 1e-8)
        assert np.allclose(got, p, rtol=0, atol=1e-15)


@pytest.mark.parametrize("W,H", [(40, 24), (23, 17)])
def test_masked_lr_refine_full_band_equals_lr_refine(svb, orc, W, H):
    pair = svb.synth.make_pair(W * H, W, H, 1.0, 12.0)
    L, R = pair.gray("left").ravel(), pair.gray("right").ravel()
    d0 = pair.disp.ravel() + np.random.default_rng(W).uniform(-3, 3, W * H)
    kw = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    ref = orc.lr_refine(L, R, d0, W, H, tol=2.0, **kw)
    a = orc.lr_refine_band(L, R, d0, None, W, H, tol=2.0, **kw)
    b = orc.lr_refine_band(L, R, d0, np.full(W * H, 10, np.uint8), W, H, tol=2.0, **kw)
    for got in (a, b):
        assert np.array_equal(got[0].view(np.uint64), np.asarray(ref[0]).view(np.uint64))
        assert np.array_equal(got[1], np.asarray(ref[1]))


def test_band_features_numpy(orc):
    W, H, dmax = 21, 13, 9
    rng = np.random.default_rng(3)
    L = rng.integers(0, 256, (H, W)).astype(np.float64) / 255.0
    R = rng.integers(0, 256, (H, W)).astype(np.float64) / 255.0
    d0 = rng.uniform(-2, 12, W * H)
    f = orc.band_features(L, R, d0, W, H, dmax).reshape(8, H, W)
    cl = orc.census(L, W, H, 4, 3).reshape(H, W)
    cr = orc.census(R, W, H, 4, 3).reshape(H, W)
    pop = np.vectorize(lambda v: bin(int(v)).count("1"))
    for y, x in [(0, 0), (6, 10), (12, 20), (3, 4), (9, 15)]:
        agg = []
        for d in range(dmax + 1):
            s = 0
            for dy in range(-4, 5):
                yy = min(max(y + dy, 0), H - 1)
                s += int(pop(cl[yy, x] ^ cr[yy, x - d])) if x - d >= 0 else 66
            agg.append(s)
        agg = np.array(agg)
        dd = d0[y * W + x]
        r = min(max(0, int(dd + 0.5)), dmax)
        dw = int(np.argmin(agg))
        lo, hi = max(0, r - 10), min(dmax, r + 10)
        exp = [dd / 64, (dw - dd) / 64, agg[dw] / 558, agg[r] / 558, agg[lo:hi + 1].min() / 558,
               L[y, x] - 0.5]
        assert np.allclose(f[:6, y, x], exp, rtol=0, atol=1e-15), (y, x)
    assert not f[6:].any()                       # no network confidence given: zero planes
    sp, pm = rng.uniform(0, 9, W * H), rng.uniform(0, 1, W * H)
    g = orc.band_features(L, R, d0, W, H, dmax, sp, pm).reshape(8, H, W)
    assert np.array_equal(g[:6], f[:6])
    assert np.array_equal(g[6].ravel(), (sp / 16).astype(np.float32).astype(np.float64))
    assert np.array_equal(g[7].ravel(), (pm - 0.5).astype(np.float32).astype(np.float64))
