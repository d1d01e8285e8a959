"""predict_auto's work-width decision (network.work_width, sv_work_width)
against the reference's own arithmetic: _peak's sorted(disp)[int(n * q)]
floored at 0.5 (stereonet.py:3866-3869) fed to the width rule
int(W * target / max(peak, 1e-6) + 0.5), clamped to [48, min(W, max_width)]
(stereonet.py:3915-3919).  The GPU never selects the quantile: it histograms
the width each value would give and reads the width at the quantile's
position, so the maps here put the quantile exactly on, and one ULP either
side of, the values where the width changes.
"""

import math
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def width_ref(vals, W, target, max_width, scale):
    v = float(np.sort(np.asarray(vals, dtype=np.float64), kind="stable")[int(len(vals) * 0.95)])
    pk = v if v > 0.5 else 0.5
    peak = pk * scale
    m = peak if peak > 1.0e-6 else 1.0e-6
    w = int(W * target / m + 0.5)
    return max(min(w, W, max_width), 48)


def _bits(x):
    return struct.unpack("<q", struct.pack("<d", x))[0]


def _float(b):
    return struct.unpack("<d", struct.pack("<q", b))[0]


def threshold(k, W, target, max_width, scale):
    """Smallest positive double v with width(v) <= k (bisection over the
    bit patterns of positive doubles, which sort as the values do)."""
    lo, hi = _bits(0.5), _bits(math.inf)
    one = lambda b: width_ref([_float(b)], W, target, max_width, scale) <= k
    if one(lo):
        return 0.5
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if one(mid):
            hi = mid
        else:
            lo = mid
    return _float(hi)


def quantile_map(rng, n, x):
    """n values whose sorted position int(0.95 n) holds x: values below x
    before it, x repeated a few times, values above after."""
    r = int(n * 0.95)
    below = x - rng.uniform(0.001, 20.0, r)
    reps = min(5, n - r)
    above = x + rng.uniform(0.0, 30.0, n - r - reps)
    above[above <= x] = np.nextafter(x, math.inf)
    out = np.concatenate([below, np.full(reps, x), above])
    rng.shuffle(out)
    return out


CASES = [  # W, target, max_width, scale
    (450, 25.0, 320, 1.0),
    (450, 25.0, 320, 450 / 64.0),
    (640, 40.0, 320, 1.0),
    (97, 30.0, 320, 1.0),
    (1400, 18.5, 560, 1.0),
]


@pytest.mark.parametrize("W,target,max_width,scale", CASES)
@pytest.mark.parametrize("n", [3392, 168750])
def test_random_maps(svb, W, target, max_width, scale, n):
    rng = np.random.default_rng(n + W)
    for trial in range(4):
        vals = rng.uniform(-2.0, 120.0 * (trial + 1), n)
        vals[rng.random(n) < 0.05] = -0.0
        got = svb.network.work_width(vals, W, target, max_width, scale)
        assert got == width_ref(vals, W, target, max_width, scale), (trial, got)


@pytest.mark.parametrize("W,target,max_width,scale", CASES)
def test_quantile_on_width_boundaries(svb, W, target, max_width, scale):
    rng = np.random.default_rng(7)
    kmax = max(min(W, max_width), 48)
    ks = sorted({48, 49, 50, (48 + kmax) // 2, kmax - 2, kmax - 1} & set(range(48, kmax)))
    for k in ks:
        t = threshold(k, W, target, max_width, scale)
        for x in (t, np.nextafter(t, -math.inf), np.nextafter(t, math.inf)):
            for n in (1000, 40000):
                vals = quantile_map(rng, n, x)
                want = width_ref(vals, W, target, max_width, scale)
                got = svb.network.work_width(vals, W, target, max_width, scale)
                assert got == want, (k, x, n, got, want)


def test_plateaus_and_tiny_maps(svb):
    for vals in (np.full(50000, 33.25), np.full(7, 0.25), np.array([5.0]),
                 np.concatenate([np.full(900, 10.0), np.full(100, 80.0)]),
                 -np.arange(20000, dtype=np.float64)):
        for W, target, max_width, scale in CASES:
            assert svb.network.work_width(vals, W, target, max_width, scale) == \
                width_ref(vals, W, target, max_width, scale)


def test_too_many_widths_rejected(svb):
    with pytest.raises(Exception):
        svb.network.work_width(np.ones(10), 5000, 25.0, 4000, 1.0)
