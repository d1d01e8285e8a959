"""The claim predict_auto's width decisions rest on, checked on the CPU in
numpy (the same FP64 operations as the host and the kernels): the width the
rule of predict_auto (stereonet.py:3915-3919) gives the 95% quantile of a map
(_peak, stereonet.py:3866-3869) equals the width read off a histogram of the
widths the rule gives every value of the map, because the rule is monotone
non-increasing in the value.  The GPU implementation of the histogram side
is tested against the same reference in tests/test_width_gpu.py."""

import math

import numpy as np
import pytest


def width_of(v, W, target, max_width, scale):
    """The rule per value, vectorised; NaN counts as the largest value."""
    v = np.asarray(v, dtype=np.float64)
    pk = np.where(v > 0.5, v, 0.5) * scale
    m = np.where(pk > 1.0e-6, pk, 1.0e-6)
    q = W * target / m + 0.5
    w = np.where(q < 2147483647.0, np.trunc(np.minimum(q, 2147483647.0)), 2147483647.0)
    w = np.minimum(np.minimum(w, W), max_width)
    w = np.maximum(w, 48).astype(np.int64)
    return np.where(np.isnan(v), 48, w)


def width_by_quantile(vals, W, target, max_width, scale):
    v = float(np.sort(vals, kind="stable")[int(len(vals) * 0.95)])
    return int(width_of([v], W, target, max_width, scale)[0])


def width_by_histogram(vals, W, target, max_width, scale):
    kmax = max(min(W, max_width), 48)
    m = kmax - 48
    bins = kmax - width_of(vals, W, target, max_width, scale)      # 0 .. m
    hist = np.bincount(bins, minlength=m + 1)
    c = np.cumsum(hist[:m])                                        # C_j, j < m
    rank = int(len(vals) * 0.95)
    return kmax - int(np.count_nonzero(c <= rank))


CASES = [(450, 25.0, 320, 1.0), (450, 25.0, 320, 450 / 64.0), (640, 40.0, 320, 1.0),
         (97, 30.0, 320, 1.0), (1400, 18.5, 560, 1.0), (30, 25.0, 320, 1.0)]


@pytest.mark.parametrize("W,target,max_width,scale", CASES)
def test_histogram_equals_quantile_on_random_maps(W, target, max_width, scale):
    rng = np.random.default_rng(W)
    for n in (7, 1000, 20000):
        for hi in (3.0, 40.0, 300.0, 1.0e7):
            vals = rng.uniform(-5.0, hi, n)
            vals[rng.random(n) < 0.1] = rng.choice([0.0, -0.0, 0.5, 0.25])
            assert width_by_histogram(vals, W, target, max_width, scale) == \
                width_by_quantile(vals, W, target, max_width, scale)


@pytest.mark.parametrize("W,target,max_width,scale", CASES)
def test_histogram_equals_quantile_at_width_boundaries(W, target, max_width, scale):
    rng = np.random.default_rng(3)
    kmax = max(min(W, max_width), 48)
    n = 2000
    r = int(n * 0.95)
    for k in range(48, kmax):
        # the real boundary W * target / ((k + 0.5) * scale) and its
        # neighbours, one and two ULP away on each side
        x0 = W * target / ((k + 0.5) * scale)
        for x in (x0, np.nextafter(x0, -math.inf), np.nextafter(x0, math.inf),
                  np.nextafter(np.nextafter(x0, math.inf), math.inf)):
            vals = np.concatenate([x - rng.uniform(0.01, 5.0, r), [x] * 3,
                                   x + rng.uniform(0.01, 5.0, n - r - 3)])
            assert width_by_histogram(vals, W, target, max_width, scale) == \
                width_by_quantile(vals, W, target, max_width, scale), (k, x)


def test_rule_is_monotone():
    v = np.sort(np.concatenate([np.linspace(-1, 1000, 20001), [0.5, 1e-9, 1e300]]))
    for W, target, max_width, scale in CASES:
        w = width_of(v, W, target, max_width, scale)
        assert np.all(np.diff(w) <= 0)
