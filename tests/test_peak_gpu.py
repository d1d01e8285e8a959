"""_peak (stereonet.py:3866-3869) on the GPU: the exact radix select against
the reference's own value (tests/golden/primitives.npz) and against sorted()
on arrays with ties, signed zeros and negatives, from one element to
307,200."""

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def ref_peak(d, q=0.95):
    s = sorted(d.tolist())
    v = s[int(len(s) * q)]
    return v if v > 0.5 else 0.5


def test_peak_reference_fixture(svb):
    g = golden("primitives.npz")
    assert svb.network._peak(g["peak_in"]) == g["peak"][0]


@pytest.mark.parametrize("n", [1, 2, 7, 1001, 4096, 168750, 204800, 204801, 307200])
def test_peak_matches_sorted(svb, n):
    rng = np.random.default_rng(n)
    d = rng.uniform(-3.0, 80.0, n)
    k = n // 5
    d[rng.choice(n, size=k, replace=False)] = np.round(d[:k], 1)
    if n > 10:
        d[::11] = -0.0
        d[5::13] = 0.0
        d[7::17] = 41.25
    for q in (0.95, 0.5, 0.999, 0.0):
        assert svb.network._peak(d, q) == ref_peak(d, q), (n, q)


def test_peak_rejects_bad_q(svb):
    with pytest.raises(ValueError):
        svb.network._peak(np.ones(10), 1.0)


@pytest.mark.parametrize("plateau", [0, 3000, 5000, 40000])
def test_peak_with_plateau_at_the_quantile(svb, plateau):
    """Many equal values at the 95% quantile: up to 4096 matches after the
    second pass finish in one CTA, more take the remaining passes."""
    rng = np.random.default_rng(plateau + 1)
    n = 168750
    d = rng.uniform(0.0, 80.0, n)
    if plateau:
        d[rng.choice(n, size=plateau, replace=False)] = 60.0 + 1.0 / 3.0
    for q in (0.95, 0.9):
        assert svb.network._peak(d, q) == ref_peak(d, q), (plateau, q)
