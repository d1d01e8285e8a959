"""The learned band's host-side harness: the full-range label radius and
the EPE / bad2 score."""

import math

import numpy as np
import pytest


@pytest.fixture(scope="module")
def bt(svb):
    from importlib import import_module
    return import_module(svb.__name__ + ".band_train")


def test_full_range_radius_covers_the_largest_disparity(bt):
    assert bt.full_range_R(np.zeros(4)) == 2
    assert bt.full_range_R(np.array([3.0, 79.2])) == 42        # (80 + 2) // 2 + 1
    rng = np.random.default_rng(5)
    for m in rng.uniform(0, 200, 50):
        R = bt.full_range_R(np.array([0.0, m]))
        assert 2 * R >= math.ceil(m) + 2                      # band [0, 2R] holds ceil(max)
        assert R == (math.ceil(m) + 2) // 2 + 1


def test_score_is_epe_and_bad2_over_valid_pixels(bt):
    gt = np.array([[0.0, 1.0], [2.0, 3.0]])
    d = [0.5, 4.0, 2.0, 100.0]
    valid = np.array([[True, True], [True, False]])
    epe, bad2 = bt._score(d, gt, valid)
    assert epe == pytest.approx((0.5 + 3.0 + 0.0) / 3)
    assert bad2 == pytest.approx(1 / 3)
