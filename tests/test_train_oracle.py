"""The FP64 training oracle (oracle/sv_train_oracle.c) against the
reference's own train_grads and Adam.step (stereonet.py:1619-1653,
1368-1387), run on seeded 48x32 crops with its checkpoint
(tests/golden/training.npz): loss, every gradient, the prediction and two
optimiser steps, bit for bit."""

import numpy as np

from conftest import bits, golden


def test_train_grads_and_adam_bit_exact(orc, net):
    g = golden("training.npz")
    assert np.array_equal(bits(g["params0"]), bits(net.flat))
    opt = orc.AdamState(g["params0"], lr=1.0e-3)
    for k in range(2):
        L = g["s%d_left" % k].astype(np.float64) / 255.0
        R = g["s%d_right" % k].astype(np.float64) / 255.0
        H, W = L.shape
        loss, grads, d2 = orc.train_grads(net, L, R, g["s%d_disp" % k], g["s%d_valid" % k], W, H,
                                          params=opt.p)
        assert loss == g["s%d_loss" % k][0]
        assert np.array_equal(bits(grads), bits(g["s%d_grads" % k]))
        assert np.array_equal(bits(d2), bits(g["s%d_d2" % k]))
        opt.step(grads)
        assert np.array_equal(bits(opt.p), bits(g["s%d_params_after" % k]))


def test_gradient_matches_central_differences(orc, net):
    """The reference's own check method (test_stereonet.py:99-215): a few
    parameters of every layer group against central differences of the
    loss."""
    g = golden("training.npz")
    L = g["s0_left"].astype(np.float64) / 255.0
    R = g["s0_right"].astype(np.float64) / 255.0
    H, W = L.shape
    p0 = g["params0"].copy()
    _, grads, _ = orc.train_grads(net, L, R, g["s0_disp"], g["s0_valid"], W, H, params=p0)
    rng = np.random.default_rng(5)
    idx = np.unique(np.concatenate([rng.choice(p0.size, 12, replace=False),
                                    np.argsort(-np.abs(grads))[:6]]))
    eps = 1e-6
    for i in idx:
        pp, pm = p0.copy(), p0.copy()
        pp[i] += eps
        pm[i] -= eps
        lp = orc.train_grads(net, L, R, g["s0_disp"], g["s0_valid"], W, H, params=pp)[0]
        lm = orc.train_grads(net, L, R, g["s0_disp"], g["s0_valid"], W, H, params=pm)[0]
        num = (lp - lm) / (2 * eps)
        assert abs(num - grads[i]) <= 1e-4 * max(1.0, abs(grads[i])), (i, num, grads[i])
