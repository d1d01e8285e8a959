"""Learned adaptive band on the GPU against its FP64 oracle.

* features, targets, band application, masked lr_refine: bit-exact (FP32
  features are the FP64 oracle values rounded once);
* band net forward and gradients (BF16 tensor-core operands, FP32
  accumulation): forward within 2% of the output range; every parameter
  block's gradient at cosine >= 0.999 and relative L2 error <= 3% of the
  FP64 oracle's (the reference-style central-difference check pins the
  oracle, tests/test_band_oracle.py);
* Adam: the GPU step equals the oracle's Adam.step applied to the same
  gradients within FP32 rounding;
* a short training run lowers the loss.
"""

import numpy as np
import pytest
import torch

from conftest import bits

pytestmark = pytest.mark.gpu

KW = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)


def _pair(svb, W, H, seed, dmax=60.0):
    p = svb.synth.make_pair(seed, W, H, 2.0, dmax, bars=2)
    d0 = p.disp.ravel() + np.random.default_rng(seed).normal(0, 4, W * H)
    return p, d0


@pytest.mark.parametrize("W,H,dmax", [(64, 48, 40), (97, 33, 120), (20, 70, 255)])
def test_features_bit_exact(svb, orc, W, H, dmax):
    p, d0 = _pair(svb, W, H, W + H)
    d0[::37] = -3.7
    d0[5] = 400.0
    rng = np.random.default_rng(W)
    sp, pm = rng.uniform(0, 9, W * H), rng.uniform(0, 1, W * H)
    ref = orc.band_features(p.gray("left"), p.gray("right"), d0, W, H, dmax, sp,
                            pm).astype(np.float32)
    for L, R in ((p.left, p.right), (p.gray("left"), p.gray("right"))):
        got = svb.band.features(L, R, d0, W, H, dmax, sp, pm).cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def _batch(svb, orc, nb, W, H, seed):
    feats, tg, ms = [], [], []
    for i in range(nb):
        p, d0 = _pair(svb, W, H, seed + i)
        feats.append(orc.band_features(p.gray("left"), p.gray("right"), d0, W, H, 80))
        t, m = orc.band_targets(p.disp.ravel() + 0.3, np.zeros(W * H, np.int32), d0)
        m[::5] = 0
        tg.append(t)
        ms.append(m)
    f = np.concatenate(feats).astype(np.float32)
    return f, np.concatenate(tg).astype(np.float32), np.concatenate(ms)


def test_forward_and_grads_vs_oracle(svb, orc):
    nb, W, H = 2, 72, 40
    f, t, m = _batch(svb, orc, nb, W, H, 10)
    params = svb.band.init_params(3)
    params[-(16 * 2 * 9 + 2):] *= 10.0          # a last layer of ordinary size
    params32 = params.astype(np.float32).astype(np.float64)
    net = svb.band.BandNet(params32)
    out = net.forward(torch.from_numpy(f).cuda(), nb, W, H).cpu().numpy()
    ref = orc.band_forward(params32, f.astype(np.float64), nb, W, H)
    assert np.abs(out - ref).max() <= 0.02 * np.abs(ref).max()
    g, loss = net.grads(f, t, m, nb, W, H)
    g = g.cpu().numpy().astype(np.float64)
    rg, rloss = orc.band_grads(params32, f.astype(np.float64), t.astype(np.float64), m, nb, W, H)
    assert abs(loss.item() - rloss) <= 1e-2 * abs(rloss)
    off = 0
    for ic, oc, _d in svb.band.LAYERS:
        for n in (oc * ic * 9, oc):
            a, b = g[off:off + n], rg[off:off + n]
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
            rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30)
            assert cos >= 0.999 and rel <= 0.03, (off, n, cos, rel)
            off += n


def test_adam_step_matches_oracle(svb, orc):
    nb, W, H = 1, 48, 32
    f, t, m = _batch(svb, orc, nb, W, H, 20)
    params = svb.band.init_params(4).astype(np.float32).astype(np.float64)
    net = svb.band.BandNet(params)
    g, _ = net.grads(f, t, m, nb, W, H)
    g = g.cpu().numpy().astype(np.float64)
    ft, tt, mt = (torch.from_numpy(a).cuda() for a in (f, t, m))
    net.train_step(ft, tt, mt, nb, W, H, lr=5e-4)
    got = net.params()
    opt = orc.Adam(params, lr=5e-4)
    exp = opt.step(g)
    assert np.allclose(got, exp, rtol=0, atol=2e-6)


@pytest.mark.parametrize("W,H", [(64, 48), (33, 90)])
def test_apply_and_masked_refine_bit_exact(svb, orc, W, H):
    p, d0 = _pair(svb, W, H, 7 * W)
    rng = np.random.default_rng(W)
    out = np.concatenate([rng.normal(0, 0.5, W * H), rng.normal(0.5, 1.5, W * H)])
    out = out.astype(np.float32)
    c_ref, r_ref = orc.band_apply(out.astype(np.float64), d0, W, H, b_thr=3.0, rad_k=3.0,
                                  rad_min=3, R=10, shift_max=40.0)
    c, r = svb.band.apply(out, d0, W, H, b_thr=3.0, rad_k=3.0, rad_min=3, R=10, shift_max=40.0)
    assert np.array_equal(bits(c.cpu().numpy()), bits(c_ref))
    assert np.array_equal(r.cpu().numpy(), r_ref)
    o_ref, s_ref = orc.lr_refine_band(p.gray("left"), p.gray("right"), c_ref, r_ref, W, H,
                                      tol=2.0, **KW)
    o, s = svb.band.lr_refine_band(p.left, p.right, c_ref, r_ref, W, H, tol=2.0, **KW)
    assert np.array_equal(bits(o), bits(o_ref))
    assert np.array_equal(np.asarray(s), s_ref)
    # the full half-width everywhere is plain lr_refine
    o2, s2 = svb.band.lr_refine_band(p.left, p.right, d0, np.full(W * H, 10, np.uint8), W, H,
                                     tol=2.0, **KW)
    o3, s3 = svb.refine.lr_refine(p.left, p.right, d0, W, H, tol=2.0, **KW)
    assert np.array_equal(bits(o2), bits(o3)) and np.array_equal(np.asarray(s2), np.asarray(s3))


def test_targets_bit_exact(svb, orc):
    rng = np.random.default_rng(2)
    n = 5000
    label, d0 = rng.uniform(0, 200, n), rng.uniform(0, 200, n)
    st = rng.integers(0, 3, n)
    t_ref, m_ref = orc.band_targets(label, st, d0, shift_max=60.0)
    t, m = svb.band.targets(label, st.astype(np.uint8), d0, shift_max=60.0)
    assert np.array_equal(t.cpu().numpy(), t_ref.astype(np.float32))
    assert np.array_equal(m.cpu().numpy(), m_ref)


def test_training_lowers_loss(svb, orc):
    nb, W, H = 4, 64, 48
    f, _, m = _batch(svb, orc, nb, W, H, 30)
    # a learnable target: the wide-search shift the features carry
    t = np.clip(64.0 * f.reshape(nb, 8, -1)[:, 1], -160, 160).astype(np.float32).ravel()
    net = svb.band.BandNet(seed=1)
    ft, tt, mt = (torch.from_numpy(a).cuda() for a in (f, t, m))
    _, l0 = net.grads(f, t, m, nb, W, H)
    l0 = l0.item()
    for _ in range(60):
        net.train_step(ft, tt, mt, nb, W, H, lr=2e-3)
    _, l1 = net.grads(f, t, m, nb, W, H)
    assert l1.item() < 0.8 * l0, (l0, l1.item())


def test_rule_centre_vs_oracle(svb, orc):
    W, H = 64, 48
    p, d0 = _pair(svb, W, H, 77)
    f = orc.band_features(p.gray("left"), p.gray("right"), d0, W, H, 80)
    for tau in (0.1, 0.3, 1.1):
        got = svb.band.rule_centre(f.astype(np.float32), d0, W, H, tau).cpu().numpy()
        ref = orc.band_rule_centre(f, d0, W, H, tau)
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
