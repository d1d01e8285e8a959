"""StereoNet training on the GPU (csrc/sv_train.cu) against the FP64 oracle,
which is itself the reference's train_grads / Adam.step bit for bit
(tests/test_train_oracle.py).

Tolerances (FP32 activations and gradients, FP64 weight-gradient sums):
per parameter block, max |g_gpu - g_ref| <= 2e-3 * max |g_ref| + 1e-6 * (the
largest gradient of any block), and
cosine similarity >= 0.9999 over the whole gradient; losses within 1e-4
relative.  Adam itself runs in FP64 and matches to 1e-12 relative."""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

GRAD_REL = 2e-3
COS_MIN = 0.9999
LOSS_REL = 1e-4


@pytest.fixture(scope="module")
def train(svb):
    from importlib import import_module
    return import_module(svb.__name__ + ".train")


def _blocks(net, flat):
    out, k = [], 0
    for n in net.arch.block_sizes():
        out.append(flat[k:k + n])
        k += n
    return out


def assert_grads_close(net, got, ref):
    # the floor (relative to the whole gradient) covers blocks whose exact
    # gradient is zero, such as the last cost-filter bias: soft-argmin's and
    # the cross-entropy's cost gradients each sum to zero over disparities
    floor = 1e-6 * np.abs(ref).max()
    for i, (g, r) in enumerate(zip(_blocks(net, got), _blocks(net, ref))):
        tol = GRAD_REL * np.abs(r).max() + floor
        assert np.abs(g - r).max() <= tol, (i, np.abs(g - r).max(), tol)
    cos = float(np.dot(got, ref) / (np.linalg.norm(got) * np.linalg.norm(ref)))
    assert cos >= COS_MIN, cos


def _crop(svb, seed, W=96, H=64, dmax=36.0):
    p = svb.synth.make_pair(seed, W, H, 2.0, dmax, n_planes=(2, 4), lowtex_frac=0.2)
    return (p.gray("left"), p.gray("right"), p.disp, p.valid)


def test_train_grads_match_reference_fixtures(svb, net, train):
    """B = 1 on the reference's own fixture crops (48x32)."""
    g = golden("training.npz")
    t = train.Trainer(net)
    params = g["params0"]
    opt_p = None
    for k in range(2):
        if opt_p is not None:
            t.set_params(opt_p)
        L = g["s%d_left" % k].astype(np.float64) / 255.0
        R = g["s%d_right" % k].astype(np.float64) / 255.0
        loss, pred = t.compute_grads(L, R, g["s%d_disp" % k], g["s%d_valid" % k], pred=True)
        assert abs(float(loss[0]) - g["s%d_loss" % k][0]) <= LOSS_REL * g["s%d_loss" % k][0]
        assert_grads_close(net, t.grads(), g["s%d_grads" % k])
        assert np.abs(pred[0].cpu().numpy().ravel() - g["s%d_d2" % k]).max() < 1e-3
        opt_p = g["s%d_params_after" % k]
    del params


def test_batch_gradient_is_mean_of_samples(svb, orc, net, train):
    """B = 4 crops of 96x64 (disparities up to 36 px, occlusions, low
    texture): the batch gradient is the mean of the oracle's per-sample
    gradients, and each sample's loss matches."""
    crops = [_crop(svb, 7100 + k) for k in range(4)]
    L, R, D, V = (np.stack([c[j] for c in crops]) for j in range(4))
    t = train.Trainer(net)
    loss = t.compute_grads(L, R, D, V).cpu().numpy()
    ref = []
    for k in range(4):
        lo, gr, _ = orc.train_grads(net, L[k], R[k], D[k], V[k], 96, 64)
        assert abs(loss[k] - lo) <= LOSS_REL * abs(lo), (k, loss[k], lo)
        ref.append(gr)
    assert_grads_close(net, t.grads(), np.mean(ref, axis=0))


def test_adam_step_matches_reference(svb, orc, net, train):
    g = golden("training.npz")
    t = train.Trainer(net)
    opt = orc.AdamState(g["params0"], lr=1.0e-3)
    for k in range(2):
        gr = g["s%d_grads" % k]
        t.lib.sv_trainer_set_grads(t.handle, gr.ctypes.data_as(__import__("ctypes").c_void_p),
                                   gr.size)
        t.adam(lr=1.0e-3)
        opt.step(gr)
        got = t.params()
        assert np.allclose(got, opt.p, rtol=1e-12, atol=1e-15)
        assert np.allclose(got, g["s%d_params_after" % k], rtol=1e-12, atol=1e-15)


def test_deterministic(svb, net, train):
    crops = [_crop(svb, 7200 + k) for k in range(3)]
    L, R, D, V = (np.stack([c[j] for c in crops]) for j in range(4))
    t = train.Trainer(net)
    a = t.compute_grads(L, R, D, V).cpu().numpy()
    ga = t.grads()
    b = t.compute_grads(L, R, D, V).cpu().numpy()
    assert np.array_equal(a, b) and np.array_equal(ga, t.grads())


def test_steps_track_the_oracle_and_reduce_the_loss(svb, orc, net, train):
    """Three Adam steps on a batch of 2: the GPU parameters follow the
    oracle's trajectory; 100 more steps fit the batch."""
    crops = [_crop(svb, 7300 + k) for k in range(2)]
    L, R, D, V = (np.stack([c[j] for c in crops]) for j in range(4))
    t = train.Trainer(net, lr=1.0e-3)
    opt = orc.AdamState(net.flat, lr=1.0e-3)
    first = None
    for _ in range(3):
        loss = t.step(L, R, D, V).cpu().numpy()
        first = loss if first is None else first
        gs = [orc.train_grads(net, L[k], R[k], D[k], V[k], 96, 64, params=opt.p)[1]
              for k in range(2)]
        opt.step(np.mean(gs, axis=0))
    # Adam moves every parameter by about lr whatever its gradient's size, so
    # compare the directions of the whole update
    moved_ref = opt.p - net.flat
    moved = t.params() - net.flat
    cos = float(np.dot(moved, moved_ref) / (np.linalg.norm(moved) * np.linalg.norm(moved_ref)))
    assert cos >= 0.95, cos
    for _ in range(100):
        loss = t.step(L, R, D, V).cpu().numpy()
    assert loss.mean() < 0.85 * first.mean(), (first, loss)


def test_drop_in_train_grads_fills_reference_lists(svb, net, train):
    """train_grads(net, sample) with a StereoNet-shaped object: the gradient
    lands in its gradient lists; train_step calls the caller's optimiser."""
    g = golden("training.npz")

    class Conv:
        def __init__(self, oc):
            self.oc = oc

    class Ref:
        def __init__(self, dil, rc):
            self.dilations = dil
            self.convs = [Conv(rc)]

    class Filt:
        def __init__(self, cm):
            self.c1 = Conv(cm)

    class FakeNet:
        def __init__(self, w):
            a = w.arch
            self.feat_C, self.D, self.max_disp, self.target_peak = a.feat_C, a.D, a.max_disp, 20
            self.filt = Filt(a.cost_C)
            self.ref1 = Ref(a.refine_dil, a.refine_C)
            self._p = [(list(b), [0.0] * len(b)) for b in w.blocks]

        def all_params(self):
            return self._p

    fake = FakeNet(net)
    H, W = g["s0_left"].shape
    sample = {"left": list(g["s0_left"].ravel() / 255.0), "right": list(g["s0_right"].ravel() / 255.0),
              "disp": list(g["s0_disp"].ravel()), "valid": list(g["s0_valid"].ravel()), "W": W, "H": H}
    total, pred, tgt = train.train_grads(fake, sample)
    flat_g = np.concatenate([np.asarray(gl) for _, gl in fake.all_params()])
    assert_grads_close(net, flat_g, g["s0_grads"])
    assert abs(total - g["s0_loss"][0]) <= LOSS_REL * g["s0_loss"][0]
    assert len(pred) == W * H and [len(x) for x in tgt["d"]] == [W * H // 16, W * H // 4, W * H]
    calls = []

    class Opt:
        def step(self):
            calls.append(1)

    train.train_step(fake, Opt(), sample)
    assert calls == [1]


def test_rejects_crops_the_reference_cannot_align(svb, net, train):
    t = train.Trainer(net)
    z = np.zeros((1, 62, 96), dtype=np.float32)
    with pytest.raises(ValueError):
        t.compute_grads(z, z, z, z.astype(bool))
    z = np.zeros((1, 64, 40), dtype=np.float32)          # quarter width 10 <= D - 2
    with pytest.raises(ValueError):
        t.compute_grads(z, z, z, z.astype(bool))
    assert torch.cuda.is_available()
