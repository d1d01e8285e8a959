"""Batched lr_refine (config 3's refinement): every pair of an uneven batch
must come out bit-identical to lr_refine on that pair alone."""

import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu

PIPE = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)


def _pairs(svb, shapes, seed0):
    out = []
    for i, (W, H) in enumerate(shapes):
        p = svb.synth.make_pair(seed0 + i, W, H, 1.0, max(4.0, min(60.0, W / 3)),
                                n_planes=(1, 4))
        rng = np.random.default_rng(seed0 + i)
        d0 = p.disp.ravel() + rng.uniform(-3, 3, W * H)
        d0[::97] = -0.0
        out.append((p.left, p.right, d0, W, H))
    return out


@pytest.mark.parametrize("kw", [PIPE, dict(R=3, P1=1.0, P2=12.0, rx=2, ry=2),
                                dict(R=10, P1=12.0, P2=400.0, rx=4, ry=3),
                                dict(R=14, P1=8.0, P2=90.0, rx=3, ry=2, paths=4)])
def test_batch_matches_single_pairs(svb, kw):
    shapes = [(1, 1), (7, 3), (64, 48), (333, 201), (41, 300), (1000, 31), (256, 192), (97, 61),
              (5, 200), (640, 17)]
    pairs = _pairs(svb, shapes, 900)
    got = svb.batch.lr_refine_batch(pairs, tol=2.0, **kw)
    for (L, R, d0, W, H), (o, s) in zip(pairs, got):
        ro, rs = svb.refine.lr_refine(L, R, d0, W, H, tol=2.0, **kw)
        assert np.array_equal(bits(o), bits(ro)), (W, H)
        assert np.array_equal(s, rs), (W, H)


def test_batch_config3_subset_vs_single(svb):
    # the batched workload's shapes (200x150 .. 1400x1100), 12 pairs
    pairs_cfg = svb.synth.config_batched(n=12, seed=3)
    pairs = []
    for i, p in enumerate(pairs_cfg):
        d0 = p.disp.ravel() + np.random.default_rng(i).uniform(-2.5, 2.5, p.W * p.H)
        pairs.append((p.left, p.right, d0, p.W, p.H))
    got = svb.batch.lr_refine_batch(pairs, tol=2.0, **PIPE)
    for (L, R, d0, W, H), (o, s) in zip(pairs, got):
        ro, rs = svb.refine.lr_refine(L, R, d0, W, H, tol=2.0, **PIPE)
        assert np.array_equal(bits(o), bits(ro)), (W, H)
        assert np.array_equal(s, rs), (W, H)


def test_batch_deterministic_and_reusable(svb):
    import torch
    pairs = _pairs(svb, [(200, 150), (450, 375), (90, 70)], 40)
    b = svb.batch.BatchRefiner([(p[3], p[4]) for p in pairs])
    for i, (L, R, d0, W, H) in enumerate(pairs):
        b.left[i].copy_(torch.from_numpy(L.ravel()))
        b.right[i].copy_(torch.from_numpy(R.ravel()))
        b.disp0[i].copy_(torch.from_numpy(d0))
    b.run()
    first = [o.clone() for o in b.out]
    b.run()
    b.data_status()
    for a, c in zip(first, b.out):
        assert torch.equal(a.view(torch.int64), c.view(torch.int64))


def test_batch_rejects_wide_band(svb):
    pairs = _pairs(svb, [(64, 48)], 7)
    with pytest.raises(ValueError):
        svb.batch.lr_refine_batch(pairs, tol=2.0, R=20, P1=12.0, P2=150.0, rx=4, ry=3)


def test_batch_nan_flagged(svb):
    pairs = _pairs(svb, [(64, 48), (80, 20)], 8)
    L, R, d0, W, H = pairs[1]
    d0 = d0.copy()
    d0[10] = 3.0e9
    pairs[1] = (L, R, d0, W, H)
    with pytest.raises(ValueError):
        svb.batch.lr_refine_batch(pairs, tol=2.0, **PIPE)


def _loaded_refiner(svb, pairs, **kw):
    import torch
    b = svb.batch.BatchRefiner([(p[3], p[4]) for p in pairs], **kw)
    for i, (L, R, d0, W, H) in enumerate(pairs):
        b.left[i].copy_(torch.from_numpy(L.ravel()))
        b.right[i].copy_(torch.from_numpy(R.ravel()))
        b.disp0[i].copy_(torch.from_numpy(d0))
    return b


def test_every_schedule_gives_the_same_bits(svb):
    """The scheduling knobs the autotuner moves change time only: each value
    of each knob reproduces lr_refine on every pair bit for bit."""
    import torch
    shapes = [(1, 1), (333, 201), (41, 300), (1000, 31), (256, 192), (5, 200)]
    pairs = _pairs(svb, shapes, 4400)
    b = _loaded_refiner(svb, pairs, **PIPE)
    ref = [svb.refine.lr_refine(L, R, d0, W, H, tol=2.0, **PIPE) for (L, R, d0, W, H) in pairs]
    for knob, values in svb.batch.TUNE_SPACE.items():
        for v in values + ((256, 8192) if knob == "px_per_block" else
                           (32,) if knob == "sgm_threads" else (1, 32) if knob == "sgm_ctas_per_sm"
                           else (128,)):
            cfg = svb.batch.BatchConfig.from_dict(dict(svb.batch.default_config().as_dict(),
                                                       **{knob: v}))
            b.config = cfg
            b.run()
            b.data_status()
            for i, (ro, rs) in enumerate(ref):
                assert np.array_equal(bits(b.out[i].cpu().numpy()), bits(ro)), (knob, v, i)
                assert np.array_equal(b.status[i].cpu().numpy(), rs), (knob, v, i)
    assert torch.cuda.is_available()


def test_autotune_picks_caches_and_keeps_results(svb, tmp_path, monkeypatch):
    monkeypatch.setenv("SV_B200_CACHE", str(tmp_path))
    pairs = _pairs(svb, [(450, 375), (200, 150), (640, 480), (97, 61)], 4500)
    b = _loaded_refiner(svb, pairs, **PIPE)
    b.run()
    want = [o.cpu().numpy().copy() for o in b.out]
    res = b.autotune(reps=2)
    assert not res["cached"] and res["ms"] <= res["default_ms"] and res["candidates"] >= 8
    assert b.config.as_dict() == res["config"]
    b.run()
    for a, o in zip(want, b.out):
        assert np.array_equal(bits(a), bits(o.cpu().numpy()))
    c = _loaded_refiner(svb, pairs, **PIPE)
    again = c.autotune()
    assert again["cached"] and again["config"] == res["config"]
    assert (tmp_path / "batch_tune.json").exists()


def test_bad_schedule_rejected(svb):
    pairs = _pairs(svb, [(64, 48)], 4600)
    b = _loaded_refiner(svb, pairs, **PIPE)
    b.config = svb.batch.BatchConfig(3000, 128, 8, 32)
    with pytest.raises(ValueError):
        b.run()
