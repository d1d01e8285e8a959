"""predict_auto + lr_refine for a batch of uneven pairs with the work-width
decisions on the device (batch.NetBatch, sv_netbatch_*), against
network.predict_auto + refine.lr_refine on each pair alone.

The batch runs the single-pair path's kernels on every pair, so each pair's
network disparity (FP64 bits), its work-width trace and final work size,
and its refined disparity and status must be identical -- including a pair
small enough to run at native resolution, a tall pair whose probe map is
larger than the one-CTA select's shared memory, and pairs that stop after
different numbers of passes.  A second run replays the recorded CUDA graph
and must give the same bits again.
"""

import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu

KW = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)


def _pairs(svb):
    s = svb.synth
    pairs = [
        s.config_small(),                                   # 160x120: native resolution
        s.config_full(),                                    # 450x375
        s.make_pair(11, 44, 40, 1.0, 8.0, n_planes=(1, 2)),      # narrower than 48 px
        s.make_pair(12, 100, 500, 2.0, 30.0, n_planes=(2, 4)),   # probe map > 16384 values
        s.make_pair(13, 97, 61, 1.0, 20.0, n_planes=(1, 3)),
        s.make_pair(14, 640, 480, 0.0, 120.0, n_planes=(4, 8), lowtex_frac=0.3),
    ]
    pairs += s.config_batched(n=4, seed=5)
    return pairs


def test_netbatch_matches_single_pair(svb, net):
    import torch
    pairs = _pairs(svb)
    nb = svb.batch.NetBatch([(p.W, p.H) for p in pairs], net, tol=2.0, **KW)
    for i, p in enumerate(pairs):
        nb.left[i].copy_(torch.from_numpy(p.left.ravel()))
        nb.right[i].copy_(torch.from_numpy(p.right.ravel()))
    nb.run()
    nb.data_status()
    torch.cuda.synchronize()
    first = [(nb.disparity(i).cpu().numpy().copy(), nb.out[i].cpu().numpy().copy(),
              nb.status[i].cpu().numpy().copy()) for i in range(len(pairs))]
    traces = nb.traces()
    nb.run()                                             # graph replay
    torch.cuda.synchronize()
    for i, p in enumerate(pairs):
        W, H = p.W, p.H
        (df, dw, Ww, Hw), trace = svb.network.predict_auto(net, p.left, p.right, W, H,
                                                           verbose=False, return_trace=True)
        d, out, st = first[i]
        assert traces[i][0] == trace and traces[i][1] == (Ww, Hw), (i, W, H, traces[i], trace)
        assert np.array_equal(bits(d), bits(df)), (i, W, H, np.abs(d - df).max())
        ro, rs = svb.refine.lr_refine(p.left, p.right, df, W, H, tol=2.0, **KW)
        assert np.array_equal(bits(out), bits(ro)), (i, W, H)
        assert np.array_equal(st, rs.astype(np.uint8)), (i, W, H)
        assert np.array_equal(bits(nb.disparity(i).cpu().numpy()), bits(d))
        assert np.array_equal(bits(nb.out[i].cpu().numpy()), bits(out))


def test_netbatch_predict_only_and_one_pair(svb, net):
    import torch
    p = svb.synth.config_full()
    nb = svb.batch.NetBatch([(p.W, p.H)], net, tol=2.0, **KW)
    nb.left[0].copy_(torch.from_numpy(p.left.ravel()))
    nb.right[0].copy_(torch.from_numpy(p.right.ravel()))
    nb.predict()
    torch.cuda.synchronize()
    (df, _, Ww, Hw), trace = svb.network.predict_auto(net, p.left, p.right, p.W, p.H,
                                                      verbose=False, return_trace=True)
    assert nb.traces()[0] == (trace, (Ww, Hw))
    assert np.array_equal(bits(nb.disparity(0).cpu().numpy()), bits(df))
