"""BF16 precision of the network (tcgen05 tensor-core convolutions).

FeatureNet c1..c4 and CostFilter c1/c2 (with the cost volume fused into c1)
run as BF16 implicit GEMMs with FP32 accumulation; CostFilter c3, the
soft-argmin and the Refinement stay FP32.

* Layout/numerics check: the GPU quarter-resolution disparity d0 must match
  a PyTorch FP64 emulation that rounds the same operands to BF16 and every
  layer output to FP32 (net_ref.front(bf16=True)) within 5e-3 px max /
  5e-4 px mean -- only the FP32 summation order and the rare BF16 rounding
  flip it causes differ.  A wrong operand layout gives errors of whole
  pixels.
* Error report: the BF16 result against the FP64 oracle is bounded
  (1.0 px max at full resolution for these inputs) and printed.
"""

import numpy as np
import pytest

import net_ref

pytestmark = pytest.mark.gpu

TOL_EMU_MAX = 5e-3
TOL_EMU_MEAN = 5e-4


def _images(svb, W, H, seed):
    p = svb.synth.make_pair(seed, W, H, 1.0, max(4.0, min(40.0, W / 4)))
    return (p.left.astype(np.float64).ravel() / 255.0,
            p.right.astype(np.float64).ravel() / 255.0)


def _random_net(svb, C, Cm, Rc, D, seed):
    arch = svb.weights.NetArch(feat_C=C, cost_C=Cm, D=D, refine_C=Rc, refine_dil=(1, 2, 4))
    rng = np.random.default_rng(seed)
    sizes = arch.block_sizes()
    blocks = []
    for i, n in enumerate(sizes):
        if i % 2 == 0:
            fan = n // (sizes[i + 1])
            blocks.append(rng.normal(0.0, np.sqrt(2.0 / fan), n))
        else:
            blocks.append(rng.normal(0.0, 0.05, n))
    return svb.weights.StereoNetWeights(arch, blocks)


def _front_check(svb, orc, w, W, H, seed):
    L, R = _images(svb, W, H, seed)
    gh, _, _ = orc.avgpool2(L, 1, H, W)
    d0, d1, d2 = svb.network.forward(w, L, R, H, W, gh, L, precision="bf16")
    emu = net_ref.front(w, L, R, H, W, bf16=True).ravel()
    err = np.abs(np.asarray(d0) - emu)
    assert err.max() < TOL_EMU_MAX and err.mean() < TOL_EMU_MEAN, (err.max(), err.mean())
    return L, R, gh, d0, d2


@pytest.mark.parametrize("W,H", [(96, 64), (97, 61), (160, 120), (333, 97)])
def test_bf16_front_matches_emulation(svb, orc, net, W, H):
    _front_check(svb, orc, net, W, H, seed=W)


@pytest.mark.parametrize("C,Cm,Rc,D", [(8, 4, 8, 8), (8, 4, 4, 12), (16, 8, 8, 16)])
def test_bf16_other_architectures(svb, orc, C, Cm, Rc, D):
    w = _random_net(svb, C, Cm, Rc, D, seed=C * 100 + D)
    _front_check(svb, orc, w, 120, 72, seed=D)


def test_bf16_error_vs_oracle_reported(svb, orc, net):
    W, H = 160, 120
    L, R, gh, d0, d2 = _front_check(svb, orc, net, W, H, seed=11)
    o0, o1, o2 = orc.stereonet_forward(net, L, R, H, W, gh, L)
    f0, f1, f2 = svb.network.forward(net, L, R, H, W, gh, L)
    e_bf = np.abs(np.asarray(d2) - np.asarray(o2))
    e_fp = np.abs(np.asarray(f2) - np.asarray(o2))
    print("\nfull-res disparity error vs FP64 oracle: BF16 max %.4f mean %.5f px, "
          "FP32 max %.2e mean %.2e px" % (e_bf.max(), e_bf.mean(), e_fp.max(), e_fp.mean()))
    assert e_fp.max() < 2e-3
    assert e_bf.max() < 1.0
    assert e_bf.mean() > e_fp.mean()          # BF16 really ran


def test_bf16_predict_auto_and_refinement_match_fraction(svb, orc, net):
    p = svb.synth.config_small()
    W, H = p.W, p.H
    (df, dw, Ww, Hw), tr = svb.network.predict_auto(net, p.left, p.right, W, H, verbose=False,
                                                     return_trace=True, precision="bf16")
    (of, ow, oWw, oHw), otr = orc.predict_auto(net, p.gray("left").ravel(),
                                               p.gray("right").ravel(), W, H, return_trace=True)
    err = np.abs(np.asarray(df) - np.asarray(of))
    kw = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    rb, sb = svb.refine.lr_refine(p.left, p.right, df, W, H, tol=2.0, **kw)
    ro, so = svb.refine.lr_refine(p.left, p.right, of, W, H, tol=2.0, **kw)
    same = np.mean((np.asarray(rb) == np.asarray(ro)) & (np.asarray(sb) == np.asarray(so)))
    print("\nconfig-small BF16 predict_auto: widths %s (oracle %s), max %.4f mean %.5f px, "
          "refinement bit-match %.4f" % (tr, otr, err.max(), err.mean(), same))
    assert err.max() < 1.5
    assert same > 0.8


def test_bf16_pipeline_graph_replay_deterministic(svb, net):
    import torch
    p = svb.synth.config_small()
    pp = svb.pipeline.PairPipeline(p.W, p.H, net, precision="bf16")
    pp.left.copy_(torch.from_numpy(p.left.ravel()))
    pp.right.copy_(torch.from_numpy(p.right.ravel()))
    outs = []
    for _ in range(3):
        pp.run_device()
        pp.stream.synchronize()
        outs.append(pp.out.clone())
    assert torch.equal(outs[0].view(torch.int64), outs[1].view(torch.int64))
    assert torch.equal(outs[0].view(torch.int64), outs[2].view(torch.int64))


def test_bad_precision_raises(svb, net):
    L, R = _images(svb, 64, 48, 1)
    with pytest.raises(ValueError):
        svb.network.predict(net, L, R, 64, 48, precision="fp16")
