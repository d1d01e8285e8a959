"""What the trained band net gains over the method without it.

Held-out 640x480 pairs of the learned-band workload (disparities 30-150 px,
thin foreground bars, 30% low texture; seeds outside the training and
validation ranges) are refined twice after the same FP32 predict_auto:
with the fixed +-10 band (lr_refine, refine_disparity's parameters) and with
the committed trained band net (weights/band_weights.npz).  Against the
generator's ground truth on valid pixels the learned band must cut both the
end-point error and the share of pixels off by more than 2 px at least in
half, at no less than 0.7x the fixed band's throughput.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SEEDS = range(3_000_500, 3_000_506)
W, H = 640, 480


def _score(d, gt, valid):
    e = np.abs(d - gt.ravel())[valid.ravel()]
    return e.mean(), (e > 2.0).mean()


def test_trained_band_beats_fixed_band(svb, net):
    band = svb.band.BandNet.load()
    pp = svb.pipeline.PairPipeline(W, H, net)
    lb = svb.band.LearnedBandRefiner(W, H, band, dmax=160)
    out = torch.empty(W * H, dtype=torch.float64, device="cuda")
    st = torch.empty(W * H, dtype=torch.uint8, device="cuda")
    fixed, learned, t_fixed, t_learned = [], [], 0.0, 0.0
    for seed in SEEDS:
        p = svb.synth.config_learned_crop(seed, W, H)
        with torch.cuda.stream(pp.stream):
            pp.left.copy_(torch.from_numpy(p.left.ravel()))
            pp.right.copy_(torch.from_numpy(p.right.ravel()))
        for k in range(2):                       # the first round records CUDA graphs
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(pp.stream)
            pp.run_device()
            e[1].record(pp.stream)
            pp.predict()
            lb.run(pp.left, pp.right, pp.code, pp.disp0, out, st, pp.stream.cuda_stream)
            e[2].record(pp.stream)
            e[2].synchronize()
            if k:
                t_fixed += e[0].elapsed_time(e[1])
                t_learned += e[1].elapsed_time(e[2])
        fixed.append(_score(pp.out.cpu().numpy(), p.disp, p.valid))
        learned.append(_score(out.cpu().numpy(), p.disp, p.valid))
    f, l = np.mean(fixed, axis=0), np.mean(learned, axis=0)
    print("\nfixed +-10: EPE %.3f bad2 %.4f; learned: EPE %.3f bad2 %.4f; throughput ratio %.2f"
          % (f[0], f[1], l[0], l[1], t_fixed / t_learned))
    assert l[0] < 0.5 * f[0] and l[1] < 0.5 * f[1]
    assert t_fixed / t_learned >= 0.7
