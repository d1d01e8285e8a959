"""Precision workload: the network on 64 pairs of 640x480 (disparities
0-120 px) in FP32 and in BF16 (tensor-core feature and cost-filter
convolutions), against the FP64 oracle of predict_auto.

Reported per precision: per-pair max and mean |disparity - oracle| (px),
whether predict_auto chose the oracle's work widths, the fraction of pixels
whose refinement (lr_refine, refine_disparity's parameters) from that
disparity is bit-identical -- value and status -- to the refinement from the
FP64 disparity, and the predict_auto throughput.  SV_PRECISION_REPORT names
an optional JSON file for the full table; SV_PRECISION_PAIRS limits the pairs.

Pixels whose refined value is the network disparity itself (edge winners,
left-right mismatches) carry the network's rounding in their bits, so the
table also gives the share of pixels within 0.01 px with the same status.
BF16 runs only in the pass no work-width decision follows (the probe and
the quantile-selecting passes stay FP32), so BF16 chooses FP32's widths --
before that rule a BF16 pass moved the 95% quantile across a width step on
28 of 64 pairs -- and only pairs that reach the last permitted pass see
BF16 at all.

Bounds: FP32 within 2e-3 px and refinement within 0.01 px on 99% of pixels
on every pair; BF16 the oracle's widths on every pair FP32 has them, the
bounds of BF16_BOUNDS (set from the measured run, with margin).
"""

import json
import os

import numpy as np
import pytest
import torch

from conftest import bits

pytestmark = pytest.mark.gpu

KW = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
# measured on the 64 pairs: max 4.25 px (local), mean 0.0447 px, refined
# within 0.01 px 89.1 %, bit-identical 82.2 %; the bounds keep a margin
BF16_BOUNDS = dict(max_px=6.0, mean_px=0.06, refined_within_001=0.86, refined_bit_match=0.78)


def _throughput(svb, net, pairs, precision):
    W, H = pairs[0].W, pairs[0].H
    pp = svb.pipeline.PairPipeline(W, H, net, precision=precision)
    total = 0.0
    for p in pairs:
        pp.left.copy_(torch.from_numpy(p.left.ravel()))
        pp.right.copy_(torch.from_numpy(p.right.ravel()))
        pp.predict()                                   # records this width's graphs
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(pp.stream)
        pp.predict()
        e1.record(pp.stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return len(pairs) * W * H / 1e6 / (total / 1e3)


def test_precision_workload(svb, orc, net):
    n = int(os.environ.get("SV_PRECISION_PAIRS", "64"))
    pairs = svb.synth.config_precision(n)
    orc.set_threads(orc.max_threads())
    rows = []
    for i, p in enumerate(pairs):
        W, H = p.W, p.H
        (of, _, _, _), otr = orc.predict_auto(net, p.gray("left").ravel(), p.gray("right").ravel(),
                                              W, H, return_trace=True)
        ref_o, ref_s = svb.refine.lr_refine(p.left, p.right, of, W, H, tol=2.0, **KW)
        row = {"pair": i, "oracle_widths": otr}
        for prec in ("fp32", "bf16"):
            (df, _, _, _), tr = svb.network.predict_auto(net, p.left, p.right, W, H,
                                                         verbose=False, return_trace=True,
                                                         precision=prec)
            e = np.abs(np.asarray(df) - of)
            o, s = svb.refine.lr_refine(p.left, p.right, df, W, H, tol=2.0, **KW)
            st_same = np.asarray(s) == np.asarray(ref_s)
            same = (bits(o) == bits(ref_o)) & st_same
            close = (np.abs(np.asarray(o) - np.asarray(ref_o)) <= 0.01) & st_same
            row[prec] = dict(max_px=float(e.max()), mean_px=float(e.mean()),
                             same_widths=tr == otr, widths=tr,
                             refined_bit_match=float(same.mean()),
                             refined_within_001=float(close.mean()))
        rows.append(row)
    summary = {}
    for prec in ("fp32", "bf16"):
        r = [row[prec] for row in rows]
        same_w = [x for x in r if x["same_widths"]]
        summary[prec] = dict(
            pairs=len(r), pairs_same_widths=len(same_w),
            max_px=max(x["max_px"] for x in r), mean_px=float(np.mean([x["mean_px"] for x in r])),
            max_px_same_widths=max((x["max_px"] for x in same_w), default=None),
            mean_px_same_widths=float(np.mean([x["mean_px"] for x in same_w])) if same_w else None,
            refined_bit_match=float(np.mean([x["refined_bit_match"] for x in r])),
            refined_within_001=float(np.mean([x["refined_within_001"] for x in r])),
            refined_within_001_same_widths=float(np.mean([x["refined_within_001"]
                                                          for x in same_w])) if same_w else None,
            predict_auto_mpix_s=_throughput(svb, net, pairs[:min(16, n)], prec))
    print("\n" + json.dumps(summary, indent=1))
    path = os.environ.get("SV_PRECISION_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump({"summary": summary, "pairs": rows}, f, indent=1)
    fp, bf = summary["fp32"], summary["bf16"]
    assert fp["pairs_same_widths"] == n and fp["max_px"] < 2e-3
    assert fp["refined_within_001"] > 0.99
    assert all(r["bf16"]["widths"] == r["fp32"]["widths"] for r in rows)
    assert bf["pairs_same_widths"] == n
    assert bf["max_px"] < BF16_BOUNDS["max_px"] and bf["mean_px"] < BF16_BOUNDS["mean_px"]
    assert bf["refined_within_001"] > BF16_BOUNDS["refined_within_001"]
    assert bf["refined_bit_match"] > BF16_BOUNDS["refined_bit_match"]
