"""Train and evaluate the learned adaptive band on the GPU.

    python from-scratch-stereo-vision_b200/band_train.py train --crops 20000 --out W.npz
    python from-scratch-stereo-vision_b200/band_train.py eval --weights W.npz --pairs 500

Training data: seeded synthetic 256x192 crops (disparities 30-150 px, 1-3
thin foreground bars 2-6 px wide, 30% low-texture area).  Per crop the GPU
runs the network (predict_auto), the band features (with the network's own
confidence), the rule centre and the label: the plain method's full-range
census + SGM disparity, lr_refine with disp0 = R and
R = (max disparity + 2) // 2 + 1 (eval_real.py:143-146); pixels whose label
fails the left-right check are unlabelled; the target is the label's shift
from the rule centre.  The rule's threshold (the wide search's cost below
which its argmin replaces the network disparity) is chosen first, on the
validation pairs, with no net.  The band
net is trained with its own BF16 kernels and Adam (lr 5e-4).  The band
application thresholds are then chosen on validation pairs, and the
evaluation scores held-out 640x480 pairs against the generator's ground
truth: EPE and bad2 (|error| > 2 px) on valid pixels for the learned band,
the fixed +-10 band and full-range SGM, each with its Mpix/s.
"""

from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import math
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)

TRAIN_SEED0, VAL_SEED0, TEST_SEED0 = 1_000_000, 2_000_000, 3_000_000
DMAX = 160                         # feature search range (disparities 30-150)
REFINE = dict(R=10, P1=12.0, P2=150.0, rx=4, ry=3)
TOL = 2.0


# ------------------------------------------------------------ host side
def _synth():
    """synth.py loaded on its own (numpy only), for the generator processes."""
    if "sv_synth" in sys.modules:
        return sys.modules["sv_synth"]
    spec = importlib.util.spec_from_file_location("sv_synth", os.path.join(HERE, "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sv_synth"] = mod          # dataclasses look their module up while it loads
    spec.loader.exec_module(mod)
    return mod


_SYN = None


def _gen(args):
    seed, W, H = args
    p = _SYN.config_learned_crop(seed, W, H)
    return seed, p.left, p.right, p.disp, p.valid


def _init_worker():
    global _SYN
    _SYN = _synth()


def make_pool(workers: int | None = None):
    """A spawn pool for the generator (start it before the first CUDA call).
    The generator is first run once in this process, so a broken worker
    set-up raises here instead of respawning workers forever."""
    _init_worker()
    _gen((0, 32, 24))
    n = workers or max(1, min(64, (os.cpu_count() or 2) - 1))
    return mp.get_context("spawn").Pool(n, initializer=_init_worker)


def generate(pool, seeds, W, H, timeout=300.0):
    """(seed, left, right, disp, valid) in seed order; each wait is bounded."""
    # one task per crop: imap then returns an iterator whose waits can time out
    it = pool.imap(_gen, [(s, W, H) for s in seeds])
    for _ in range(len(seeds)):
        yield it.next(timeout)


def full_range_R(disp) -> int:
    """Band radius of full-range SGM for a pair whose largest disparity is
    max(disp): the band [0, 2R] covers it (eval_real.py:143-146)."""
    return (int(math.ceil(float(np.max(disp)))) + 2) // 2 + 1


# ------------------------------------------------------------- GPU side
def _package():
    sys.path.insert(0, REPO)
    import __graft_entry__
    return __graft_entry__.load_package()


class FullRange:
    """Device-resident full-range lr_refine (disp0 = R everywhere) of one size."""

    def __init__(self, svb, W, H):
        import torch
        self.svb, self.torch, self.W, self.H = svb, torch, W, H
        self.lib = svb._lib.load()
        self.out = torch.empty(W * H, dtype=torch.float64, device="cuda")
        self.status = torch.empty(W * H, dtype=torch.uint8, device="cuda")
        self.cache = {}

    def run(self, left, right, code, R, stream):
        torch, W, H = self.torch, self.W, self.H
        if R not in self.cache:
            p = self.svb.refine._params(**dict(REFINE, R=R))
            need = self.lib.sv_lr_refine_workspace_size(W, H, ctypes.byref(p))
            if need == 0:
                self.svb._lib.raise_last("full-range lr_refine")
            self.cache[R] = (p, torch.empty(need, dtype=torch.uint8, device="cuda"), need,
                             torch.full((W * H,), float(R), dtype=torch.float64, device="cuda"))
        p, ws, need, d0 = self.cache[R]
        vp = lambda t: ctypes.c_void_p(t.data_ptr())                     # noqa: E731
        self.svb._lib.check(self.lib.sv_lr_refine(vp(left), vp(right), code, vp(d0), W, H, TOL,
                                                  ctypes.byref(p), vp(self.out),
                                                  vp(self.status), vp(ws), need, stream),
                            "full-range lr_refine")
        return self.out, self.status


class Labeller:
    """Network disparity, features and full-range labels of one crop size."""

    def __init__(self, svb, net, W, H, tau):
        import torch
        self.svb, self.torch, self.tau = svb, torch, float(tau)
        self.pipe = svb.pipeline.PairPipeline(W, H, net)
        self.base = torch.empty(W * H, dtype=torch.float64, device="cuda")
        self.full = FullRange(svb, W, H)
        self.W, self.H = W, H
        N = W * H
        self.feat = torch.empty(svb.band.N_FEATURES * N, dtype=torch.float32, device="cuda")
        self.fneed = self.full.lib.sv_band_features_workspace_size(W, H)
        self.fws = torch.empty(self.fneed, dtype=torch.uint8, device="cuda")
        self.t = torch.empty(N, dtype=torch.float32, device="cuda")
        self.m = torch.empty(N, dtype=torch.uint8, device="cuda")

    def __call__(self, left, right, disp):
        torch, svb, lib = self.torch, self.svb, self.full.lib
        pp, W, H = self.pipe, self.W, self.H
        vp = lambda t: ctypes.c_void_p(t.data_ptr())                     # noqa: E731
        s = pp.stream.cuda_stream
        with torch.cuda.stream(pp.stream):
            pp.left.copy_(torch.from_numpy(left.ravel()), non_blocking=False)
            pp.right.copy_(torch.from_numpy(right.ravel()), non_blocking=False)
        pp.predict()
        sp, pm = pp.confidence()
        lab, st = self.full.run(pp.left, pp.right, pp.code, full_range_R(disp), s)
        svb._lib.check(lib.sv_band_features(vp(pp.left), vp(pp.right), pp.code, vp(pp.disp0),
                                            W, H, DMAX, vp(self.feat), vp(self.fws), self.fneed,
                                            s), "band_features")
        svb._lib.check(lib.sv_band_conf_features(vp(sp), vp(pm), W, H, vp(self.feat), s),
                       "band_conf_features")
        # the net learns the shift from the rule centre
        svb._lib.check(lib.sv_band_rule_centre(vp(self.feat), vp(pp.disp0), W, H, self.tau,
                                               vp(self.base), s), "band_rule_centre")
        svb._lib.check(lib.sv_band_targets(vp(lab), vp(st), vp(self.base), W * H, 160.0,
                                           vp(self.t), vp(self.m), s), "band_targets")
        return self.feat, self.t, self.m


def make_dataset(svb, pool, n, tau, W=256, H=192, seed0=TRAIN_SEED0, log=print):
    import torch
    net = svb.weights.load_model()
    lab = Labeller(svb, net, W, H, tau)
    N = W * H
    feats = torch.empty(n, svb.band.N_FEATURES * N, dtype=torch.float32, device="cuda")
    tgt = torch.empty(n, N, dtype=torch.float32, device="cuda")
    msk = torch.empty(n, N, dtype=torch.uint8, device="cuda")
    t0 = time.time()
    st = lab.pipe.stream
    for i, (seed, L, R, D, V) in enumerate(generate(pool, range(seed0, seed0 + n), W, H)):
        f, t, m = lab(L, R, D)
        with torch.cuda.stream(st):
            feats[i].copy_(f)
            tgt[i].copy_(t)
            msk[i].copy_(m)
        if (i + 1) % 1000 == 0:
            st.synchronize()
            log("  %d / %d crops (%.1f s)" % (i + 1, n, time.time() - t0))
    st.synchronize()
    return feats, tgt, msk


def train(svb, feats, tgt, msk, W, H, epochs=8, nb=16, lr=5e-4, seed=0, log=print):
    import torch
    band = svb.band.BandNet(seed=seed)
    n = feats.shape[0]
    rng = np.random.default_rng(seed)
    t0 = time.time()
    steps = 0
    losses = []
    for ep in range(epochs):
        order = torch.from_numpy(rng.permutation(n)).cuda()
        acc = torch.zeros(1, dtype=torch.float64, device="cuda")
        nbat = n // nb
        for b in range(nbat):
            idx = order[b * nb:(b + 1) * nb]
            f = feats.index_select(0, idx).contiguous()
            t = tgt.index_select(0, idx).contiguous()
            m = msk.index_select(0, idx).contiguous()
            band.train_step(f, t, m, nb, W, H, lr=lr)
            acc += band._step_loss()
            steps += 1
        torch.cuda.synchronize()
        losses.append(acc.item() / max(1, nbat))
        log("  epoch %d: mean loss %.4f (%.1f s, %d steps)"
            % (ep + 1, losses[-1], time.time() - t0, steps))
    return band, dict(epochs=epochs, batch=nb, lr=lr, steps=steps, epoch_loss=losses,
                      seconds=round(time.time() - t0, 2))


# -------------------------------------------------------------- scoring
def _score(d, gt, valid):
    e = np.abs(np.asarray(d) - gt.ravel())[valid.ravel()]
    return float(e.mean()), float((e > 2.0).mean())


class Evaluator:
    """The three methods on one W x H size, device resident, on one stream."""

    def __init__(self, svb, net, band, W, H):
        import torch
        self.svb, self.torch, self.W, self.H = svb, torch, W, H
        self.pp = svb.pipeline.PairPipeline(W, H, net)
        self.lb = svb.band.LearnedBandRefiner(W, H, band, dmax=DMAX, **REFINE, tol=TOL)
        self.full = FullRange(svb, W, H)
        N = W * H
        self.out_l = torch.empty(N, dtype=torch.float64, device="cuda")
        self.st_l = torch.empty(N, dtype=torch.uint8, device="cuda")

    def load(self, left, right):
        with self.torch.cuda.stream(self.pp.stream):
            self.pp.left.copy_(self.torch.from_numpy(left.ravel()))
            self.pp.right.copy_(self.torch.from_numpy(right.ravel()))

    def fixed(self):
        self.pp.run_device()
        return self.pp.out

    def learned(self):
        pp = self.pp
        pp.predict()
        sp, pm = pp.confidence()
        self.lb.run(pp.left, pp.right, pp.code, pp.disp0, self.out_l, self.st_l,
                    pp.stream.cuda_stream, sp, pm)
        return self.out_l

    def full_range(self, R):
        return self.full.run(self.pp.left, self.pp.right, self.pp.code, R,
                             self.pp.stream.cuda_stream)[0]

    def rule(self, tau):
        """The ablation without the net: lr_refine with the full +-R band
        around the rule centre (the network disparity moved to the wide
        search's argmin wherever that argmin's 9-row cost is below tau) --
        the learned band's starting point, with no net on top."""
        torch, pp, lb, W, H = self.torch, self.pp, self.lb, self.W, self.H
        lib = lb.lib
        vp = lambda t: ctypes.c_void_p(t.data_ptr())                     # noqa: E731
        s = pp.stream.cuda_stream
        pp.predict()
        self.svb._lib.check(lib.sv_band_features(vp(pp.left), vp(pp.right), pp.code,
                                                 vp(pp.disp0), W, H, DMAX, vp(lb.feat),
                                                 vp(lb.fws), lb.fneed, s), "band_features")
        self.svb._lib.check(lib.sv_band_rule_centre(vp(lb.feat), vp(pp.disp0), W, H,
                                                    float(tau), vp(lb.centre), s),
                            "band_rule_centre")
        with torch.cuda.stream(pp.stream):
            lb.rad.fill_(REFINE["R"])
        self.svb._lib.check(lib.sv_lr_refine_band(vp(pp.left), vp(pp.right), pp.code,
                                                  vp(lb.centre), vp(lb.rad), W, H, TOL,
                                                  ctypes.byref(lb.p), vp(self.out_l),
                                                  vp(self.st_l), vp(lb.rws), lb.rneed, s),
                            "lr_refine_band")
        return self.out_l


def _timed(torch, stream, fn):
    """(result, device ms) of a second fn() on `stream` (host syncs inside
    included).  The untimed first run records the CUDA graphs of a new
    predict_auto work width and allocates any new workspace, so every method
    is timed in the same steady state."""
    fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r = fn()
    e1.record(stream)
    e1.synchronize()
    return r, e0.elapsed_time(e1)


def evaluate(svb, pool, band, n, W=640, H=480, seed0=TEST_SEED0, apply_grid=None,
             rule_taus=None, learned=True, log=print):
    """Scores of the methods on n pairs: the fixed band, full-range SGM, the
    learned band and the no-net rule (Evaluator.rule).  With apply_grid
    every band application setting is scored and the best (bad2, then EPE)
    kept; with rule_taus every rule threshold likewise (else the band's
    rule_tau).  The learned band's half-width histogram is reported."""
    import torch
    net = svb.weights.load_model()
    ev = Evaluator(svb, net, band, W, H)
    grid = (apply_grid or [dict(band.meta)]) if learned else []
    taus = rule_taus or [float(band.meta.get("rule_tau", 0.1))]
    acc = {"fixed": [], "full": []}
    acc_l = [[] for _ in grid]
    acc_r = [[] for _ in taus]
    hist_l = [torch.zeros(11, dtype=torch.int64, device="cuda") for _ in grid]
    times = {"fixed": 0.0, "learned": 0.0, "full": 0.0, "rule": 0.0}
    st = ev.pp.stream
    # warm-up: the first predict_auto per work width records its CUDA graphs
    for seed, L, R, D, V in generate(pool, range(seed0 - 2, seed0), W, H):
        ev.load(L, R)
        ev.fixed()
        if learned:
            ev.learned()
        ev.rule(taus[0])
    for i, (seed, L, R, D, V) in enumerate(generate(pool, range(seed0, seed0 + n), W, H)):
        ev.load(L, R)
        out, dt = _timed(torch, st, ev.fixed)
        times["fixed"] += dt
        acc["fixed"].append(_score(out.cpu().numpy(), D, V))
        Rf = full_range_R(D)
        out, dt = _timed(torch, st, lambda: ev.full_range(Rf))
        times["full"] += dt
        acc["full"].append(_score(out.cpu().numpy(), D, V))
        for j, g in enumerate(grid):
            band.meta.update(g)
            out, dt = _timed(torch, st, ev.learned)
            if j == 0:
                times["learned"] += dt
            acc_l[j].append(_score(out.cpu().numpy(), D, V))
            with torch.cuda.stream(st):
                hist_l[j] += torch.bincount(ev.lb.rad.long(), minlength=11)[:11]
        for j, tau in enumerate(taus):
            out, dt = _timed(torch, st, lambda: ev.rule(tau))
            if j == 0:
                times["rule"] += dt
            acc_r[j].append(_score(out.cpu().numpy(), D, V))
        if (i + 1) % 100 == 0:
            log("  %d / %d pairs" % (i + 1, n))
    mpix = n * W * H / 1e6
    res = {"pairs": n, "size": [W, H]}
    for key, name in (("fixed", "fixed_pm10"), ("full", "full_range")):
        a = np.array(acc[key])
        res[name] = dict(epe=float(a[:, 0].mean()), bad2=float(a[:, 1].mean()),
                         mpix_s=mpix / (times[key] / 1e3))
    scores = [np.array(a) for a in acc_l]
    if grid:
        best = min(range(len(grid)),
                   key=lambda j: (scores[j][:, 1].mean(), scores[j][:, 0].mean()))
        band.meta.update(grid[best])
        h = hist_l[best].cpu().numpy()
        res["learned"] = dict(epe=float(scores[best][:, 0].mean()),
                              bad2=float(scores[best][:, 1].mean()),
                              mpix_s=mpix / (times["learned"] / 1e3), apply=dict(grid[best]),
                              half_width_hist={str(r): int(h[r]) for r in range(11) if h[r]})
    rs = [np.array(a) for a in acc_r]
    rb = min(range(len(taus)), key=lambda j: (rs[j][:, 1].mean(), rs[j][:, 0].mean()))
    res["rule_no_net"] = dict(epe=float(rs[rb][:, 0].mean()), bad2=float(rs[rb][:, 1].mean()),
                              mpix_s=mpix / (times["rule"] / 1e3), tau=float(taus[rb]))
    if apply_grid:
        res["grid"] = [dict(g, epe=float(s[:, 0].mean()), bad2=float(s[:, 1].mean()))
                       for g, s in zip(grid, scores)]
    if rule_taus:
        res["rule_grid"] = [dict(tau=float(t), epe=float(s[:, 0].mean()),
                                 bad2=float(s[:, 1].mean())) for t, s in zip(taus, rs)]
    return res


def apply_grid():
    """Band application settings tried on the validation pairs: thresholds on
    the predicted Laplace scale b, and half-widths ceil(rad_k * b) clamped
    to [rad_min, 10] that vary with b (the full +-10 width around a moved
    centre, rad_k = 100, is not among them)."""
    out = []
    for b_thr in (2.5, 4.0, 6.0, 10.0, 16.0, 32.0):
        for rad_k in (1.0, 1.5, 2.0, 3.0, 4.0):
            out.append(dict(b_thr=b_thr, rad_k=rad_k, rad_min=3, R=10, shift_max=160.0))
    return out


RULE_TAUS = (0.15, 0.2, 0.3, 0.4, 0.5, 0.7, 1.1)   # 1.1: always the argmin


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--crops", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--val", type=int, default=24)
    ap.add_argument("--pairs", type=int, default=500)
    ap.add_argument("--weights", default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    ap.add_argument("--workers", type=int, default=None)
    a = ap.parse_args(argv)
    pool = make_pool(a.workers)           # before any CUDA call
    svb = _package()
    import torch
    torch.cuda.init()
    report = {"host_cores": os.cpu_count()}
    if a.cmd == "train":
        # the rule's threshold first: the net learns the shift from its centre
        t0 = time.time()
        probe = svb.band.BandNet(seed=0)
        rv = evaluate(svb, pool, probe, a.val, seed0=VAL_SEED0, rule_taus=list(RULE_TAUS),
                      learned=False)
        tau = rv["rule_no_net"]["tau"]
        report["rule_validation"] = dict(rv["rule_no_net"], grid=rv["rule_grid"],
                                         seconds=round(time.time() - t0, 1))
        print("rule: tau %.2f, EPE %.3f bad2 %.4f on %d validation pairs"
              % (tau, rv["rule_no_net"]["epe"], rv["rule_no_net"]["bad2"], a.val), flush=True)
        del probe
        t0 = time.time()
        feats, tgt, msk = make_dataset(svb, pool, a.crops, tau)
        report["data"] = dict(crops=a.crops, size=[256, 192], seconds=round(time.time() - t0, 1),
                              labelled=float(msk.float().mean()))
        print("dataset: %d crops, %.1f%% labelled, %.1f s"
              % (a.crops, 100 * report["data"]["labelled"], time.time() - t0), flush=True)
        band, info = train(svb, feats, tgt, msk, 256, 192, epochs=a.epochs, nb=a.batch, lr=a.lr)
        band.meta["rule_tau"] = tau
        report["train"] = info
        del feats, tgt, msk
        torch.cuda.empty_cache()
        if a.val > 0:
            val = evaluate(svb, pool, band, a.val, seed0=VAL_SEED0, apply_grid=apply_grid())
            report["validation"] = val
            print("validation:", json.dumps(val["learned"]), flush=True)
        if a.out:
            band.save(a.out)
    else:
        band = svb.band.BandNet.load(a.weights)
    if a.pairs > 0:
        res = evaluate(svb, pool, band, a.pairs)
        report["test"] = res
        print(json.dumps(res), flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    pool.close()
    return report


if __name__ == "__main__":
    main()
