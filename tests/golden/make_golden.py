"""Generate the golden fixtures by running the reference itself.

Run where the reference checkout is available (read-only is fine), giving
its directory as the argument or in SV_REFERENCE_DIR:

    python tests/golden/make_golden.py <reference checkout>

It executes ``stereonet.py`` into a namespace exactly the way the reference's
own test suite does (test_stereonet.py:18-22: strip the ``run_demo()`` guard,
``exec`` into a dict), feeds it seeded synthetic pairs from this package's
generator, and stores the reference's outputs.  Small outputs are stored as
arrays; large ones (the 450x375 workload) as SHA-256 digests of their FP64
bytes.  The fixtures are what pins the C oracle: tests/test_oracle_golden.py
checks the oracle against every one of them.  Nothing on the GPU box reads the
reference; it only reads these files.
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "from-scratch-stereo-vision_b200"))
import synth  # noqa: E402


def load_reference(ref_dir):
    src = open(os.path.join(ref_dir, "stereonet.py")).read().replace(
        "if __name__ == '__main__':\n    run_demo()\n", "")
    SN = {"__name__": "stereonet_golden"}
    exec(src, SN)
    return SN


def sha(a, dtype=np.float64) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=dtype)).tobytes()).hexdigest()


def as_int_array(vals, dtype):
    a = np.asarray(vals, dtype=np.float64)
    assert np.all(a == np.round(a)), "expected integer-valued output"
    return a.astype(dtype)


def tricky_disp0(pair, rng, noise=3.0):
    """Ground truth + noise, plus the values that exercise the rounding and
    tie rules: negative zeros, exact halves, values in (-1, 0), block jumps
    larger than a band, and ties that land on the same right-image column."""
    W, H = pair.W, pair.H
    d = pair.disp.ravel() + rng.uniform(-noise, noise, W * H)
    idx = rng.choice(W * H, size=W * H // 40, replace=False)
    d[idx[0::5]] = -0.0
    d[idx[1::5]] = np.floor(d[idx[1::5]]) + 0.5
    d[idx[2::5]] = -rng.uniform(0.0, 1.0, len(idx[2::5]))
    d[idx[3::5]] = np.floor(d[idx[3::5]]) - 0.5
    d[idx[4::5]] = 0.0
    # a block far off the truth: band re-centring jumps larger than K
    y0, x0 = H // 3, W // 3
    blk = d.reshape(H, W)
    blk[y0:y0 + H // 4, x0:x0 + W // 4] += 25.0
    # ties on one row: equal disparities that warp to the same column
    r = H // 2
    for x in range(4, min(W, 12)):
        blk[r, x] = float(x - 3)          # x - d + 0.5 = 3.5 -> column 3 for all
    return blk.ravel().copy()


def main(ref_dir):
    t0 = time.time()
    SN = load_reference(ref_dir)
    net = SN["load_model"](os.path.join(ref_dir, "stereonet_weights.txt"))
    flat = [v for p, _ in net.all_params() for v in p]
    meta = {"weights_sha256": sha(flat), "n_params": len(flat),
            "target_peak": net.target_peak}
    print("reference loaded: %d params (%.1fs)" % (len(flat), time.time() - t0))

    # ------------------------------------------------------------ primitives
    rng = np.random.default_rng(7)
    fx = np.array([-701.0, -50.3, -3.7, -0.5, -1e-9, 0.0, 1e-9, 0.25, 0.6931471805599453,
                   1.0, 3.3, 20.0, 88.5, 699.9, 701.0])
    fexp = np.array([SN["fexp"](float(v)) for v in fx])
    img = rng.random(13 * 9)
    rs = {}
    for (W2, H2) in ((13, 9), (7, 5), (29, 17), (20, 9), (13, 30)):
        rs["resize_%dx%d" % (W2, H2)] = np.array(SN["resize_gray"](list(img), 13, 9, W2, H2))
    ap, _, _ = SN["avgpool2"](list(img), 1, 9, 13)
    pk_in = rng.uniform(-1, 30, 1001)
    pk_in[::7] = -0.0
    pk = SN["_peak"](list(pk_in))
    np.savez_compressed(os.path.join(HERE, "primitives.npz"), fexp_x=fx, fexp=fexp,
                        img=img, avgpool=np.array(ap), peak_in=pk_in, peak=np.array([pk]),
                        **rs)
    print("primitives done (%.1fs)" % (time.time() - t0))

    # ------------------------------------------------------ refinement, small
    pair = synth.make_pair(11, 64, 48, 2.0, 20.0, n_planes=(2, 4))
    W, H = pair.W, pair.H
    L = list(pair.gray("left").ravel())
    R = list(pair.gray("right").ravel())
    d0 = tricky_disp0(pair, np.random.default_rng(12))
    d0l = [float(v) for v in d0]
    out = {"left": pair.left, "right": pair.right, "disp0": d0}
    cl = SN["census"](L, W, H, 4, 3)
    cr = SN["census"](R, W, H, 4, 3)
    out["census_l_4x3"] = np.array(cl, dtype=np.uint64)
    out["census_r_4x3"] = np.array(cr, dtype=np.uint64)
    out["census_l_2x2"] = np.array(SN["census"](L, W, H, 2, 2), dtype=np.uint64)
    out["census_r_1x1"] = np.array(SN["census"](R, W, H, 1, 1), dtype=np.uint64)
    Rb = 10
    base = [max(0, int(v + 0.5)) for v in d0l]
    out["base"] = np.array(base, dtype=np.int64)
    C = SN["band_costs"](cl, cr, L, R, base, W, H, Rb, 0.0, 20.0, 66.0, d0l, 0.0, 4.0)
    out["costs_R10"] = as_int_array(C, np.uint8)
    K = 2 * Rb + 1
    dirs = [(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, 1), (1, -1), (-1, -1)]
    for i, (dx, dy) in enumerate(dirs):
        S1 = [0.0] * (W * H * K)
        SN["_aggregate_path"](C, base, W, H, K, 12.0, 150.0, dx, dy, S1)
        out["path%d_R10" % i] = as_int_array(S1, np.uint8)
    S = [0.0] * (W * H * K)
    for dx, dy in dirs:
        SN["_aggregate_path"](C, base, W, H, K, 12.0, 150.0, dx, dy, S)
    out["S_R10"] = as_int_array(S, np.uint16)
    o, conf = SN["refine_fullres"](L, R, d0l, W, H, R=10, P1=12.0, P2=150.0, rx=4, ry=3,
                                  return_conf=True)
    out["refine_R10"] = np.array(o)
    out["conf_R10"] = np.array(conf)
    out["refine_default"] = np.array(SN["refine_fullres"](L, R, d0l, W, H))
    out["refine_R4_paths4"] = np.array(SN["refine_fullres"](L, R, d0l, W, H, R=4, P1=12.0,
                                                            P2=150.0, paths=4, rx=4, ry=3))
    out["refine_uniq"] = np.array(SN["refine_fullres"](L, R, d0l, W, H, R=6, P1=8.0,
                                                       P2=96.0, rx=3, ry=3, uniq=0.15))
    out["l2r"] = np.array(SN["left_to_right"](d0l, W, H))
    lo, st = SN["lr_refine"](L, R, d0l, W, H, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4, ry=3)
    out["lr_out"] = np.array(lo)
    out["lr_status"] = np.array(st, dtype=np.int8)
    lo1, st1 = SN["lr_refine"](L, R, d0l, W, H)
    out["lr_default_out"] = np.array(lo1)
    out["lr_default_status"] = np.array(st1, dtype=np.int8)
    # full-range mode (eval_real.py:143-146): disp0 == R everywhere
    Rf = int(np.max(pair.disp) + 2) // 2 + 1
    out["fullrange_R"] = np.array([Rf])
    out["fullrange"] = np.array(SN["refine_fullres"](L, R, [float(Rf)] * (W * H), W, H, R=Rf,
                                                     P1=12.0, P2=150.0, rx=4, ry=3))
    np.savez_compressed(os.path.join(HERE, "refine_small.npz"), **out)
    print("refine_small done (%.1fs)" % (time.time() - t0))

    # --------------------------------------------------------- network, small
    npair = synth.make_pair(21, 64, 48, 2.0, 24.0, n_planes=(2, 3))
    Wn, Hn = npair.W, npair.H
    Ln = list(npair.gray("left").ravel())
    Rn = list(npair.gray("right").ravel())
    gh, _, _ = SN["avgpool2"](Ln, 1, Hn, Wn)
    f0, f1, f2 = net.forward(Ln, Rn, Hn, Wn, gh, Ln)
    ps = SN["predict_at_scale"](net, Ln, Rn, Wn, Hn, 48, False)
    np.savez_compressed(os.path.join(HERE, "network_small.npz"), left=npair.left,
                        right=npair.right, d0=np.array(f0), d1=np.array(f1), d2=np.array(f2),
                        pas_full=np.array(ps[0]), pas_work=np.array(ps[1]),
                        pas_dims=np.array([ps[2], ps[3]]))
    print("network_small done (%.1fs)" % (time.time() - t0))

    # ------------------------------------ the 160x120 workload, end to end
    p1 = synth.config_small()
    L1 = list(p1.gray("left").ravel())
    R1 = list(p1.gray("right").ravel())
    df, dw, Ww, Hw = SN["predict_auto"](net, L1, R1, p1.W, p1.H, verbose=False)
    ro, rst = SN["lr_refine"](L1, R1, df, p1.W, p1.H, tol=2.0, R=10, P1=12.0, P2=150.0,
                              rx=4, ry=3)
    np.savez_compressed(os.path.join(HERE, "config_small.npz"), left=p1.left, right=p1.right,
                        disp0=np.array(df), disp_work=np.array(dw), dims=np.array([Ww, Hw]),
                        out=np.array(ro), status=np.array(rst, dtype=np.int8))
    print("config_small done: work %dx%d (%.1fs)" % (Ww, Hw, time.time() - t0))

    # ------------------------------------ the 450x375 workload, as digests
    p2 = synth.config_full()
    L2 = list(p2.gray("left").ravel())
    R2 = list(p2.gray("right").ravel())
    df2, dw2, Ww2, Hw2 = SN["predict_auto"](net, L2, R2, p2.W, p2.H, verbose=False)
    ro2, rst2 = SN["lr_refine"](L2, R2, df2, p2.W, p2.H, tol=2.0, R=10, P1=12.0, P2=150.0,
                                rx=4, ry=3)
    meta["config_full"] = {
        "W": p2.W, "H": p2.H, "images_sha256": sha(np.concatenate([p2.left.ravel(),
                                                                   p2.right.ravel()]),
                                                   np.uint8),
        "work": [Ww2, Hw2], "disp0_sha256": sha(df2), "disp_work_sha256": sha(dw2),
        "out_sha256": sha(ro2), "status_sha256": sha(rst2, np.int8),
        "status_counts": [int(np.sum(np.array(rst2) == s)) for s in (0, 1, 2)],
        "disp0_mean": float(np.mean(df2)), "out_mean": float(np.mean(ro2)),
    }
    print("config_full done: work %dx%d (%.1fs)" % (Ww2, Hw2, time.time() - t0))
    with open(os.path.join(HERE, "golden_meta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("all fixtures written (%.1fs)" % (time.time() - t0))


def pseudo_rgb(pair):
    """A deterministic colour image for the plane_snap / SLIC inputs
    (interleaved RGB in [0, 1], as read_image gives): the left gray level
    and two smooth transforms of it."""
    g = pair.left.astype(np.float64) / 255.0
    h, w = g.shape
    yy, xx = np.mgrid[0:h, 0:w]
    rgb = np.stack([g, 0.5 * g + 0.5 * (xx / max(1, w - 1)), 1.0 - 0.7 * g * (yy / max(1, h - 1))],
                   axis=-1)
    return np.round(rgb * 255.0) / 255.0


def postproc(ref_dir):
    """The rest of refine_disparity (stereonet.py:5865-5883): SLIC, plane_snap,
    median_filter and refine_disparity itself, on small seeded pairs."""
    SN = load_reference(ref_dir)
    out = {}
    for tag, (W, H, seed, step) in {"a": (64, 48, 31, 12), "b": (90, 70, 32, 8)}.items():
        p = synth.make_pair(seed, W, H, 2.0, 24.0, n_planes=(3, 5))
        L = list(p.gray("left").ravel())
        R = list(p.gray("right").ravel())
        rgb = pseudo_rgb(p)
        rl = list(rgb.ravel())
        rng = np.random.default_rng(seed)
        d0 = list(p.disp.ravel() + rng.uniform(-2.5, 2.5, W * H))
        d, st = SN["lr_refine"](L, R, d0, W, H, tol=2.0, R=10, P1=12.0, P2=150.0, rx=4, ry=3)
        valid = [s == 0 for s in st]
        lab, nseg = SN["slic"](rl, W, H, step)
        out[tag + "_left"], out[tag + "_right"] = p.left, p.right
        out[tag + "_rgb"], out[tag + "_disp0"] = rgb.ravel(), np.array(d0)
        out[tag + "_lr"], out[tag + "_status"] = np.array(d), np.array(st, dtype=np.int8)
        out[tag + "_slic"] = np.array(lab, dtype=np.int32)
        out[tag + "_slic_c20_it3"] = np.array(SN["slic"](rl, W, H, step, 20.0, 3)[0], dtype=np.int32)
        out[tag + "_snap"] = np.array(SN["plane_snap"](d, rl, W, H, valid=valid, step=step,
                                                       thr=1.0, min_inl=0.4))
        out[tag + "_snap_novalid"] = np.array(SN["plane_snap"](d, rl, W, H, step=step))
        out[tag + "_median"] = np.array(SN["median_filter"](d, W, H))
        out[tag + "_median_r2p2"] = np.array(SN["median_filter"](d, W, H, radius=2, passes=2))
        rd, rs = SN["refine_disparity"](L, R, rl, d0, W, H, plane_step=step)
        out[tag + "_refine_disparity"] = np.array(rd)
        out[tag + "_refine_disparity_status"] = np.array(rs, dtype=np.int8)
        rd2, _ = SN["refine_disparity"](L, R, rl, d0, W, H, planes=False)
        out[tag + "_refine_disparity_noplanes"] = np.array(rd2)
        out[tag + "_dims"] = np.array([W, H, step])
    # An 11x17 binary image where some pixels lie in no cluster window in
    # SLIC iterations 3 and 4 (they keep their labels): found by a seeded
    # search, regenerated here from its seed.
    rng = np.random.default_rng(0)
    for trial in range(111):
        W, H, step = (int(rng.integers(8, 40)), int(rng.integers(8, 40)), int(rng.integers(3, 12)))
        img = rng.random((H, W, 3))
        if trial % 3 == 1:
            img[:, :W // 2] = 0.0
            img[:, W // 2:] = 1.0
        if trial % 3 == 2:
            img = (rng.random((H, W, 1)) > 0.5) * np.ones((1, 1, 3))
        comp = float(rng.choice([0.1, 1.0, 10.0]))
    rgb = (np.round(img * 255) / 255.0).ravel()
    d = np.random.default_rng(7).uniform(0, 20, W * H)
    out["u_rgb"], out["u_disp"], out["u_dims"] = rgb, d, np.array([W, H, step])
    out["u_comp"] = np.array(comp)
    out["u_slic"] = np.array(SN["slic"](list(rgb), W, H, step, comp)[0], dtype=np.int32)
    out["u_snap"] = np.array(SN["plane_snap"](list(d), list(rgb), W, H, step=step, thr=5.0,
                                              min_inl=0.3))
    # network-level left-right consistency (stereonet.py:4974-5076)
    net = SN["load_model"](os.path.join(ref_dir, "stereonet_weights.txt"))
    for tag, (W, H, seed, ww) in {"c": (112, 80, 41, None), "d": (96, 72, 42, 64)}.items():
        p = synth.make_pair(seed, W, H, 2.0, 30.0, n_planes=(3, 5))
        L, R = list(p.gray("left").ravel()), list(p.gray("right").ravel())
        dc, frac = SN["predict_consistent"](net, L, R, W, H, work_width=ww, verbose=False)
        out[tag + "_left"], out[tag + "_right"] = p.left, p.right
        out[tag + "_consistent"], out[tag + "_frac"] = np.array(dc), np.array(frac)
        out[tag + "_dims"] = np.array([W, H, 0 if ww is None else ww])
        rng = np.random.default_rng(seed)
        dl = list(p.disp.ravel() + rng.normal(0, 1.0, W * H))
        dr = list(rng.uniform(0, 30, W * H))
        v = SN["lr_consistency"](dl, dr, W, H, 1.5)
        out[tag + "_lrc_in"] = np.array([dl, dr])
        out[tag + "_lrc"] = np.array(v)
        out[tag + "_fill"] = np.array(SN["fill_invalid"](dl, v, W, H))
    np.savez_compressed(os.path.join(HERE, "postproc.npz"), **out)
    print("postproc fixtures written")


# ------------------------------------------------------------------ images
def image_cases():
    """(name, file bytes) of every decoded case, and of the error cases."""
    import zlib
    make_png = synth.make_png
    rng = np.random.default_rng(8086)

    def noise(W, H, ch, hi):
        return rng.integers(0, hi + 1, size=(H, W * ch)).tolist()

    def smooth(W, H, ch, hi):
        yy, xx = np.mgrid[0:H, 0:W * ch]
        v = (np.sin(xx / 7.0) + np.cos(yy / 5.0) + 2) / 4 * hi
        v = v + rng.integers(0, 3, size=v.shape)
        return np.clip(v, 0, hi).astype(int).tolist()

    ok = []
    F = (0, 1, 2, 3, 4)
    ok.append(("rgb8_dyn", make_png(37, 23, 8, 2, noise(37, 23, 3, 255), F, 9)[0]))
    ok.append(("gray8_rle", make_png(40, 30, 8, 0, smooth(40, 30, 1, 255), (4,), 6,
                                     zlib.Z_RLE)[0]))
    ok.append(("rgb16_fixed", make_png(21, 13, 16, 2, noise(21, 13, 3, 65535), F, 6,
                                       zlib.Z_FIXED)[0]))
    ok.append(("gray16_stored", make_png(19, 11, 16, 0, noise(19, 11, 1, 65535), (2, 1), 0)[0]))
    ok.append(("ga8", make_png(17, 9, 8, 4, noise(17, 9, 2, 255), F, 6)[0]))
    ok.append(("rgba8_huff", make_png(23, 15, 8, 6, noise(23, 15, 4, 255), (3,), 6,
                                      zlib.Z_HUFFMAN_ONLY)[0]))
    ok.append(("rgba16", make_png(9, 7, 16, 6, noise(9, 7, 4, 65535), F, 9)[0]))
    ok.append(("ga16", make_png(11, 5, 16, 4, noise(11, 5, 2, 65535), (4, 3), 9)[0]))
    for d, W, H in ((1, 29, 7), (2, 27, 9), (4, 13, 11)):
        ok.append(("gray%d" % d, make_png(W, H, d, 0, noise(W, H, 1, (1 << d) - 1), F, 9)[0]))
    for d, W, H, n in ((1, 21, 6, 2), (2, 19, 7, 4), (4, 15, 9, 16), (8, 33, 12, 200)):
        pal = rng.integers(0, 256, size=3 * n).tolist()
        ok.append(("pal%d" % d, make_png(W, H, d, 3, noise(W, H, 1, n - 1), F, 9,
                                         palette=pal)[0]))
    ok.append(("rgb8_smooth_split", make_png(96, 64, 8, 2, smooth(96, 64, 3, 255), F, 9,
                                             idat_parts=3, extra=True)[0]))
    ok.append(("gray8_stored_multi", make_png(300, 230, 8, 0, smooth(300, 230, 1, 255),
                                              (0,), 0)[0]))

    def pnm(magic, W, H, maxval, vals, comment=True, sep=b" "):
        hdr = magic + b"\n" + (b"# golden fixture\n" if comment else b"")
        hdr += b"%d %d\n%d\n" % (W, H, maxval)
        if magic in (b"P2", b"P3"):
            body = b""
            for i, v in enumerate(vals):
                body += b"%d" % v + (b"\n" if i % 11 == 10 else sep)
            return hdr + body
        if maxval < 256:
            return hdr + bytes(vals)
        return hdr + b"".join(int(v).to_bytes(2, "big") for v in vals)

    def flat(W, H, ch, hi):
        return rng.integers(0, hi + 1, size=W * H * ch).tolist()

    ok.append(("p5_8", pnm(b"P5", 25, 20, 255, flat(25, 20, 1, 255))))
    ok.append(("p5_16", pnm(b"P5", 17, 13, 65535, flat(17, 13, 1, 65535), comment=False)))
    ok.append(("p5_1000", pnm(b"P5", 12, 9, 1000, flat(12, 9, 1, 1000))))
    ok.append(("p6_8", pnm(b"P6", 19, 11, 255, flat(19, 11, 3, 255))))
    ok.append(("p6_100", pnm(b"P6", 14, 8, 100, flat(14, 8, 3, 100))))
    ok.append(("p6_4095", pnm(b"P6", 9, 6, 4095, flat(9, 6, 3, 4095))))
    ok.append(("p2_15", pnm(b"P2", 13, 7, 15, flat(13, 7, 1, 15), sep=b"\t ")))
    ok.append(("p3_255", pnm(b"P3", 8, 5, 255, flat(8, 5, 3, 255), sep=b"\r\n")))
    ok.append(("p2_65535", pnm(b"P2", 6, 4, 65535, flat(6, 4, 1, 65535))))

    err = []
    base, raw = make_png(8, 4, 8, 0, noise(8, 4, 1, 255), (0,), 9)
    good = zlib.compress(raw, 9)
    err.append(("interlaced", make_png(8, 4, 8, 0, noise(8, 4, 1, 255), interlace=1)[0]))
    err.append(("depth3", make_png(8, 4, 8, 0, noise(8, 4, 1, 255))[0].replace(
        b"IHDR" + (8).to_bytes(4, "big") + (4).to_bytes(4, "big") + bytes([8, 0]),
        b"IHDR" + (8).to_bytes(4, "big") + (4).to_bytes(4, "big") + bytes([3, 0]))))
    err.append(("colortype5", make_png(8, 4, 8, 0, noise(8, 4, 1, 255))[0].replace(
        b"IHDR" + (8).to_bytes(4, "big") + (4).to_bytes(4, "big") + bytes([8, 0]),
        b"IHDR" + (8).to_bytes(4, "big") + (4).to_bytes(4, "big") + bytes([8, 5]))))
    err.append(("zlib_method", make_png(8, 4, 8, 0, noise(8, 4, 1, 255),
                                        zlib_stream=bytes([0x77, 0x01]) + good[2:])[0]))
    err.append(("zlib_check", make_png(8, 4, 8, 0, noise(8, 4, 1, 255),
                                       zlib_stream=bytes([0x78, 0x02]) + good[2:])[0]))
    err.append(("zlib_dict", make_png(8, 4, 8, 0, noise(8, 4, 1, 255),
                                      zlib_stream=bytes([0x78, 0xBB]) + good[2:])[0]))
    bad_filter = bytearray(raw)
    bad_filter[9] = 5                           # second row's filter byte
    err.append(("filter5", make_png(8, 4, 8, 0, noise(8, 4, 1, 255),
                                    zlib_stream=zlib.compress(bytes(bad_filter), 9))[0]))
    err.append(("btype3", make_png(8, 4, 8, 0, noise(8, 4, 1, 255),
                                   zlib_stream=bytes([0x78, 0x01, 0x07]) + bytes(40))[0]))
    stored = zlib.compress(raw, 0)
    bad_len = bytearray(stored)
    bad_len[5] ^= 0xFF                          # NLEN no longer the complement
    err.append(("stored_len", make_png(8, 4, 8, 0, noise(8, 4, 1, 255),
                                       zlib_stream=bytes(bad_len))[0]))
    # fixed block whose first code is a length/distance pair (distance 1
    # with empty output): literal/length 257 = 7-bit code 0000001
    err.append(("backref", make_png(8, 4, 8, 0, noise(8, 4, 1, 255),
                                    zlib_stream=bytes([0x78, 0x01, 0x03, 0x02, 0x00, 0x00]))[0]))
    err.append(("not_png_magic", b"P4\n8 4\n" + bytes(4)))
    return ok, err


def images(ref_dir):
    """read_png / read_pnm / read_image of the reference on every case."""
    import shutil
    import tempfile
    SN = load_reference(ref_dir)
    ok, err = image_cases()
    tmp = tempfile.mkdtemp(dir=HERE)
    out = {}
    errors = {}
    try:
        for name, data in ok:
            path = os.path.join(tmp, name)
            with open(path, "wb") as f:
                f.write(data)
            g, c, W, H = SN["read_image"](path)
            out[name + "_file"] = np.frombuffer(data, dtype=np.uint8)
            out[name + "_wh"] = np.array([W, H])
            if W * H > 2000:                    # large: digests of the FP64 bytes
                out[name + "_gray_sha"] = np.array(sha(g))
                out[name + "_rgb_sha"] = np.array(sha(c))
            else:
                out[name + "_gray"] = np.asarray(g, dtype=np.float64)
                out[name + "_rgb"] = np.asarray(c, dtype=np.float64)
        for name, data in err:
            path = os.path.join(tmp, name)
            with open(path, "wb") as f:
                f.write(data)
            try:
                SN["read_image"](path)
                kind = "none"
            except Exception as e:          # the reference's own exception type
                kind = type(e).__name__
            out["err_" + name + "_file"] = np.frombuffer(data, dtype=np.uint8)
            errors[name] = kind
    finally:
        shutil.rmtree(tmp)
    out["err_kinds"] = np.array(json.dumps(errors, sort_keys=True))
    np.savez_compressed(os.path.join(HERE, "images.npz"), **out)
    print("image fixtures written:", len(ok), "decoded,", errors)


# ---------------------------------------------------------------- training
def training(ref_dir):
    """train_grads (stereonet.py:1619-1653) and two Adam steps of the
    reference on seeded 48x32 crops with its own checkpoint."""
    t0 = time.time()
    SN = load_reference(ref_dir)
    net = SN["load_model"](os.path.join(ref_dir, "stereonet_weights.txt"))
    out = {"params0": np.array(SN["flat_params"](net))}
    opt = SN["Adam"](net.all_params(), lr=1.0e-3)
    for k, (seed, dmax) in enumerate(((61, 20.0), (62, 34.0))):
        pair = synth.make_pair(seed, 48, 32, 2.0, dmax, n_planes=(2, 3))
        W, H = pair.W, pair.H
        sample = {"left": list(pair.gray("left").ravel()),
                  "right": list(pair.gray("right").ravel()),
                  "disp": [float(v) for v in pair.disp.ravel()],
                  "valid": [bool(v) for v in pair.valid.ravel()], "W": W, "H": H}
        total, pred, tgt = SN["train_grads"](net, sample)
        out["s%d_left" % k] = pair.left
        out["s%d_right" % k] = pair.right
        out["s%d_disp" % k] = pair.disp
        out["s%d_valid" % k] = pair.valid
        out["s%d_loss" % k] = np.array([total])
        out["s%d_grads" % k] = np.array(SN["flat_grads"](net))
        out["s%d_d2" % k] = np.array(pred)
        opt.step()
        out["s%d_params_after" % k] = np.array(SN["flat_params"](net))
        print("training sample %d: loss %.6f (%.1fs)" % (k, total, time.time() - t0))
    np.savez_compressed(os.path.join(HERE, "training.npz"), **out)
    print("training fixtures written")


HOT_PATH = ["census", "band_costs", "_aggregate_path", "refine_fullres", "left_to_right",
            "lr_refine", "resize_gray", "avgpool2", "predict", "predict_at_scale",
            "predict_auto", "refine_disparity", "median_filter", "slic", "plane_snap",
            "predict_consistent", "lr_consistency", "fill_invalid", "read_png", "read_pnm",
            "read_image", "train_grads", "train_step", "_peak"]


def signatures(ref_dir):
    """The reference's signatures of the hot-path functions (and
    StereoNet.forward), which the drop-ins must keep."""
    import inspect
    SN = load_reference(ref_dir)
    sig = {n: str(inspect.signature(SN[n])) for n in HOT_PATH}
    sig["StereoNet.forward"] = str(inspect.signature(SN["StereoNet"].forward))
    with open(os.path.join(HERE, "signatures.json"), "w") as f:
        json.dump(sig, f, indent=1, sort_keys=True)
    print("signatures written")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref = args[0] if args else os.environ.get("SV_REFERENCE_DIR")
    if not ref or not os.path.isfile(os.path.join(ref, "stereonet.py")):
        sys.exit("usage: make_golden.py <reference checkout> [--...-only] "
                 "(or set SV_REFERENCE_DIR)")
    if "--postproc-only" in sys.argv:
        postproc(ref)
    elif "--images-only" in sys.argv:
        images(ref)
    elif "--training-only" in sys.argv:
        training(ref)
    elif "--signatures-only" not in sys.argv:
        main(ref)
        postproc(ref)
        images(ref)
        training(ref)
    signatures(ref)
