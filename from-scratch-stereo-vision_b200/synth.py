"""Seeded synthetic rectified stereo pairs with exact left-view disparity.

The scenes are modelled on the reference's random-dot stereograms
(``make_stereogram``, stereonet.py:1435-1565) and its z-buffered forward warp
(``_warp_to_right``, stereonet.py:3658-3712): a slanted background plane,
slanted planar foreground rectangles at larger disparity, and a right view in
which the nearer surface (larger disparity) wins where two surfaces land on
the same column.  Differences, all deliberate:

* texture is uniform noise blurred by a Gaussian of sigma 1.0, per surface;
* the warp is exact for fractional disparity: every surface is solved in
  closed form for the left-image column it shows at each right-image pixel,
  and its texture is sampled there by linear interpolation, so pixels that
  only the right camera sees show the hidden surface's own (fresh) texture
  instead of a stretched neighbour;
* images are quantised to uint8 (the network and the oracle see u/255.0).

Everything is driven by one ``numpy.random.Generator`` seeded per pair, so a
(seed, shape, config) triple always gives the same bytes.
"""

from __future__ import annotations

import dataclasses

import numpy as np


def _gauss_kernel(sigma: float) -> np.ndarray:
    r = max(1, int(np.ceil(3.0 * sigma)))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    return k / k.sum()


def _blur(img: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian blur with reflected borders."""
    k = _gauss_kernel(sigma)
    r = len(k) // 2
    p = np.pad(img, ((r, r), (r, r)), mode="reflect")
    tmp = np.zeros((p.shape[0], img.shape[1]))
    for i, w in enumerate(k):
        tmp += w * p[:, i:i + img.shape[1]]
    out = np.zeros(img.shape)
    for i, w in enumerate(k):
        out += w * tmp[i:i + img.shape[0], :]
    return out


@dataclasses.dataclass
class _Surface:
    # disparity d(x, y) = a + bx * x + cy * y in left-image pixel coordinates
    a: float
    bx: float
    cy: float
    # left-image footprint, half-open pixel rectangle [x0, x1) x [y0, y1)
    x0: float
    y0: float
    x1: float
    y1: float
    tex: np.ndarray          # texture rows over left columns [tx0, tx0 + tw)
    amp: np.ndarray          # texture amplitude per texel (0.1x inside low-texture patches)
    tx0: int

    def disp(self, x, y):
        return self.a + self.bx * x + self.cy * y

    def covers(self, x, y):
        return (x >= self.x0 - 0.5) & (x < self.x1 - 0.5) & \
               (y >= self.y0) & (y < self.y1)


def _make_texture(rng, H, tw, mean, amp, lowtex_patches=()):
    noise = rng.random((H, tw))
    t = _blur(noise, 1.0)
    t = (t - t.mean()) / (t.std() + 1e-12)
    scale = np.full((H, tw), amp)
    for (py0, py1, px0, px1) in lowtex_patches:
        scale[py0:py1, px0:px1] *= 0.1
    return mean + scale * t * 0.5, scale


@dataclasses.dataclass
class StereoPair:
    left: np.ndarray      # uint8 [H, W]
    right: np.ndarray     # uint8 [H, W]
    disp: np.ndarray      # float64 [H, W], left-view ground truth in pixels
    valid: np.ndarray     # bool [H, W], False where the left pixel is unseen on the right
    lowtex: np.ndarray    # bool [H, W], left pixels on low-texture regions
    seed: int

    @property
    def W(self) -> int:
        return self.left.shape[1]

    @property
    def H(self) -> int:
        return self.left.shape[0]

    def gray(self, which: str = "left") -> np.ndarray:
        """The reference's float gray in [0, 1] (u / 255.0, FP64)."""
        return getattr(self, which).astype(np.float64) / 255.0


def make_pair(seed: int, W: int, H: int, d_min: float, d_max: float,
              n_planes=(3, 6), lowtex_frac: float = 0.0,
              occl_target: float | None = None, bars: int = 0,
              bar_width=(2, 6)) -> StereoPair:
    """One seeded pair.

    ``n_planes`` is an inclusive range for the number of slanted foreground
    rectangles, ``lowtex_frac`` the target share of image area whose texture
    amplitude is scaled by 0.1, ``bars`` the number of thin vertical
    foreground bars (``bar_width`` px wide, inclusive range).
    ``occl_target`` steers object size so that roughly that share of left
    pixels is occluded in the right view (it is reported, not enforced).
    """
    rng = np.random.default_rng(seed)
    span = d_max - d_min
    tw = W + int(np.ceil(d_max)) + 8          # texture reaches every column a right pixel can see
    tx0 = -4

    def lowtex_patches(hh, ww, frac):
        pts = []
        if frac <= 0:
            return pts
        area = 0.0
        while area < frac * hh * ww:
            ph = int(rng.integers(max(4, hh // 8), max(5, hh // 3)))
            pw = int(rng.integers(max(4, ww // 8), max(5, ww // 3)))
            py = int(rng.integers(0, max(1, hh - ph)))
            px = int(rng.integers(0, max(1, ww - pw)))
            pts.append((py, py + ph, px, px + pw))
            area += ph * pw
        return pts

    surfaces = []
    # background: a plane slanted in y (far at the top, nearer at the bottom)
    b_far = d_min + rng.uniform(0.0, 0.15) * span
    b_near = b_far + rng.uniform(0.05, 0.25) * span
    cy = (b_near - b_far) / max(1, H - 1)
    bx = rng.uniform(-0.02, 0.02) * span / max(1, W)
    mean = rng.uniform(0.35, 0.65)
    base_amp = rng.uniform(0.35, 0.6)
    tex, amp = _make_texture(rng, H, tw, mean, base_amp,
                             lowtex_patches(H, tw, lowtex_frac))
    surfaces.append(_Surface(b_far, bx, cy, -1e9, 0, 1e9, H, tex, amp, tx0))

    n_obj = int(rng.integers(n_planes[0], n_planes[1] + 1))
    size_hi = 0.5 if occl_target is None else float(np.clip(0.25 + 1.5 * occl_target, 0.3, 0.6))
    for _ in range(n_obj):
        ow = int(rng.integers(max(6, W // 8), max(7, int(W * size_hi))))
        oh = int(rng.integers(max(6, H // 8), max(7, int(H * size_hi))))
        ox = int(rng.integers(0, max(1, W - ow)))
        oy = int(rng.integers(0, max(1, H - oh)))
        dc = d_min + rng.uniform(0.35, 1.0) * span
        sx = rng.uniform(-0.08, 0.08) * min(1.0, span / max(1.0, ow))
        sy = rng.uniform(-0.08, 0.08) * min(1.0, span / max(1.0, oh))
        cx, cyy = ox + ow / 2.0, oy + oh / 2.0
        a = dc - sx * cx - sy * cyy
        low = rng.random() < lowtex_frac
        amp = rng.uniform(0.35, 0.6) * (0.1 if low else 1.0)
        tex, ampm = _make_texture(rng, H, tw, rng.uniform(0.2, 0.8), amp)
        surfaces.append(_Surface(a, sx, sy, ox, oy, ox + ow, oy + oh, tex, ampm, tx0))
    for _ in range(bars):
        bw = int(rng.integers(bar_width[0], bar_width[1] + 1))
        bh = int(rng.integers(H // 3, H + 1))
        bxp = int(rng.integers(0, max(1, W - bw)))
        byp = int(rng.integers(0, max(1, H - bh + 1)))
        dc = d_min + rng.uniform(0.8, 1.0) * span
        tex, ampm = _make_texture(rng, H, tw, rng.uniform(0.15, 0.85), rng.uniform(0.4, 0.6))
        surfaces.append(_Surface(dc, 0.0, 0.0, bxp, byp, bxp + bw, byp + bh, tex, ampm, tx0))

    ys, xs = np.mgrid[0:H, 0:W]
    ys = ys.ravel()
    xs = xs.ravel().astype(np.float64)

    def render(view_x, solve):
        best_d = np.full(W * H, -np.inf)
        val = np.zeros(W * H)
        amp = np.zeros(W * H)
        for s in surfaces:
            if solve:
                # right pixel xr shows left column x with x - d(x, y) = xr
                x = (view_x + s.a + s.cy * ys) / (1.0 - s.bx)
            else:
                x = view_x
            d = s.disp(x, ys)
            m = s.covers(x, ys) & (d > best_d)
            if not m.any():
                continue
            best_d[m] = d[m]
            u = np.clip(x[m] - s.tx0, 0.0, s.tex.shape[1] - 1.000001)
            i = np.floor(u).astype(np.int64)
            f = u - i
            yy = ys[m]
            val[m] = s.tex[yy, i] * (1.0 - f) + s.tex[yy, i + 1] * f
            amp[m] = s.amp[yy, i]
        return best_d, val, amp

    dl, vl, al = render(xs, solve=False)
    dr, vr, _ = render(xs, solve=True)
    to_u8 = lambda v: np.clip(np.rint(v * 255.0), 0, 255).astype(np.uint8)
    left = to_u8(vl).reshape(H, W)
    right = to_u8(vr).reshape(H, W)
    disp = dl.reshape(H, W)
    # a left pixel is valid when it lands inside the right image and the
    # surface seen there is not nearer than it by more than half a pixel
    xr = np.rint(xs - dl).astype(np.int64)
    inside = (xr >= 0) & (xr < W)
    seen = np.full(W * H, False)
    idx = np.where(inside)[0]
    seen[idx] = dr[ys[idx] * W + xr[idx]] <= dl[idx] + 0.5
    valid = seen.reshape(H, W)
    lowtex = (al < 0.1).reshape(H, W)
    return StereoPair(left, right, disp, valid, lowtex, seed)


# --------------------------------------------------------------------------
# The five workloads.  Each returns a list of pairs (or one pair).
# --------------------------------------------------------------------------

def config_small(seed: int = 1) -> StereoPair:
    """160x120, 3-6 slanted planes at disparities 2-30 px."""
    return make_pair(seed, 160, 120, 2.0, 30.0, n_planes=(3, 6))


def config_full(seed: int = 2) -> StereoPair:
    """450x375, 8-15 planes at 0-80 px, ~10% occluded, ~20% low texture."""
    return make_pair(seed, 450, 375, 0.0, 80.0, n_planes=(8, 15),
                     lowtex_frac=0.2, occl_target=0.10)


def config_batched(n: int = 256, seed: int = 3, size_lo=(200, 150),
                   size_hi=(1400, 1100), disp_lo=10.0, disp_hi=200.0):
    """``n`` pairs of uneven sizes and disparity ranges, per-pair seeds."""
    rng = np.random.default_rng(seed)
    pairs = []
    for i in range(n):
        W = int(rng.integers(size_lo[0], size_hi[0] + 1))
        H = int(rng.integers(size_lo[1], size_hi[1] + 1))
        dmax = float(rng.uniform(disp_lo, disp_hi))
        dmax = min(dmax, 0.6 * W)
        pairs.append(make_pair(seed * 100003 + i, W, H, 0.0, dmax,
                               n_planes=(3, 10), lowtex_frac=0.1))
    return pairs


def config_precision(n: int = 64, seed: int = 4):
    """``n`` pairs of 640x480 at disparities 0-120 px."""
    return [make_pair(seed * 100003 + i, 640, 480, 0.0, 120.0, n_planes=(4, 10),
                      lowtex_frac=0.1) for i in range(n)]


def config_learned_crop(seed: int, W: int = 256, H: int = 192) -> StereoPair:
    """Training crop: 30-150 px, thin 2-6 px bars, 30% low texture."""
    rng = np.random.default_rng(seed)
    return make_pair(seed, W, H, 30.0, 150.0, n_planes=(2, 5),
                     lowtex_frac=0.3, bars=int(rng.integers(1, 4)))


# ------------------------------------------------------- file formats
def _png_chunk(tag: bytes, body: bytes) -> bytes:
    import zlib
    return (len(body).to_bytes(4, "big") + tag + body +
            (zlib.crc32(tag + body) & 0xFFFFFFFF).to_bytes(4, "big"))


def _filter_rows(rows, bpp, filters):
    """PNG row filters 0-4 applied forward (PNG 1.2 section 6)."""
    out = bytearray()
    prev = bytes(len(rows[0]))
    for y, row in enumerate(rows):
        ft = filters[y % len(filters)]
        out.append(ft)
        for i, x in enumerate(row):
            a = row[i - bpp] if i >= bpp else 0
            b = prev[i] if y > 0 else 0
            c = prev[i - bpp] if (y > 0 and i >= bpp) else 0
            if ft == 0:
                pr = 0
            elif ft == 1:
                pr = a
            elif ft == 2:
                pr = b
            elif ft == 3:
                pr = (a + b) >> 1
            else:
                p = a + b - c
                pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                pr = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            out.append((x - pr) & 0xFF)
        prev = row
    return bytes(out)


def make_png(W, H, depth, ct, samples, filters=(0,), level=9, strategy=0, palette=None,
             idat_parts=1, extra=False, interlace=0, zlib_stream=None):
    """A PNG of `samples` ([H][W*channels] ints) encoded with Python's zlib."""
    import zlib
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ct]
    rows = []
    for y in range(H):
        vals = samples[y]
        if depth == 16:
            r = b"".join(int(v).to_bytes(2, "big") for v in vals)
        elif depth == 8:
            r = bytes(int(v) for v in vals)
        else:
            bits = 0
            r = bytearray((W * depth + 7) // 8)
            for v in vals:
                r[bits >> 3] |= int(v) << (8 - depth - (bits & 7))
                bits += depth
            r = bytes(r)
        rows.append(r)
    raw = _filter_rows(rows, max(1, ch * depth // 8), list(filters))
    if zlib_stream is None:
        co = zlib.compressobj(level, zlib.DEFLATED, 15, 9, strategy)
        zlib_stream = co.compress(raw) + co.flush()
    ihdr = W.to_bytes(4, "big") + H.to_bytes(4, "big") + bytes([depth, ct, 0, 0, interlace])
    out = b"\x89PNG\r\n\x1a\n" + _png_chunk(b"IHDR", ihdr)
    if extra:
        out += _png_chunk(b"tEXt", b"Comment\x00golden fixture")
    if palette is not None:
        out += _png_chunk(b"PLTE", bytes(palette))
    step = (len(zlib_stream) + idat_parts - 1) // idat_parts
    for k in range(idat_parts):
        out += _png_chunk(b"IDAT", zlib_stream[k * step:(k + 1) * step])
    out += _png_chunk(b"IEND", b"")
    if extra:
        out += b"trailing bytes after IEND"
    return out, raw
