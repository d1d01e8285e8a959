/*
 * sv_band_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 definition of the learned adaptive band, the checker for its CUDA
 * kernels.  The band predictor has no counterpart in the reference; its
 * building blocks follow the reference's own layers:
 *   Conv2d.forward / backward   stereonet.py:489-570
 *   LeakyReLU forward/backward  stereonet.py:698-723
 *   Adam.step                   stereonet.py:1354-1387
 * and the masked refinement reuses this oracle's census / band_costs /
 * aggregate_path / left_to_right restatements (sv_oracle.c).
 *
 * Band net: 4 convolutions 3x3, BAND_F -> 16 -> 16 -> 16 -> 2, dilations
 * 1, 2, 4, 1, same padding, leaky ReLU 0.2 after the first three.  Output
 * channel 0 is the band-centre shift s = 32 * o0 (px), channel 1 the log of
 * a Laplace scale rho = o1 + 1 (b = exp(clamp(rho)) px).
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_EBADARG 1
#define ORC_ENOMEM 2
#define ORC_ERANGE 3

#define BAND_F 8               /* net inputs: the 6 features below + 2 given planes */
#define BAND_C 16
#define BAND_O 2
#define BAND_L 4
#define BAND_INVALID 66        /* 62 census bits + 4, the pipeline's invalid cost */
#define BAND_ROWS 4            /* vertical aggregation half-height: 9 rows */
#define BAND_SHIFT_SCALE 32.0
#define BAND_RHO0 1.0
#define BAND_RHO_MIN (-1.3862943611198906)   /* log(0.25) */
#define BAND_RHO_MAX 4.852030263919617       /* log(128) */

static const int band_ic[BAND_L] = {BAND_F, BAND_C, BAND_C, BAND_C};
static const int band_oc[BAND_L] = {BAND_C, BAND_C, BAND_C, BAND_O};
static const int band_dil[BAND_L] = {1, 2, 4, 1};

long orc_band_param_count(void) {
    long n = 0;
    for (int l = 0; l < BAND_L; l++) n += (long)band_oc[l] * band_ic[l] * 9 + band_oc[l];
    return n;
}

/* ---------------------------------------------------------------- features
 * Per pixel, from the 9x7 census words of both views and the network
 * disparity d0, with agg(d) = sum over the 9 rows y-4..y+4 (clamped to the
 * image) of popcount(cl[y'][x] ^ cr[y'][x-d]) (BAND_INVALID where x-d < 0),
 * d in [0, dmax]:
 *   f0 = d0 / 64
 *   f1 = (dw - d0) / 64          dw = first argmin of agg over [0, dmax]
 *   f2 = agg(dw) / 558
 *   f3 = agg(r0) / 558           r0 = min(max(0, int(d0 + 0.5)), dmax)
 *   f4 = min of agg over [max(0, r0-10), min(dmax, r0+10)] / 558
 *   f5 = gray(left) - 0.5
 * feat is [6][H][W] here; the net reads BAND_F = 8 planes per item, the
 * last two being the network's spread / 16 and peak probability - 0.5,
 * which are inputs (copied, not computed). */
int orc_band_features(const uint64_t *cl, const uint64_t *cr, const double *d0,
                      const double *gray, int W, int H, int dmax, double *feat) {
    if (W < 1 || H < 1 || dmax < 0) return ORC_EBADARG;
    long N = (long)W * H;
    for (long p = 0; p < N; p++) {
        double t = d0[p] + 0.5;
        if (!(t > -9.0e15 && t < 9.0e15)) return ORC_ERANGE;
    }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++) {
        int *agg = (int *)malloc(sizeof(int) * (dmax + 1));
        for (int x = 0; x < W; x++) {
            for (int d = 0; d <= dmax; d++) {
                int s = 0;
                for (int dy = -BAND_ROWS; dy <= BAND_ROWS; dy++) {
                    int yy = y + dy;
                    if (yy < 0) yy = 0; else if (yy >= H) yy = H - 1;
                    long q = (long)yy * W + x;
                    s += x - d >= 0 ? __builtin_popcountll(cl[q] ^ cr[q - d]) : BAND_INVALID;
                }
                agg[d] = s;
            }
            long p = (long)y * W + x;
            int dw = 0;
            for (int d = 1; d <= dmax; d++) if (agg[d] < agg[dw]) dw = d;
            int64_t r = (int64_t)(d0[p] + 0.5);
            if (r < 0) r = 0;
            if (r > dmax) r = dmax;
            int lo = r - 10 < 0 ? 0 : (int)r - 10, hi = r + 10 > dmax ? dmax : (int)r + 10;
            int band = agg[lo];
            for (int d = lo + 1; d <= hi; d++) if (agg[d] < band) band = agg[d];
            feat[0 * N + p] = d0[p] / 64.0;
            feat[1 * N + p] = ((double)dw - d0[p]) / 64.0;
            feat[2 * N + p] = agg[dw] / 558.0;
            feat[3 * N + p] = agg[r] / 558.0;
            feat[4 * N + p] = band / 558.0;
            feat[5 * N + p] = gray[p] - 0.5;
        }
        free(agg);
    }
    return ORC_OK;
}

/* --------------------------------------------------------- conv layers
 * Conv2d.forward (stereonet.py:489-526): acc starts at the bias, then
 * channel, ky, kx in order; out-of-image taps are skipped. */
static void conv_fwd(const double *x, int ic, int H, int W, const double *w,
                     const double *b, int oc, int dil, double *y) {
    long HW = (long)H * W;
#pragma omp parallel for collapse(2) schedule(static)
    for (int o = 0; o < oc; o++) {
        for (int oy = 0; oy < H; oy++) {
            for (int ox = 0; ox < W; ox++) {
                double acc = b[o];
                for (int c = 0; c < ic; c++) {
                    for (int ky = 0; ky < 3; ky++) {
                        int iy = oy - dil + ky * dil;
                        if (iy < 0 || iy >= H) continue;
                        for (int kx = 0; kx < 3; kx++) {
                            int ix = ox - dil + kx * dil;
                            if (ix < 0 || ix >= W) continue;
                            acc += x[c * HW + (long)iy * W + ix] * w[((o * ic + c) * 3 + ky) * 3 + kx];
                        }
                    }
                }
                y[o * HW + (long)oy * W + ox] = acc;
            }
        }
    }
}

/* Conv2d.backward (stereonet.py:528-570): gw += x * g, gx += w * g, gb += g. */
static void conv_bwd(const double *x, int ic, int H, int W, const double *w, int oc,
                     int dil, const double *gy, double *gw, double *gb, double *gx) {
    long HW = (long)H * W;
    if (gx) memset(gx, 0, sizeof(double) * ic * HW);
    for (int o = 0; o < oc; o++) {
        double gsum = 0.0;
        for (int oy = 0; oy < H; oy++) {
            for (int ox = 0; ox < W; ox++) {
                double g = gy[o * HW + (long)oy * W + ox];
                if (g == 0.0) continue;
                gsum += g;
                for (int c = 0; c < ic; c++) {
                    for (int ky = 0; ky < 3; ky++) {
                        int iy = oy - dil + ky * dil;
                        if (iy < 0 || iy >= H) continue;
                        for (int kx = 0; kx < 3; kx++) {
                            int ix = ox - dil + kx * dil;
                            if (ix < 0 || ix >= W) continue;
                            long wi = ((o * ic + c) * 3 + ky) * 3 + kx;
                            long xi = c * HW + (long)iy * W + ix;
                            gw[wi] += x[xi] * g;
                            if (gx) gx[xi] += w[wi] * g;
                        }
                    }
                }
            }
        }
        gb[o] += gsum;
    }
}

/* parameter blocks in order w0, b0, w1, b1, w2, b2, w3, b3 */
static void band_bind(const double *params, const double **w, const double **b) {
    const double *p = params;
    for (int l = 0; l < BAND_L; l++) {
        w[l] = p; p += (long)band_oc[l] * band_ic[l] * 9;
        b[l] = p; p += band_oc[l];
    }
}

/* One item: feat [6][H][W] -> out [2][H][W] (raw o0, o1).  acts, when not
 * NULL, receives the three hidden activations (post leaky ReLU) and the
 * three pre-activations, each [16][H][W]: acts[0..2] post, acts[3..5] pre. */
static int band_forward_item(const double *params, const double *feat, int W, int H,
                             double *out, double **acts) {
    const double *w[BAND_L], *b[BAND_L];
    band_bind(params, w, b);
    long HW = (long)H * W;
    double *z = (double *)malloc(sizeof(double) * BAND_C * HW);
    double *a = (double *)malloc(sizeof(double) * BAND_C * HW);
    double *prev = (double *)malloc(sizeof(double) * BAND_C * HW);
    if (!z || !a || !prev) { free(z); free(a); free(prev); return ORC_ENOMEM; }
    memcpy(prev, feat, sizeof(double) * BAND_F * HW);
    for (int l = 0; l < BAND_L; l++) {
        if (l == BAND_L - 1) {
            conv_fwd(prev, band_ic[l], H, W, w[l], b[l], band_oc[l], band_dil[l], out);
            break;
        }
        conv_fwd(prev, band_ic[l], H, W, w[l], b[l], band_oc[l], band_dil[l], z);
        for (long i = 0; i < BAND_C * HW; i++) a[i] = z[i] > 0.0 ? z[i] : z[i] * 0.2;
        if (acts) {
            memcpy(acts[l], a, sizeof(double) * BAND_C * HW);
            memcpy(acts[3 + l], z, sizeof(double) * BAND_C * HW);
        }
        memcpy(prev, a, sizeof(double) * BAND_C * HW);
    }
    free(z); free(a); free(prev);
    return ORC_OK;
}

int orc_band_forward(const double *params, const double *feat, int nb, int W, int H,
                     double *out) {
    long HW = (long)H * W;
    for (int i = 0; i < nb; i++) {
        int rc = band_forward_item(params, feat + (long)i * BAND_F * HW, W, H,
                                   out + (long)i * BAND_O * HW, NULL);
        if (rc) return rc;
    }
    return ORC_OK;
}

/* Laplace negative log-likelihood of the target shift t under the predicted
 * shift s = 32 o0 and scale b = exp(rho), rho = clamp(o1 + 1):
 *   loss = sum over labelled pixels of (|t - s| / b + rho) / n_total
 * n_total = nb * W * H (every pixel, labelled or not).  g receives dloss/do. */
double orc_band_loss(const double *out, const double *target, const uint8_t *mask, int nb,
                     int W, int H, double *g) {
    long HW = (long)H * W;
    double n = (double)nb * HW, total = 0.0;
    for (int i = 0; i < nb; i++) {
        const double *o0 = out + (long)i * BAND_O * HW, *o1 = o0 + HW;
        double *g0 = g ? g + (long)i * BAND_O * HW : NULL, *g1 = g0 ? g0 + HW : NULL;
        for (long p = 0; p < HW; p++) {
            long q = (long)i * HW + p;
            if (g) { g0[p] = 0.0; g1[p] = 0.0; }
            if (!mask[q]) continue;
            double s = BAND_SHIFT_SCALE * o0[p];
            double rho = o1[p] + BAND_RHO0;
            int inside = rho > BAND_RHO_MIN && rho < BAND_RHO_MAX;
            if (rho < BAND_RHO_MIN) rho = BAND_RHO_MIN;
            if (rho > BAND_RHO_MAX) rho = BAND_RHO_MAX;
            double b = exp(rho);
            double e = target[q] - s;
            double ae = e < 0 ? -e : e;
            total += (ae / b + rho) / n;
            if (g) {
                double sg = e > 0 ? 1.0 : (e < 0 ? -1.0 : 0.0);
                g0[p] = -sg / b * BAND_SHIFT_SCALE / n;
                g1[p] = inside ? (1.0 - ae / b) / n : 0.0;
            }
        }
    }
    return total;
}

/* Gradients of orc_band_loss with respect to all parameters (all_params
 * order), accumulated into grads (zeroed first). */
int orc_band_grads(const double *params, const double *feat, const double *target,
                   const uint8_t *mask, int nb, int W, int H, double *grads, double *loss) {
    const double *w[BAND_L], *b[BAND_L];
    band_bind(params, w, b);
    long np = orc_band_param_count();
    memset(grads, 0, sizeof(double) * np);
    double *gw[BAND_L], *gb[BAND_L];
    {
        double *p = grads;
        for (int l = 0; l < BAND_L; l++) {
            gw[l] = p; p += (long)band_oc[l] * band_ic[l] * 9;
            gb[l] = p; p += band_oc[l];
        }
    }
    long HW = (long)H * W;
    double *acts[6];
    for (int k = 0; k < 6; k++) acts[k] = (double *)malloc(sizeof(double) * BAND_C * HW);
    double *out = (double *)malloc(sizeof(double) * nb * BAND_O * HW);
    double *gout = (double *)malloc(sizeof(double) * nb * BAND_O * HW);
    double *ga = (double *)malloc(sizeof(double) * BAND_C * HW);
    double *gz = (double *)malloc(sizeof(double) * BAND_C * HW);
    int rc = orc_band_forward(params, feat, nb, W, H, out);
    if (!rc) {
        double l = orc_band_loss(out, target, mask, nb, W, H, gout);
        if (loss) *loss = l;
    }
    for (int i = 0; i < nb && !rc; i++) {
        const double *f = feat + (long)i * BAND_F * HW;
        rc = band_forward_item(params, f, W, H, out + (long)i * BAND_O * HW, acts);
        if (rc) break;
        /* layer 3: input acts[2] */
        conv_bwd(acts[2], BAND_C, H, W, w[3], BAND_O, band_dil[3],
                 gout + (long)i * BAND_O * HW, gw[3], gb[3], ga);
        for (int l = 2; l >= 0; l--) {
            /* LeakyReLU.backward on the pre-activation acts[3 + l] */
            for (long k = 0; k < BAND_C * HW; k++)
                gz[k] = acts[3 + l][k] > 0.0 ? ga[k] : ga[k] * 0.2;
            const double *xin = l == 0 ? f : acts[l - 1];
            conv_bwd(xin, band_ic[l], H, W, w[l], BAND_C, band_dil[l], gz, gw[l], gb[l],
                     l == 0 ? NULL : ga);
        }
    }
    for (int k = 0; k < 6; k++) free(acts[k]);
    free(out); free(gout); free(ga); free(gz);
    return rc;
}

/* Adam.step (stereonet.py:1368-1387): running products for the bias
 * correction, per-element clip of the gradient to [-clip, clip]. */
void orc_adam_step(double *p, const double *g, double *m, double *v, long n, double lr,
                   double b1, double b2, double eps, double clip, double *b1t, double *b2t) {
    *b1t *= b1;
    *b2t *= b2;
    double c1 = 1.0 / (1.0 - *b1t);
    double c2 = 1.0 / (1.0 - *b2t);
    for (long i = 0; i < n; i++) {
        double gi = g[i];
        if (gi > clip) gi = clip;
        else if (gi < -clip) gi = -clip;
        double mi = b1 * m[i] + (1.0 - b1) * gi;
        double vi = b2 * v[i] + (1.0 - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrt(vi * c2) + eps);
    }
}

/* ------------------------------------------------------ band application
 * From the band net's raw output: b = exp(clamp(o1 + 1)); where b <= b_thr
 * the band centre moves to d0 + clamp(32 o0, +-shift_max) and its half-width
 * is min(R, max(rad_min, ceil(rad_k * b))); elsewhere (low confidence) the
 * fixed band stays: centre d0, half-width R. */
void orc_band_apply(const double *out, const double *d0, int W, int H, double b_thr,
                    double rad_k, int rad_min, int R, double shift_max, double *centre,
                    uint8_t *rad) {
    long HW = (long)H * W;
    for (long p = 0; p < HW; p++) {
        double rho = out[HW + p] + BAND_RHO0;
        if (rho < BAND_RHO_MIN) rho = BAND_RHO_MIN;
        if (rho > BAND_RHO_MAX) rho = BAND_RHO_MAX;
        double b = exp(rho);
        if (b <= b_thr) {
            double s = BAND_SHIFT_SCALE * out[p];
            if (s > shift_max) s = shift_max;
            if (s < -shift_max) s = -shift_max;
            centre[p] = d0[p] + s;
            double r = ceil(rad_k * b);
            if (r < rad_min) r = rad_min;
            if (r > R) r = R;
            rad[p] = (uint8_t)r;
        } else {
            centre[p] = d0[p];
            rad[p] = (uint8_t)R;
        }
    }
}

/* Training targets: t = clamp(label - d0, +-shift_max), labelled where the
 * label's LR status is 0. */
void orc_band_targets(const double *label, const int32_t *status, const double *d0, long n,
                      double shift_max, double *target, uint8_t *mask) {
    for (long p = 0; p < n; p++) {
        double t = label[p] - d0[p];
        if (t > shift_max) t = shift_max;
        if (t < -shift_max) t = -shift_max;
        target[p] = t;
        mask[p] = status[p] == 0;
    }
}

/* ------------------------------------------------ masked lr_refine
 * lr_refine (stereonet.py:5343-5391) around the band centres `centre`, with
 * the left view's band costs outside |k - R| <= rad[p] set to the invalid
 * cost; the right view is refined around left_to_right(centre) with the full
 * band, as lr_refine does.  ad_weight = prior_w = 0, uniq = 0, 8 paths. */
int orc_census(const double *img, int W, int H, int rx, int ry, uint64_t *out);
void orc_band_costs(const uint64_t *cl, const uint64_t *cr, const double *gl,
                    const double *gr, const int64_t *base, int W, int H, int R,
                    double ad_weight, double ad_trunc, double invalid,
                    const double *prior, double prior_w, double prior_t, double *C);
void orc_aggregate_path(const double *C, const int64_t *base, int W, int H, int K,
                        double P1, double P2, int dx, int dy, double *S);
int orc_left_to_right(const double *dl, int W, int H, double *dr);
void orc_mirror(const double *img, int W, int H, double *out);

static int refine_masked(const double *left, const double *right, const double *disp0,
                         const uint8_t *rad, int W, int H, int R, double P1, double P2,
                         int rx, int ry, double *out) {
    long N = (long)W * H;
    int K = 2 * R + 1;
    int nbits = (2 * rx + 1) * (2 * ry + 1) - 1;
    if (nbits > 64 || R < 0) return ORC_EBADARG;
    int64_t *base = (int64_t *)malloc(sizeof(int64_t) * N);
    uint64_t *cl = (uint64_t *)malloc(sizeof(uint64_t) * N);
    uint64_t *cr = (uint64_t *)malloc(sizeof(uint64_t) * N);
    double *C = (double *)malloc(sizeof(double) * N * K);
    double *S = (double *)calloc((size_t)N * K, sizeof(double));
    if (!base || !cl || !cr || !C || !S) {
        free(base); free(cl); free(cr); free(C); free(S);
        return ORC_ENOMEM;
    }
    for (long i = 0; i < N; i++) {
        double t = disp0[i] + 0.5;
        if (!(t > -9.0e15 && t < 9.0e15)) {
            free(base); free(cl); free(cr); free(C); free(S);
            return ORC_ERANGE;
        }
        int64_t v = (int64_t)t;
        base[i] = v > 0 ? v : 0;
    }
    orc_census(left, W, H, rx, ry, cl);
    orc_census(right, W, H, rx, ry, cr);
    double invalid = nbits + 4.0;
    orc_band_costs(cl, cr, left, right, base, W, H, R, 0.0, 20.0, invalid, disp0, 0.0, 4.0, C);
    if (rad) {
        for (long p = 0; p < N; p++)
            for (int k = 0; k < K; k++)
                if (abs(k - R) > rad[p]) C[p * K + k] = invalid;
    }
    static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1},
                                   {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
    for (int d = 0; d < 8; d++)
        orc_aggregate_path(C, base, W, H, K, P1, P2, dirs[d][0], dirs[d][1], S);
    for (long p = 0; p < N; p++) {
        long o = p * K;
        int bk = 0;
        double bv = S[o];
        for (int k = 1; k < K; k++)
            if (S[o + k] < bv) { bv = S[o + k]; bk = k; }
        if (bk == 0 || bk == K - 1) { out[p] = disp0[p]; continue; }
        double a = S[o + bk - 1], b = S[o + bk + 1];
        double den = a - 2.0 * bv + b;
        double off = 0.0;
        if (den > 1.0e-9) off = 0.5 * (a - b) / den;
        out[p] = (double)(base[p] - R + bk) + off;
    }
    free(base); free(cl); free(cr); free(C); free(S);
    return ORC_OK;
}

int orc_lr_refine_band(const double *left, const double *right, const double *centre,
                       const uint8_t *rad, int W, int H, double tol, int R, double P1,
                       double P2, int rx, int ry, double *out, int32_t *status) {
    long N = (long)W * H;
    double *dl = (double *)malloc(sizeof(double) * N);
    double *d0r = (double *)malloc(sizeof(double) * N);
    double *m1 = (double *)malloc(sizeof(double) * N);
    double *m2 = (double *)malloc(sizeof(double) * N);
    double *m3 = (double *)malloc(sizeof(double) * N);
    double *drm = (double *)malloc(sizeof(double) * N);
    double *dr = (double *)malloc(sizeof(double) * N);
    int rc = refine_masked(left, right, centre, rad, W, H, R, P1, P2, rx, ry, dl);
    if (!rc) rc = orc_left_to_right(centre, W, H, d0r);
    if (!rc) {
        orc_mirror(right, W, H, m1);
        orc_mirror(left, W, H, m2);
        orc_mirror(d0r, W, H, m3);
        rc = refine_masked(m1, m2, m3, NULL, W, H, R, P1, P2, rx, ry, drm);
    }
    if (rc) {
        free(dl); free(d0r); free(m1); free(m2); free(m3); free(drm); free(dr);
        return rc;
    }
    orc_mirror(drm, W, H, dr);
    for (long i = 0; i < N; i++) { status[i] = 0; out[i] = dl[i]; }
    for (int y = 0; y < H; y++) {
        long r = (long)y * W;
        for (int x = 0; x < W; x++) {
            double d = dl[r + x];
            int64_t xr = (int64_t)(x - d + 0.5);
            if (xr < 0 || xr >= W) { status[r + x] = 1; continue; }
            double e = dr[r + xr];
            if (fabs(d - e) <= tol) continue;
            status[r + x] = e > d ? 1 : 2;
        }
    }
    for (long i = 0; i < N; i++)
        if (status[i] == 2) out[i] = centre[i];
    for (int y = 0; y < H; y++) {
        long r = (long)y * W;
        for (int x = 0; x < W; x++) {
            if (status[r + x] != 1) continue;
            int a = x - 1;
            while (a >= 0 && status[r + a] == 1) a--;
            int b = x + 1;
            while (b < W && status[r + b] == 1) b++;
            double va = a >= 0 ? out[r + a] : 1.0e9;
            double vb = b < W ? out[r + b] : 1.0e9;
            double v = va < vb ? va : vb;
            out[r + x] = v < 1.0e8 ? v : centre[r + x];
        }
    }
    free(dl); free(d0r); free(m1); free(m2); free(m3); free(drm); free(dr);
    return ORC_OK;
}
