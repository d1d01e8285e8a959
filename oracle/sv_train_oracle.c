/*
 * sv_train_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 restatement of the reference's StereoNet training step
 * (stereonet.py): build_targets 1572-1611, StereoNet.forward with the layer
 * caches 1203-1233, the losses pseudo_huber 1326-1351 and disparity_ce
 * 1274-1323, StereoNet.backward 1235-1267 with every layer's backward
 * (Conv2d 528-570, Conv3d 643-693, LeakyReLU 714-719, CostVolume 801-824,
 * SoftArgmin 887-901, BilinearUpsample 958-974, FeatureNet 1047-1054,
 * CostFilter 1095-1101, Refinement 1153-1165), train_grads 1619-1653 and
 * Adam.step 1368-1387.  Every loop keeps the reference's order, including
 * the order in which gradients accumulate (the right siamese branch before
 * the left), so the gradients are the reference's bit for bit; the golden
 * fixtures made by running the reference pin that.  Only tests and the
 * benchmark's CPU-baseline leg call this file.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

double orc_fexp(double x);
long orc_param_count(const int *arch);

static const double LN2 = 0.6931471805599453;

/* fsqrt -- stereonet.py:34-56 (Newton from an exponent-halving seed) */
double orc_fsqrt(double x) {
    if (x <= 0.0) return 0.0;
    double y = x;
    if (y > 4.0) {
        double s = 1.0;
        while (y > 4.0) { y *= 0.25; s *= 2.0; }
        y = s;
    } else if (y < 0.25) {
        double s = 1.0;
        while (y < 0.25) { y *= 4.0; s *= 0.5; }
        y = s;
    } else {
        y = 1.0;
    }
    for (int i = 0; i < 24; i++) y = 0.5 * (y + x / y);
    return y;
}

/* flog -- stereonet.py:84-104 (atanh series) */
double orc_flog(double x) {
    if (x <= 0.0) return -1.0e308;
    long k = 0;
    while (x > 1.5) { x *= 0.5; k++; }
    while (x < 0.5) { x *= 2.0; k--; }
    double z = (x - 1.0) / (x + 1.0), z2 = z * z, total = 0.0, term = z;
    for (int n = 1; n < 40; n += 2) {
        total += term / n;
        term *= z2;
    }
    return 2.0 * total + k * LN2;
}

/* ----------------------------------------------------------------- layers */
static double *dalloc(long n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* Conv2d forward (489-526) with the reference's zero padding dil*(k-1)/2 */
static void conv2d_f(const double *x, int ic, int H, int W, const double *w, const double *b,
                     int oc, int s, int d, double *y, int *pOH, int *pOW) {
    const int k = 3, p = d, kk = 9, ickk = ic * 9;
    const int OH = (H + 2 * p - (2 * d + 1)) / s + 1, OW = (W + 2 * p - (2 * d + 1)) / s + 1;
    const long HW = (long)H * W;
    for (int o = 0; o < oc; o++)
        for (int oy = 0; oy < OH; oy++)
            for (int ox = 0; ox < OW; ox++) {
                double acc = b[o];
                const int iy0 = oy * s - p, ix0 = ox * s - p;
                for (int c = 0; c < ic; c++)
                    for (int ky = 0; ky < k; ky++) {
                        const int iy = iy0 + ky * d;
                        if (iy < 0 || iy >= H) continue;
                        for (int kx = 0; kx < k; kx++) {
                            const int ix = ix0 + kx * d;
                            if (ix < 0 || ix >= W) continue;
                            acc += x[c * HW + (long)iy * W + ix] * w[o * ickk + c * kk + ky * k + kx];
                        }
                    }
                y[(long)o * OH * OW + (long)oy * OW + ox] = acc;
            }
    *pOH = OH;
    *pOW = OW;
}

/* Conv2d.backward (528-570): gw, gb accumulate; gx (may be NULL) is set */
static void conv2d_b(const double *x, int ic, int H, int W, const double *w, int oc, int s,
                     int d, const double *gy, int OH, int OW, double *gw, double *gb,
                     double *gx) {
    const int k = 3, p = d, kk = 9, ickk = ic * 9;
    const long HW = (long)H * W;
    if (gx) memset(gx, 0, sizeof(double) * ic * HW);
    for (int o = 0; o < oc; o++) {
        double gsum = 0.0;
        for (int oy = 0; oy < OH; oy++)
            for (int ox = 0; ox < OW; ox++) {
                const double g = gy[(long)o * OH * OW + (long)oy * OW + ox];
                if (g == 0.0) continue;
                gsum += g;
                const int iy0 = oy * s - p, ix0 = ox * s - p;
                for (int c = 0; c < ic; c++)
                    for (int ky = 0; ky < k; ky++) {
                        const int iy = iy0 + ky * d;
                        if (iy < 0 || iy >= H) continue;
                        for (int kx = 0; kx < k; kx++) {
                            const int ix = ix0 + kx * d;
                            if (ix < 0 || ix >= W) continue;
                            const long xi = c * HW + (long)iy * W + ix;
                            const int wi = o * ickk + c * kk + ky * k + kx;
                            gw[wi] += x[xi] * g;
                            if (gx) gx[xi] += w[wi] * g;
                        }
                    }
            }
        gb[o] += gsum;
    }
}

/* Conv3d forward (596-641), stride 1, same padding */
static void conv3d_f(const double *x, int ic, int D, int H, int W, const double *w,
                     const double *b, int oc, double *y) {
    const long HW = (long)H * W, DHW = (long)D * HW;
    for (int o = 0; o < oc; o++)
        for (int od = 0; od < D; od++)
            for (int oy = 0; oy < H; oy++)
                for (int ox = 0; ox < W; ox++) {
                    double acc = b[o];
                    for (int c = 0; c < ic; c++)
                        for (int kd = 0; kd < 3; kd++) {
                            const int dd = od - 1 + kd;
                            if (dd < 0 || dd >= D) continue;
                            for (int ky = 0; ky < 3; ky++) {
                                const int yy = oy - 1 + ky;
                                if (yy < 0 || yy >= H) continue;
                                for (int kx = 0; kx < 3; kx++) {
                                    const int xx = ox - 1 + kx;
                                    if (xx < 0 || xx >= W) continue;
                                    acc += x[c * DHW + dd * HW + (long)yy * W + xx] *
                                           w[o * ic * 27 + c * 27 + kd * 9 + ky * 3 + kx];
                                }
                            }
                        }
                    y[o * DHW + od * HW + (long)oy * W + ox] = acc;
                }
}

/* Conv3d.backward (643-693) */
static void conv3d_b(const double *x, int ic, int D, int H, int W, const double *w, int oc,
                     const double *gy, double *gw, double *gb, double *gx) {
    const long HW = (long)H * W, DHW = (long)D * HW;
    memset(gx, 0, sizeof(double) * ic * DHW);
    for (int o = 0; o < oc; o++) {
        double gsum = 0.0;
        for (int od = 0; od < D; od++)
            for (int oy = 0; oy < H; oy++)
                for (int ox = 0; ox < W; ox++) {
                    const double g = gy[o * DHW + od * HW + (long)oy * W + ox];
                    if (g == 0.0) continue;
                    gsum += g;
                    for (int c = 0; c < ic; c++)
                        for (int kd = 0; kd < 3; kd++) {
                            const int dd = od - 1 + kd;
                            if (dd < 0 || dd >= D) continue;
                            for (int ky = 0; ky < 3; ky++) {
                                const int yy = oy - 1 + ky;
                                if (yy < 0 || yy >= H) continue;
                                for (int kx = 0; kx < 3; kx++) {
                                    const int xx = ox - 1 + kx;
                                    if (xx < 0 || xx >= W) continue;
                                    const long xi = c * DHW + dd * HW + (long)yy * W + xx;
                                    const int wi = o * ic * 27 + c * 27 + kd * 9 + ky * 3 + kx;
                                    gw[wi] += x[xi] * g;
                                    gx[xi] += w[wi] * g;
                                }
                            }
                        }
                }
        gb[o] += gsum;
    }
}

/* LeakyReLU forward (705-712) into y; backward (714-719) in place on g */
static void lrelu_f(const double *x, long n, double s, double *y) {
    for (long i = 0; i < n; i++) y[i] = x[i] > 0.0 ? x[i] : x[i] * s;
}
static void lrelu_b(const double *x, long n, double s, double *g) {
    for (long i = 0; i < n; i++) g[i] = x[i] > 0.0 ? g[i] : g[i] * s;
}

/* BilinearUpsample forward (913-956) and backward (958-974), one channel */
typedef struct { long i00, i01, i10, i11; double w00, w01, w10, w11; } tap_t;

static tap_t *up_taps(int H, int W, int H2, int W2) {
    tap_t *t = (tap_t *)malloc(sizeof(tap_t) * (size_t)H2 * W2);
    const double sy = H / (double)H2, sx = W / (double)W2;
    for (int oy = 0; oy < H2; oy++) {
        double fy = (oy + 0.5) * sy - 0.5;
        if (fy < 0.0) fy = 0.0;
        int y0 = (int)fy;
        if (y0 > H - 1) y0 = H - 1;
        const int y1 = y0 + 1 < H ? y0 + 1 : y0;
        const double wy = fy - y0;
        for (int ox = 0; ox < W2; ox++) {
            double fx = (ox + 0.5) * sx - 0.5;
            if (fx < 0.0) fx = 0.0;
            int x0 = (int)fx;
            if (x0 > W - 1) x0 = W - 1;
            const int x1 = x0 + 1 < W ? x0 + 1 : x0;
            const double wx = fx - x0;
            tap_t *p = &t[(long)oy * W2 + ox];
            p->w00 = (1.0 - wy) * (1.0 - wx);
            p->w01 = (1.0 - wy) * wx;
            p->w10 = wy * (1.0 - wx);
            p->w11 = wy * wx;
            p->i00 = (long)y0 * W + x0;
            p->i01 = (long)y0 * W + x1;
            p->i10 = (long)y1 * W + x0;
            p->i11 = (long)y1 * W + x1;
        }
    }
    return t;
}

static void up_f(const double *x, const tap_t *t, long n2, double *out) {
    for (long i = 0; i < n2; i++)
        out[i] = x[t[i].i00] * t[i].w00 + x[t[i].i01] * t[i].w01 + x[t[i].i10] * t[i].w10 +
                 x[t[i].i11] * t[i].w11;
}

static void up_b(const double *gy, const tap_t *t, long n2, long n, double *gx) {
    memset(gx, 0, sizeof(double) * n);
    for (long i = 0; i < n2; i++) {
        const double g = gy[i];
        if (g == 0.0) continue;
        gx[t[i].i00] += g * t[i].w00;
        gx[t[i].i01] += g * t[i].w01;
        gx[t[i].i10] += g * t[i].w10;
        gx[t[i].i11] += g * t[i].w11;
    }
}

/* avgpool2 (979-995), one channel */
static void pool2(const double *img, int H, int W, double *out) {
    const int H2 = H / 2, W2 = W / 2;
    for (int y = 0; y < H2; y++)
        for (int x = 0; x < W2; x++) {
            const long r0 = (long)(2 * y) * W, r1 = r0 + W;
            const int x0 = 2 * x;
            out[(long)y * W2 + x] = 0.25 * (img[r0 + x0] + img[r0 + x0 + 1] + img[r1 + x0] +
                                            img[r1 + x0 + 1]);
        }
}

/* ------------------------------------------------------------------ net */
typedef struct {
    int C, Cm, D, Rc, nd, dil[8];
    long off_fw[4], off_fb[4], off_cw[3], off_cb[3], off_rw[2][9], off_rb[2][9];
} layout_t;

static void layout(const int *arch, layout_t *L) {
    L->C = arch[0]; L->Cm = arch[1]; L->D = arch[2]; L->Rc = arch[3]; L->nd = arch[4];
    for (int i = 0; i < L->nd; i++) L->dil[i] = arch[5 + i];
    long p = 0;
    const int fic[4] = {1, L->C, L->C, L->C};
    for (int i = 0; i < 4; i++) {
        L->off_fw[i] = p; p += (long)L->C * fic[i] * 9;
        L->off_fb[i] = p; p += L->C;
    }
    const int cic[3] = {L->C, L->Cm, L->Cm}, coc[3] = {L->Cm, L->Cm, 1};
    for (int i = 0; i < 3; i++) {
        L->off_cw[i] = p; p += (long)coc[i] * cic[i] * 27;
        L->off_cb[i] = p; p += coc[i];
    }
    for (int lv = 0; lv < 2; lv++) {
        int prev = 2;
        for (int i = 0; i < L->nd; i++) {
            L->off_rw[lv][i] = p; p += (long)L->Rc * prev * 9;
            L->off_rb[lv][i] = p; p += L->Rc;
            prev = L->Rc;
        }
        L->off_rw[lv][L->nd] = p; p += (long)prev * 9;
        L->off_rb[lv][L->nd] = p; p += 1;
    }
}

/* FeatureNet caches of one image */
typedef struct {
    int h1, w1, h, w;
    double *y1, *a1, *y2, *a2, *y3, *a3, *f;
} feat_t;

static void feat_f(const layout_t *L, const double *P, const double *img, int H, int W,
                   feat_t *t) {
    const int C = L->C;
    const int h1 = (H - 1) / 2 + 1, w1 = (W - 1) / 2 + 1, h = (h1 - 1) / 2 + 1,
              w = (w1 - 1) / 2 + 1;
    int oh, ow;
    t->h1 = h1; t->w1 = w1; t->h = h; t->w = w;
    t->y1 = dalloc((long)C * h1 * w1); t->a1 = dalloc((long)C * h1 * w1);
    t->y2 = dalloc((long)C * h * w); t->a2 = dalloc((long)C * h * w);
    t->y3 = dalloc((long)C * h * w); t->a3 = dalloc((long)C * h * w);
    t->f = dalloc((long)C * h * w);
    conv2d_f(img, 1, H, W, P + L->off_fw[0], P + L->off_fb[0], C, 2, 1, t->y1, &oh, &ow);
    lrelu_f(t->y1, (long)C * h1 * w1, 0.2, t->a1);
    conv2d_f(t->a1, C, h1, w1, P + L->off_fw[1], P + L->off_fb[1], C, 2, 1, t->y2, &oh, &ow);
    lrelu_f(t->y2, (long)C * h * w, 0.2, t->a2);
    conv2d_f(t->a2, C, h, w, P + L->off_fw[2], P + L->off_fb[2], C, 1, 1, t->y3, &oh, &ow);
    lrelu_f(t->y3, (long)C * h * w, 0.2, t->a3);
    conv2d_f(t->a3, C, h, w, P + L->off_fw[3], P + L->off_fb[3], C, 1, 1, t->f, &oh, &ow);
}

/* FeatureNet.backward (1047-1054); the image gradient is not needed */
static void feat_b(const layout_t *L, const double *P, double *G, const double *img, int H,
                   int W, const feat_t *t, const double *gf) {
    const int C = L->C, h1 = t->h1, w1 = t->w1, h = t->h, w = t->w;
    double *g1 = dalloc((long)C * h * w), *g2 = dalloc((long)C * h * w);
    double *g3 = dalloc((long)C * h1 * w1);
    conv2d_b(t->a3, C, h, w, P + L->off_fw[3], C, 1, 1, gf, h, w, G + L->off_fw[3],
             G + L->off_fb[3], g1);
    lrelu_b(t->y3, (long)C * h * w, 0.2, g1);
    conv2d_b(t->a2, C, h, w, P + L->off_fw[2], C, 1, 1, g1, h, w, G + L->off_fw[2],
             G + L->off_fb[2], g2);
    lrelu_b(t->y2, (long)C * h * w, 0.2, g2);
    conv2d_b(t->a1, C, h1, w1, P + L->off_fw[1], C, 2, 1, g2, h, w, G + L->off_fw[1],
             G + L->off_fb[1], g3);
    lrelu_b(t->y1, (long)C * h1 * w1, 0.2, g3);
    conv2d_b(img, 1, H, W, P + L->off_fw[0], C, 2, 1, g3, h1, w1, G + L->off_fw[0],
             G + L->off_fb[0], NULL);
    free(g1); free(g2); free(g3);
}

static void feat_free(feat_t *t) {
    free(t->y1); free(t->a1); free(t->y2); free(t->a2); free(t->y3); free(t->a3); free(t->f);
}

/* Refinement caches of one level */
typedef struct {
    int H, W;
    double *x;            /* [2][H][W] input (disp, guide)       */
    double *y[8], *a[8];  /* conv outputs before / after lrelu   */
    double *summed, *out;
} ref_t;

static void ref_f(const layout_t *L, const double *P, int lv, const double *disp,
                  const double *guide, int H, int W, ref_t *t) {
    const long HW = (long)H * W;
    const int Rc = L->Rc;
    int oh, ow;
    t->H = H; t->W = W;
    t->x = dalloc(2 * HW);
    memcpy(t->x, disp, sizeof(double) * HW);
    memcpy(t->x + HW, guide, sizeof(double) * HW);
    const double *cur = t->x;
    int prev = 2;
    for (int i = 0; i < L->nd; i++) {
        t->y[i] = dalloc(Rc * HW);
        t->a[i] = dalloc(Rc * HW);
        conv2d_f(cur, prev, H, W, P + L->off_rw[lv][i], P + L->off_rb[lv][i], Rc, 1, L->dil[i],
                 t->y[i], &oh, &ow);
        lrelu_f(t->y[i], Rc * HW, 0.2, t->a[i]);
        cur = t->a[i];
        prev = Rc;
    }
    double *res = dalloc(HW);
    conv2d_f(cur, prev, H, W, P + L->off_rw[lv][L->nd], P + L->off_rb[lv][L->nd], 1, 1, 1, res,
             &oh, &ow);
    t->summed = dalloc(HW);
    t->out = dalloc(HW);
    for (long i = 0; i < HW; i++) t->summed[i] = disp[i] + res[i];
    lrelu_f(t->summed, HW, 0.0, t->out);
    free(res);
}

/* Refinement.backward (1153-1165) -> gradient on the disparity input */
static void ref_b(const layout_t *L, const double *P, double *G, int lv, const ref_t *t,
                  const double *gout, double *gdisp) {
    const int H = t->H, W = t->W, Rc = L->Rc, nd = L->nd;
    const long HW = (long)H * W;
    double *g = dalloc(HW);
    memcpy(g, gout, sizeof(double) * HW);
    lrelu_b(t->summed, HW, 0.0, g);
    double *gres = dalloc(Rc * HW), *gtmp = dalloc((Rc > 2 ? Rc : 2) * HW);
    conv2d_b(t->a[nd - 1], Rc, H, W, P + L->off_rw[lv][nd], 1, 1, 1, g, H, W,
             G + L->off_rw[lv][nd], G + L->off_rb[lv][nd], gres);
    for (int i = nd - 1; i >= 0; i--) {
        lrelu_b(t->y[i], Rc * HW, 0.2, gres);
        const double *xin = i > 0 ? t->a[i - 1] : t->x;
        const int ic = i > 0 ? Rc : 2;
        conv2d_b(xin, ic, H, W, P + L->off_rw[lv][i], Rc, 1, L->dil[i], gres, H, W,
                 G + L->off_rw[lv][i], G + L->off_rb[lv][i], gtmp);
        memcpy(gres, gtmp, sizeof(double) * ic * HW);
    }
    for (long i = 0; i < HW; i++) gdisp[i] = gres[i] + g[i];
    free(g); free(gres); free(gtmp);
}

static void ref_free(const layout_t *L, ref_t *t) {
    free(t->x);
    for (int i = 0; i < L->nd; i++) { free(t->y[i]); free(t->a[i]); }
    free(t->summed); free(t->out);
}

/* pseudo_huber (1326-1351) -> loss; grad = wgt * x / r / count */
static double huber(const double *pred, const double *tgt, const uint8_t *valid, long n,
                    double wgt, double *grad) {
    const double alpha = 1.0, a2 = alpha * alpha;
    double total = 0.0;
    long count = 0;
    for (long i = 0; i < n; i++) grad[i] = 0.0;
    for (long i = 0; i < n; i++) {
        if (!valid[i]) continue;
        const double x = pred[i] - tgt[i];
        const double r = orc_fsqrt(x * x + a2);
        total += r - alpha;
        grad[i] = x / r;
        count++;
    }
    if (count == 0) return 0.0;
    const double inv = 1.0 / count;
    for (long i = 0; i < n; i++) grad[i] *= inv;
    for (long i = 0; i < n; i++) grad[i] = grad[i] * wgt;
    return total * inv;
}

/* disparity_ce (1274-1323) with sigma 0.8 -> loss; gcost[d][i] = q - p
 * (scaled by 1 / count) */
static double dist_ce(const double *probs, const double *tgt, const uint8_t *valid, int D,
                      long HW, double *gcost) {
    const double sigma = 0.8, inv2s2 = 1.0 / (2.0 * sigma * sigma);
    double total = 0.0, q[64];
    long count = 0;
    for (long i = 0; i < (long)D * HW; i++) gcost[i] = 0.0;
    for (long i = 0; i < HW; i++) {
        if (!valid[i]) continue;
        const double dg = tgt[i];
        double qsum = 0.0;
        for (int d = 0; d < D; d++) {
            const double e = d - dg;
            q[d] = orc_fexp(-e * e * inv2s2);
            qsum += q[d];
        }
        if (qsum <= 0.0) continue;
        const double qinv = 1.0 / qsum;
        for (int d = 0; d < D; d++) {
            q[d] *= qinv;
            const double pk = probs[d * HW + i];
            if (pk > 1.0e-12) total -= q[d] * orc_flog(pk);
            gcost[d * HW + i] = q[d] - pk;
        }
        count++;
    }
    if (count == 0) return 0.0;
    const double inv = 1.0 / count;
    for (long i = 0; i < (long)D * HW; i++) gcost[i] *= inv;
    return total * inv;
}

/*
 * train_grads (1619-1653) on one sample.  left/right/disp are [H][W] FP64,
 * valid [H][W] (nonzero = valid); W and H must be multiples of 4 (the
 * reference's pyramid targets and outputs only line up then).  grads gets
 * the full gradient in all_params() order; loss the weighted total; d2 (may
 * be NULL) the full-resolution prediction.
 */
int orc_train_grads(const int *arch, const double *P, const double *left, const double *right,
                    const double *disp, const uint8_t *valid, int W, int H, double *grads,
                    double *loss, double *d2_out) {
    if (W % 4 || H % 4 || W < 8 || H < 8) return 1;
    layout_t L;
    layout(arch, &L);
    const long np = orc_param_count(arch);
    memset(grads, 0, sizeof(double) * np);
    const int D = L.D, C = L.C, Cm = L.Cm;
    /* build_targets (1595-1611) */
    const int H2 = H / 2, W2 = W / 2, H4 = H2 / 2, W4 = W2 / 2;
    const long HW = (long)H * W, HW2 = (long)H2 * W2, HW4 = (long)H4 * W4;
    double *dh = dalloc(HW2), *dq = dalloc(HW4), *gh = dalloc(HW2);
    uint8_t *vh = (uint8_t *)calloc(HW2, 1), *vq = (uint8_t *)calloc(HW4, 1);
    uint8_t *vf = (uint8_t *)calloc(HW, 1);
    for (long i = 0; i < HW; i++) vf[i] = valid[i] != 0;
    pool2(disp, H, W, dh);
    for (long i = 0; i < HW2; i++) dh[i] = dh[i] * 0.5;
    for (int y = 0; y < H2; y++)
        for (int x = 0; x < W2; x++) {
            const long r0 = (long)(2 * y) * W, r1 = r0 + W;
            vh[(long)y * W2 + x] = vf[r0 + 2 * x] && vf[r0 + 2 * x + 1] && vf[r1 + 2 * x] &&
                                   vf[r1 + 2 * x + 1];
        }
    pool2(left, H, W, gh);
    pool2(dh, H2, W2, dq);
    for (long i = 0; i < HW4; i++) dq[i] = dq[i] * 0.5;
    for (int y = 0; y < H4; y++)
        for (int x = 0; x < W4; x++) {
            const long r0 = (long)(2 * y) * W2, r1 = r0 + W2;
            vq[(long)y * W4 + x] = vh[r0 + 2 * x] && vh[r0 + 2 * x + 1] && vh[r1 + 2 * x] &&
                                   vh[r1 + 2 * x + 1];
        }
    /* forward (1203-1233) */
    feat_t tl, tr;
    feat_f(&L, P, left, H, W, &tl);
    feat_f(&L, P, right, H, W, &tr);
    const int h = tl.h, w = tl.w;
    const long hw = (long)h * w, DHW = (long)D * hw;
    double *vol = dalloc(C * DHW), *sign = dalloc(C * DHW);
    for (int c = 0; c < C; c++)
        for (int d = 0; d < D; d++)
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++) {
                    const long idx = c * DHW + d * hw + (long)y * w + x;
                    const int xr = x - d;
                    if (xr < 0) { vol[idx] = 2.0; continue; }
                    const double v = tl.f[c * hw + (long)y * w + x] - tr.f[c * hw + (long)y * w + xr];
                    if (v < 0.0) { vol[idx] = -v; sign[idx] = -1.0; }
                    else { vol[idx] = v; sign[idx] = 1.0; }
                }
    double *q1 = dalloc(Cm * DHW), *b1 = dalloc(Cm * DHW), *q2 = dalloc(Cm * DHW),
           *b2 = dalloc(Cm * DHW), *cost = dalloc(DHW);
    conv3d_f(vol, C, D, h, w, P + L.off_cw[0], P + L.off_cb[0], Cm, q1);
    lrelu_f(q1, Cm * DHW, 0.2, b1);
    conv3d_f(b1, Cm, D, h, w, P + L.off_cw[1], P + L.off_cb[1], Cm, q2);
    lrelu_f(q2, Cm * DHW, 0.2, b2);
    conv3d_f(b2, Cm, D, h, w, P + L.off_cw[2], P + L.off_cb[2], 1, cost);
    /* SoftArgmin.forward with the invalid mask (858-885, 827-840) */
    double *probs = dalloc(DHW), *d0 = dalloc(hw), *cm = dalloc(DHW);
    for (int d = 0; d < D; d++)
        for (long i = 0; i < hw; i++) {
            const int x = (int)(i % w);
            cm[d * hw + i] = cost[d * hw + i] + ((d >= 1 && x < d) ? 8.0 : 0.0);
        }
    for (long i = 0; i < hw; i++) {
        double best = -cm[i];
        for (int d = 1; d < D; d++) {
            const double v = -cm[d * hw + i];
            if (v > best) best = v;
        }
        double total = 0.0;
        for (int d = 0; d < D; d++) {
            const double e = orc_fexp(-cm[d * hw + i] - best);
            probs[d * hw + i] = e;
            total += e;
        }
        const double inv = 1.0 / total;
        double acc = 0.0;
        for (int d = 0; d < D; d++) {
            const double p = probs[d * hw + i] * inv;
            probs[d * hw + i] = p;
            acc += d * p;
        }
        d0[i] = acc;
    }
    tap_t *t1 = up_taps(h, w, H2, W2), *t2 = up_taps(H2, W2, H, W);
    double *u1 = dalloc(HW2), *u2 = dalloc(HW);
    up_f(d0, t1, HW2, u1);
    for (long i = 0; i < HW2; i++) u1[i] = u1[i] * 2.0;
    ref_t r1, r2;
    ref_f(&L, P, 0, u1, gh, H2, W2, &r1);
    up_f(r1.out, t2, HW, u2);
    for (long i = 0; i < HW; i++) u2[i] = u2[i] * 2.0;
    ref_f(&L, P, 1, u2, left, H, W, &r2);
    /* losses (train_grads 1628-1649) */
    static const double LEVEL_W[3] = {0.5, 0.7, 1.0};
    const double CE_W = 2.0;
    double *g0 = dalloc(HW4), *g1 = dalloc(HW2), *g2 = dalloc(HW);
    double total = 0.0;
    total += LEVEL_W[0] * huber(d0, dq, vq, hw, LEVEL_W[0], g0);
    total += LEVEL_W[1] * huber(r1.out, dh, vh, HW2, LEVEL_W[1], g1);
    total += LEVEL_W[2] * huber(r2.out, disp, vf, HW, LEVEL_W[2], g2);
    double *gce = dalloc(DHW);
    total += CE_W * dist_ce(probs, dq, vq, D, hw, gce);
    for (long i = 0; i < DHW; i++) gce[i] = CE_W * gce[i];
    /* StereoNet.backward (1235-1267) */
    double *gd = dalloc(HW), *gu = dalloc(HW);
    ref_b(&L, P, grads, 1, &r2, g2, gd);
    for (long i = 0; i < HW; i++) gd[i] = gd[i] * 2.0;
    up_b(gd, t2, HW, HW2, gu);
    for (long i = 0; i < HW2; i++) gu[i] += g1[i];
    double *gd1 = dalloc(HW2), *gq = dalloc(hw);
    ref_b(&L, P, grads, 0, &r1, gu, gd1);
    for (long i = 0; i < HW2; i++) gd1[i] = gd1[i] * 2.0;
    up_b(gd1, t1, HW2, hw, gq);
    for (long i = 0; i < hw; i++) gq[i] += g0[i];
    double *gcost = dalloc(DHW);
    for (long i = 0; i < hw; i++) {
        const double g = gq[i];
        if (g == 0.0) continue;
        const double di = d0[i];
        for (int d = 0; d < D; d++) gcost[d * hw + i] = g * probs[d * hw + i] * (di - d);
    }
    for (long i = 0; i < DHW; i++) gcost[i] += gce[i];
    double *gb2 = dalloc(Cm * DHW), *gb1 = dalloc(Cm * DHW), *gvol = dalloc(C * DHW);
    conv3d_b(b2, Cm, D, h, w, P + L.off_cw[2], 1, gcost, grads + L.off_cw[2], grads + L.off_cb[2],
             gb2);
    lrelu_b(q2, Cm * DHW, 0.2, gb2);
    conv3d_b(b1, Cm, D, h, w, P + L.off_cw[1], Cm, gb2, grads + L.off_cw[1], grads + L.off_cb[1],
             gb1);
    lrelu_b(q1, Cm * DHW, 0.2, gb1);
    conv3d_b(vol, C, D, h, w, P + L.off_cw[0], Cm, gb1, grads + L.off_cw[0], grads + L.off_cb[0],
             gvol);
    double *gfl = dalloc(C * hw), *gfr = dalloc(C * hw);
    for (int c = 0; c < C; c++)
        for (int d = 0; d < D; d++)
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++) {
                    const int xr = x - d;
                    if (xr < 0) continue;
                    const long idx = c * DHW + d * hw + (long)y * w + x;
                    const double g = gvol[idx] * sign[idx];
                    if (g == 0.0) continue;
                    gfl[c * hw + (long)y * w + x] += g;
                    gfr[c * hw + (long)y * w + xr] -= g;
                }
    feat_b(&L, P, grads, right, H, W, &tr, gfr);
    feat_b(&L, P, grads, left, H, W, &tl, gfl);
    if (loss) *loss = total;
    if (d2_out) memcpy(d2_out, r2.out, sizeof(double) * HW);
    free(dh); free(dq); free(gh); free(vh); free(vq); free(vf);
    feat_free(&tl); feat_free(&tr);
    free(vol); free(sign); free(q1); free(b1); free(q2); free(b2); free(cost);
    free(probs); free(d0); free(cm); free(t1); free(t2); free(u1); free(u2);
    ref_free(&L, &r1); ref_free(&L, &r2);
    free(g0); free(g1); free(g2); free(gce); free(gd); free(gu); free(gd1); free(gq);
    free(gcost); free(gb2); free(gb1); free(gvol); free(gfl); free(gfr);
    return 0;
}

/* Adam.step (1368-1387) with the reference's fsqrt: one step over n parameters; *b1t, *b2t are the
 * running products (start at 1.0) */
void orc_train_adam_step(double *p, const double *g, double *m, double *v, long n, double lr,
                   double *b1t, double *b2t, double clip) {
    const double b1 = 0.9, b2 = 0.999, eps = 1.0e-8;
    *b1t *= b1;
    *b2t *= b2;
    const double c1 = 1.0 / (1.0 - *b1t), c2 = 1.0 / (1.0 - *b2t);
    for (long i = 0; i < n; i++) {
        double gi = g[i];
        if (gi > clip) gi = clip;
        else if (gi < -clip) gi = -clip;
        const double mi = b1 * m[i] + (1.0 - b1) * gi;
        const double vi = b2 * v[i] + (1.0 - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (orc_fsqrt(vi * c2) + eps);
    }
}
