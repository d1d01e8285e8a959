/*
 * sv_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C FP64 restatement of the reference's disparity hot path
 * (stereonet.py, Ray-5106/From-Scratch-Stereo-Vision), used as the checker
 * for the CUDA path.  Only the tests, the smoke check and bench.py's CPU
 * baseline leg load this library; the product path never calls it.
 *
 * Every function states the reference lines it follows.  The arithmetic is
 * written in the reference's own evaluation order (Python evaluates left to
 * right, one IEEE double rounding per operation), and the file is compiled
 * with -ffp-contract=off so no multiply-add is fused: the results are
 * bit-identical to the Python reference, which the golden fixtures under
 * tests/golden/ (generated by running the reference itself) pin.
 *
 * Parallelism (OpenMP) only splits work whose per-element operation order
 * does not depend on the split: output pixels of a convolution, rows of a
 * census, scanlines of one SGM path.  SGM paths still run one after another
 * and add into S in the reference's direction order.
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_EBADARG 1
#define ORC_ENOMEM 2
#define ORC_ERANGE 3

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------
 * fexp -- stereonet.py:59-81 (range reduction + 15-term Taylor series)
 * ---------------------------------------------------------------------- */
static const double LN2 = 0.6931471805599453;

double orc_fexp(double x) {
    if (x > 700.0) return 1.0e308;
    if (x < -700.0) return 0.0;
    double q = x / LN2 + (x >= 0.0 ? 0.5 : -0.5);
    long k = (long)q;                       /* Python int(): toward zero */
    double r = x - (double)k * LN2;
    double term = 1.0, total = 1.0;
    for (int n = 1; n < 16; n++) {
        term = term * r / (double)n;
        total += term;
    }
    if (k >= 0) {
        for (long i = 0; i < k; i++) total *= 2.0;
    } else {
        for (long i = 0; i < -k; i++) total *= 0.5;
    }
    return total;
}

/* ------------------------------------------------------------------------
 * Conv2d.forward -- stereonet.py:482-526.  x [ic][H][W] -> y [oc][OH][OW]
 * ---------------------------------------------------------------------- */
static void conv2d(const double *x, int ic, int H, int W, const double *w,
                   const double *b, int oc, int k, int s, int d, double *y,
                   int *pOH, int *pOW) {
    int p = (d * (k - 1)) / 2;
    int eff = d * (k - 1) + 1;
    int OH = (H + 2 * p - eff) / s + 1;
    int OW = (W + 2 * p - eff) / s + 1;
    long HW = (long)H * W;
    int kk = k * k, ickk = ic * kk;
#pragma omp parallel for collapse(2) schedule(static)
    for (int o = 0; o < oc; o++) {
        for (int oy = 0; oy < OH; oy++) {
            int wo = o * ickk;
            long orow = (long)o * OH * OW + (long)oy * OW;
            int iy0 = oy * s - p;
            for (int ox = 0; ox < OW; ox++) {
                int ix0 = ox * s - p;
                double acc = b[o];
                for (int c = 0; c < ic; c++) {
                    long xb = c * HW;
                    int wc = wo + c * kk;
                    for (int ky = 0; ky < k; ky++) {
                        int iy = iy0 + ky * d;
                        if (iy < 0 || iy >= H) continue;
                        long xr = xb + (long)iy * W;
                        int wr = wc + ky * k;
                        for (int kx = 0; kx < k; kx++) {
                            int ix = ix0 + kx * d;
                            if (ix < 0 || ix >= W) continue;
                            acc += x[xr + ix] * w[wr + kx];
                        }
                    }
                }
                y[orow + ox] = acc;
            }
        }
    }
    *pOH = OH;
    *pOW = OW;
}

/* Conv3d.forward -- stereonet.py:596-641, stride 1, same padding.
 * x [ic][D][H][W] -> y [oc][D][H][W] */
static void conv3d(const double *x, int ic, int D, int H, int W,
                   const double *w, const double *b, int oc, int k, double *y) {
    int p = k / 2;
    long HW = (long)H * W, DHW = (long)D * HW;
    int kk = k * k, kkk = k * k * k, ickkk = ic * kkk;
#pragma omp parallel for collapse(3) schedule(static)
    for (int o = 0; o < oc; o++) {
        for (int od = 0; od < D; od++) {
            for (int oy = 0; oy < H; oy++) {
                int wo = o * ickkk;
                int d0 = od - p, y0 = oy - p;
                long orow = (long)o * DHW + (long)od * HW + (long)oy * W;
                for (int ox = 0; ox < W; ox++) {
                    int x0 = ox - p;
                    double acc = b[o];
                    for (int c = 0; c < ic; c++) {
                        long xb = c * DHW;
                        int wc = wo + c * kkk;
                        for (int kd = 0; kd < k; kd++) {
                            int dd = d0 + kd;
                            if (dd < 0 || dd >= D) continue;
                            long xd = xb + (long)dd * HW;
                            int wd = wc + kd * kk;
                            for (int ky = 0; ky < k; ky++) {
                                int yy = y0 + ky;
                                if (yy < 0 || yy >= H) continue;
                                long xr = xd + (long)yy * W;
                                int wr = wd + ky * k;
                                for (int kx = 0; kx < k; kx++) {
                                    int xx = x0 + kx;
                                    if (xx < 0 || xx >= W) continue;
                                    acc += x[xr + xx] * w[wr + kx];
                                }
                            }
                        }
                    }
                    y[orow + ox] = acc;
                }
            }
        }
    }
}

/* LeakyReLU.forward -- stereonet.py:705-712 (slope 0.0 gives v*0.0) */
static void lrelu(double *x, long n, double s) {
    for (long i = 0; i < n; i++) {
        double v = x[i];
        x[i] = v > 0.0 ? v : v * s;
    }
}

/* CostVolume.forward -- stereonet.py:771-799.  [C][h][w] x2 -> [C][D][h][w] */
static void cost_volume(const double *fl, const double *fr, int C, int D,
                        int H, int W, double *vol) {
    long HW = (long)H * W, DHW = (long)D * HW;
    for (int c = 0; c < C; c++) {
        long cb = c * HW, vb = c * DHW;
        for (int d = 0; d < D; d++) {
            long db = vb + d * HW;
            for (int y = 0; y < H; y++) {
                long row = (long)y * W;
                for (int x = 0; x < W; x++) {
                    long idx = db + row + x;
                    int xr = x - d;
                    if (xr < 0) { vol[idx] = 2.0; continue; }   /* INVALID_COST */
                    double v = fl[cb + row + x] - fr[cb + row + xr];
                    vol[idx] = v < 0.0 ? -v : v;
                }
            }
        }
    }
}

/* SoftArgmin.forward with CostVolume.invalid_mask -- stereonet.py:858-885,
 * 827-840 (penalty 8.0 where x < d). */
static void soft_argmin(const double *cost, int D, int H, int W, double *disp) {
    long HW = (long)H * W;
    double *c = (double *)malloc(sizeof(double) * D);
    double *pr = (double *)malloc(sizeof(double) * D);
    for (long i = 0; i < HW; i++) {
        int x = (int)(i % W);
        for (int d = 0; d < D; d++) {
            double pen = (d >= 1 && x < d) ? 8.0 : 0.0;
            c[d] = cost[d * HW + i] + pen;
        }
        double best = -c[0];
        for (int d = 1; d < D; d++) {
            double v = -c[d];
            if (v > best) best = v;
        }
        double total = 0.0;
        for (int d = 0; d < D; d++) {
            double e = orc_fexp(-c[d] - best);
            pr[d] = e;
            total += e;
        }
        double inv = 1.0 / total;
        double acc = 0.0;
        for (int d = 0; d < D; d++) {
            double p = pr[d] * inv;
            acc += (double)d * p;
        }
        disp[i] = acc;
    }
    free(c);
    free(pr);
}

/* BilinearUpsample.forward -- stereonet.py:913-956 (half-pixel centres).
 * x [C][H][W] -> out [C][H2][W2] */
static void bilinear(const double *x, int C, int H, int W, int H2, int W2,
                     double *out) {
    double sy = H / (double)H2;
    double sx = W / (double)W2;
    long HW = (long)H * W;
#pragma omp parallel for schedule(static)
    for (int oy = 0; oy < H2; oy++) {
        double fy = (oy + 0.5) * sy - 0.5;
        if (fy < 0.0) fy = 0.0;
        int y0 = (int)fy;
        if (y0 > H - 1) y0 = H - 1;
        int y1 = y0 + 1 < H ? y0 + 1 : y0;
        double wy = fy - y0;
        for (int ox = 0; ox < W2; ox++) {
            double fx = (ox + 0.5) * sx - 0.5;
            if (fx < 0.0) fx = 0.0;
            int x0 = (int)fx;
            if (x0 > W - 1) x0 = W - 1;
            int x1 = x0 + 1 < W ? x0 + 1 : x0;
            double wx = fx - x0;
            double w00 = (1.0 - wy) * (1.0 - wx);
            double w01 = (1.0 - wy) * wx;
            double w10 = wy * (1.0 - wx);
            double w11 = wy * wx;
            long i00 = (long)y0 * W + x0, i01 = (long)y0 * W + x1;
            long i10 = (long)y1 * W + x0, i11 = (long)y1 * W + x1;
            for (int c = 0; c < C; c++) {
                long cb = c * HW;
                out[(long)c * H2 * W2 + (long)oy * W2 + ox] =
                    x[cb + i00] * w00 + x[cb + i01] * w01 +
                    x[cb + i10] * w10 + x[cb + i11] * w11;
            }
        }
    }
}

/* resize_gray -- stereonet.py:3843-3845 */
void orc_resize(const double *img, int W, int H, int W2, int H2, double *out) {
    bilinear(img, 1, H, W, H2, W2, out);
}

/* avgpool2 -- stereonet.py:979-995 */
void orc_avgpool2(const double *img, int C, int H, int W, double *out) {
    int H2 = H / 2, W2 = W / 2;
    for (int c = 0; c < C; c++) {
        long cb = (long)c * H * W, ob = (long)c * H2 * W2;
        for (int y = 0; y < H2; y++) {
            long r0 = cb + (long)(2 * y) * W, r1 = r0 + W;
            for (int x = 0; x < W2; x++) {
                int x0 = 2 * x;
                out[ob + (long)y * W2 + x] =
                    0.25 * (img[r0 + x0] + img[r0 + x0 + 1] + img[r1 + x0] +
                            img[r1 + x0 + 1]);
            }
        }
    }
}

/* ------------------------------------------------------------------------
 * StereoNet -- stereonet.py:1022-1233.  Parameters arrive as one flat array
 * of the blocks in StereoNet.all_params() order (stereonet.py:1193-1195):
 *   feat  c1.w c1.b c2.w c2.b c3.w c3.b c4.w c4.b
 *   filt  c1.w c1.b c2.w c2.b c3.w c3.b
 *   ref1  conv[i].w conv[i].b (per dilation) c3.w c3.b
 *   ref2  same
 * arch = {feat_C, cost_C, D, refine_C, ndil, dil[0..ndil-1]}
 * ---------------------------------------------------------------------- */
typedef struct {
    int C, Cm, D, Rc, ndil, dil[8];
    const double *f_w[4], *f_b[4];
    const double *c_w[3], *c_b[3];
    const double *r_w[2][9], *r_b[2][9];   /* per level: ndil convs + final */
} net_t;

static int net_bind(const int *arch, const double *params, net_t *n) {
    n->C = arch[0];
    n->Cm = arch[1];
    n->D = arch[2];
    n->Rc = arch[3];
    n->ndil = arch[4];
    if (n->ndil < 1 || n->ndil > 8) return ORC_EBADARG;
    for (int i = 0; i < n->ndil; i++) n->dil[i] = arch[5 + i];
    const double *p = params;
    int C = n->C, Cm = n->Cm, Rc = n->Rc;
    int fic[4] = {1, C, C, C};
    for (int i = 0; i < 4; i++) {
        n->f_w[i] = p; p += C * fic[i] * 9;
        n->f_b[i] = p; p += C;
    }
    int cic[3] = {C, Cm, Cm}, coc[3] = {Cm, Cm, 1};
    for (int i = 0; i < 3; i++) {
        n->c_w[i] = p; p += coc[i] * cic[i] * 27;
        n->c_b[i] = p; p += coc[i];
    }
    for (int lv = 0; lv < 2; lv++) {
        int prev = 2;
        for (int i = 0; i < n->ndil; i++) {
            n->r_w[lv][i] = p; p += Rc * prev * 9;
            n->r_b[lv][i] = p; p += Rc;
            prev = Rc;
        }
        n->r_w[lv][n->ndil] = p; p += prev * 9;
        n->r_b[lv][n->ndil] = p; p += 1;
    }
    return ORC_OK;
}

long orc_param_count(const int *arch) {
    int C = arch[0], Cm = arch[1], Rc = arch[3], nd = arch[4];
    long n = 0;
    n += (long)C * 1 * 9 + C + 3 * ((long)C * C * 9 + C);
    n += (long)Cm * C * 27 + Cm + (long)Cm * Cm * 27 + Cm + (long)Cm * 27 + 1;
    long lv = 0;
    int prev = 2;
    for (int i = 0; i < nd; i++) { lv += (long)Rc * prev * 9 + Rc; prev = Rc; }
    lv += (long)prev * 9 + 1;
    return n + 2 * lv;
}

/* FeatureNet.forward -- stereonet.py:1037-1045 */
static double *feature_net(const net_t *n, const double *img, int H, int W,
                           int *ph, int *pw) {
    int C = n->C;
    int h1, w1, h2, w2, h3, w3, h4, w4;
    int eh = (H - 1) / 2 + 1, ew = (W - 1) / 2 + 1;
    double *a = (double *)malloc(sizeof(double) * C * (long)eh * ew);
    double *b = (double *)malloc(sizeof(double) * C * (long)eh * ew);
    conv2d(img, 1, H, W, n->f_w[0], n->f_b[0], C, 3, 2, 1, a, &h1, &w1);
    lrelu(a, (long)C * h1 * w1, 0.2);
    conv2d(a, C, h1, w1, n->f_w[1], n->f_b[1], C, 3, 2, 1, b, &h2, &w2);
    lrelu(b, (long)C * h2 * w2, 0.2);
    conv2d(b, C, h2, w2, n->f_w[2], n->f_b[2], C, 3, 1, 1, a, &h3, &w3);
    lrelu(a, (long)C * h3 * w3, 0.2);
    conv2d(a, C, h3, w3, n->f_w[3], n->f_b[3], C, 3, 1, 1, b, &h4, &w4);
    free(a);
    *ph = h4;
    *pw = w4;
    return b;
}

/* Refinement.forward -- stereonet.py:1138-1151 */
static void refinement(const net_t *n, int lv, const double *disp,
                       const double *guide, int H, int W, double *out) {
    long HW = (long)H * W;
    int Rc = n->Rc;
    double *x = (double *)malloc(sizeof(double) * 2 * HW);
    double *a = (double *)malloc(sizeof(double) * Rc * HW);
    double *b = (double *)malloc(sizeof(double) * Rc * HW);
    memcpy(x, disp, sizeof(double) * HW);
    memcpy(x + HW, guide, sizeof(double) * HW);
    const double *cur = x;
    int prev = 2, oh, ow;
    double *dst = a;
    for (int i = 0; i < n->ndil; i++) {
        conv2d(cur, prev, H, W, n->r_w[lv][i], n->r_b[lv][i], Rc, 3, 1,
               n->dil[i], dst, &oh, &ow);
        lrelu(dst, Rc * HW, 0.2);
        cur = dst;
        dst = (dst == a) ? b : a;
        prev = Rc;
    }
    double *res = (double *)malloc(sizeof(double) * HW);
    conv2d(cur, prev, H, W, n->r_w[lv][n->ndil], n->r_b[lv][n->ndil], 1, 3, 1,
           1, res, &oh, &ow);
    for (long i = 0; i < HW; i++) {
        double v = disp[i] + res[i];
        out[i] = v > 0.0 ? v : v * 0.0;
    }
    free(x); free(a); free(b); free(res);
}

/* StereoNet.forward -- stereonet.py:1203-1233.  Note the (H, W) order. */
int orc_stereonet_forward(const int *arch, const double *params,
                          const double *left, const double *right, int H, int W,
                          const double *guide_half, const double *guide_full,
                          double *d0, double *d1, double *d2, int *ph, int *pw) {
    net_t n;
    if (net_bind(arch, params, &n) != ORC_OK) return ORC_EBADARG;
    int h, w;
    {
        int qh = ((H - 1) / 2 + 1 - 1) / 2 + 1, qw = ((W - 1) / 2 + 1 - 1) / 2 + 1;
        /* CostVolume.invalid_mask (stereonet.py:837-839) indexes past the end
         * of its list, and the reference raises IndexError, when the quarter
         * width is at most D-2. */
        if (qw <= n.D - 2 || qh < 1) return ORC_EBADARG;
    }
    double *fl = feature_net(&n, left, H, W, &h, &w);
    double *fr = feature_net(&n, right, H, W, &h, &w);
    long hw = (long)h * w, DHW = (long)n.D * hw;
    double *vol = (double *)malloc(sizeof(double) * n.C * DHW);
    cost_volume(fl, fr, n.C, n.D, h, w, vol);
    double *t1 = (double *)malloc(sizeof(double) * n.Cm * DHW);
    double *t2 = (double *)malloc(sizeof(double) * n.Cm * DHW);
    conv3d(vol, n.C, n.D, h, w, n.c_w[0], n.c_b[0], n.Cm, 3, t1);
    lrelu(t1, n.Cm * DHW, 0.2);
    conv3d(t1, n.Cm, n.D, h, w, n.c_w[1], n.c_b[1], n.Cm, 3, t2);
    lrelu(t2, n.Cm * DHW, 0.2);
    conv3d(t2, n.Cm, n.D, h, w, n.c_w[2], n.c_b[2], 1, 3, t1);
    soft_argmin(t1, n.D, h, w, d0);
    int H2 = H / 2, W2 = W / 2;
    long HW2 = (long)H2 * W2, HW = (long)H * W;
    double *up = (double *)malloc(sizeof(double) * (HW > HW2 ? HW : HW2));
    bilinear(d0, 1, h, w, H2, W2, up);
    for (long i = 0; i < HW2; i++) up[i] = up[i] * 2.0;
    refinement(&n, 0, up, guide_half, H2, W2, d1);
    bilinear(d1, 1, H2, W2, H, W, up);
    for (long i = 0; i < HW; i++) up[i] = up[i] * 2.0;
    refinement(&n, 1, up, guide_full, H, W, d2);
    free(fl); free(fr); free(vol); free(t1); free(t2); free(up);
    if (ph) *ph = h;
    if (pw) *pw = w;
    return ORC_OK;
}

/* predict -- stereonet.py:5891-5897 */
int orc_predict(const int *arch, const double *params, const double *left,
                const double *right, int W, int H, double *out) {
    int H2 = H / 2, W2 = W / 2;
    int eh = (H - 1) / 2 + 1, ew = (W - 1) / 2 + 1;
    int qh = (eh - 1) / 2 + 1, qw = (ew - 1) / 2 + 1;
    double *gh = (double *)malloc(sizeof(double) * ((long)H2 * W2 + 1));
    double *d0 = (double *)malloc(sizeof(double) * (long)qh * qw);
    double *d1 = (double *)malloc(sizeof(double) * ((long)H2 * W2 + 1));
    orc_avgpool2(left, 1, H, W, gh);
    int rc = orc_stereonet_forward(arch, params, left, right, H, W, gh, left,
                                   d0, d1, out, NULL, NULL);
    free(gh); free(d0); free(d1);
    return rc;
}

/* predict_at_scale -- stereonet.py:3932-3960.  disp_work must hold W*H. */
int orc_predict_at_scale(const int *arch, const double *params,
                         const double *left, const double *right, int W, int H,
                         int work_width, double *disp_full, double *disp_work,
                         int *pWw, int *pHw) {
    if (work_width >= W) {
        int rc = orc_predict(arch, params, left, right, W, H, disp_full);
        memcpy(disp_work, disp_full, sizeof(double) * (long)W * H);
        *pWw = W;
        *pHw = H;
        return rc;
    }
    double scale = work_width / (double)W;
    int Ww = work_width;
    int Hw = (int)(H * scale + 0.5);
    if (Hw < 8) Hw = 8;
    long n = (long)Ww * Hw;
    double *lw = (double *)malloc(sizeof(double) * n);
    double *rw = (double *)malloc(sizeof(double) * n);
    orc_resize(left, W, H, Ww, Hw, lw);
    orc_resize(right, W, H, Ww, Hw, rw);
    int rc = orc_predict(arch, params, lw, rw, Ww, Hw, disp_work);
    orc_resize(disp_work, Ww, Hw, W, H, disp_full);
    double inv = 1.0 / scale;
    for (long i = 0; i < (long)W * H; i++) disp_full[i] = disp_full[i] * inv;
    free(lw); free(rw);
    *pWw = Ww;
    *pHw = Hw;
    return rc;
}

static int cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* _peak -- stereonet.py:3866-3869 */
double orc_peak(const double *disp, long n, double q) {
    double *s = (double *)malloc(sizeof(double) * n);
    memcpy(s, disp, sizeof(double) * n);
    qsort(s, n, sizeof(double), cmp_double);
    double v = s[(long)(n * q)];
    free(s);
    return v > 0.5 ? v : 0.5;
}

static int width_for(int W, double target_peak, int max_width, double pk) {
    double m = pk > 1.0e-6 ? pk : 1.0e-6;          /* fmax(pk, 1e-6) */
    int w = (int)(W * target_peak / m + 0.5);
    if (w > W) w = W;
    if (w > max_width) w = max_width;
    if (w < 48) w = 48;
    return w;
}

/* predict_auto -- stereonet.py:3872-3929.  Returns the number of network
 * passes after the probe in *passes_run (for tests). */
int orc_predict_auto(const int *arch, const double *params, const double *left,
                     const double *right, int W, int H, double target_peak,
                     int probe_width, int max_width, int passes,
                     double *disp_full, double *disp_work, int *pWw, int *pHw,
                     int *work_trace) {
    int pw = probe_width < W ? probe_width : W;
    int ph = (int)(H * pw / (double)W + 0.5);   /* H*pw is an int product */
    if (ph < 8) ph = 8;
    long pn = (long)pw * ph;
    double *lp = (double *)malloc(sizeof(double) * pn);
    double *rp = (double *)malloc(sizeof(double) * pn);
    double *dp = (double *)malloc(sizeof(double) * pn);
    orc_resize(left, W, H, pw, ph, lp);
    orc_resize(right, W, H, pw, ph, rp);
    orc_predict(arch, params, lp, rp, pw, ph, dp);
    double peak = orc_peak(dp, pn, 0.95) * (W / (double)pw);
    free(lp); free(rp); free(dp);
    int work = width_for(W, target_peak, max_width, peak);
    int ntrace = 0;
    if (work_trace) work_trace[ntrace++] = work;
    int rc = orc_predict_at_scale(arch, params, left, right, W, H, work,
                                  disp_full, disp_work, pWw, pHw);
    for (int it = 0; it < passes - 1; it++) {
        double np_ = orc_peak(disp_full, (long)W * H, 0.95);
        int nw = width_for(W, target_peak, max_width, np_);
        if (abs(nw - work) <= 0.08 * work) break;
        work = nw;
        if (work_trace) work_trace[ntrace++] = work;
        rc = orc_predict_at_scale(arch, params, left, right, W, H, work,
                                  disp_full, disp_work, pWw, pHw);
    }
    if (work_trace) work_trace[ntrace] = 0;
    return rc;
}

/* ------------------------------------------------------------------------
 * Full-resolution refinement -- stereonet.py:5115-5391
 * ---------------------------------------------------------------------- */

/* census -- stereonet.py:5115-5142.  First offset ends in the top bit. */
int orc_census(const double *img, int W, int H, int rx, int ry, uint64_t *out) {
    int nb = (2 * rx + 1) * (2 * ry + 1) - 1;
    if (nb > 64 || rx < 0 || ry < 0) return ORC_EBADARG;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            double c = img[(long)y * W + x];
            uint64_t s = 0;
            for (int dy = -ry; dy <= ry; dy++) {
                for (int dx = -rx; dx <= rx; dx++) {
                    if (!dx && !dy) continue;
                    int xx = x + dx, yy = y + dy;
                    if (xx < 0) xx = 0; else if (xx >= W) xx = W - 1;
                    if (yy < 0) yy = 0; else if (yy >= H) yy = H - 1;
                    s = s + s;
                    if (img[(long)yy * W + xx] < c) s += 1;
                }
            }
            out[(long)y * W + x] = s;
        }
    }
    return ORC_OK;
}

/* band_costs -- stereonet.py:5156-5189.  C [N][K]. */
void orc_band_costs(const uint64_t *cl, const uint64_t *cr, const double *gl,
                    const double *gr, const int64_t *base, int W, int H, int R,
                    double ad_weight, double ad_trunc, double invalid,
                    const double *prior, double prior_w, double prior_t,
                    double *C) {
    int K = 2 * R + 1;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++) {
        long row = (long)y * W;
        for (int x = 0; x < W; x++) {
            long p = row + x;
            int64_t b = base[p] - R;
            uint64_t a = cl[p];
            double il = gl[p];
            long o = p * K;
            for (int k = 0; k < K; k++) {
                C[o + k] = invalid;
                int64_t xr = x - (b + k);
                if (b + k < 0 || xr < 0 || xr >= W) continue;
                long q = row + xr;
                double ad = il - gr[q];
                if (ad < 0) ad = -ad;
                ad = ad * 255.0;
                if (ad > ad_trunc) ad = ad_trunc;
                double c = (double)__builtin_popcountll(a ^ cr[q]) + ad_weight * ad;
                if (prior_w > 0.0) {
                    double e = (double)(b + k) - prior[p];
                    if (e < 0) e = -e;
                    if (e > prior_t) e = prior_t;
                    c += prior_w * e;
                }
                C[o + k] = c;
            }
        }
    }
}

/* One pixel of _aggregate_path (stereonet.py:5207-5237).  Lq/mq describe
 * the predecessor; Lq == NULL means it lies outside the image. */
static inline double agg_pixel(const double *Cp, const double *Lq, double mq,
                               long shift, int K, double P1, double P2,
                               double *Lp) {
    double m = 1.0e30;
    if (!Lq) {
        for (int k = 0; k < K; k++) {
            double v = Cp[k];
            Lp[k] = v;
            if (v < m) m = v;
        }
        return m;
    }
    for (int k = 0; k < K; k++) {
        long kq = k + shift;
        double best = mq + P2;
        if (0 <= kq && kq < K) {
            double v = Lq[kq];
            if (v < best) best = v;
        }
        if (0 <= kq - 1 && kq - 1 < K) {
            double v = Lq[kq - 1] + P1;
            if (v < best) best = v;
        }
        if (0 <= kq + 1 && kq + 1 < K) {
            double v = Lq[kq + 1] + P1;
            if (v < best) best = v;
        }
        double v = Cp[k] + best - mq;
        Lp[k] = v;
        if (v < m) m = v;
    }
    return m;
}

/* _aggregate_path -- stereonet.py:5192-5241, S += L for direction (dx, dy).
 * The recurrence only reads the predecessor p - (dx, dy), so the sweep keeps
 * one row (dy != 0) or one pixel (dy == 0) of L and adds into S as it goes;
 * S still receives the paths one after another, in call order. */
void orc_aggregate_path(const double *C, const int64_t *base, int W, int H,
                        int K, double P1, double P2, int dx, int dy, double *S) {
    if (dy == 0) {
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; y++) {
            double *Lq = (double *)malloc(sizeof(double) * K);
            double *Lp = (double *)malloc(sizeof(double) * K);
            double mq = 0.0;
            for (int i = 0; i < W; i++) {
                int x = dx >= 0 ? i : W - 1 - i;
                long p = (long)y * W + x;
                int qx = x - dx;
                int outside = qx < 0 || qx >= W;
                long shift = outside ? 0 : (long)(base[p] - base[p - dx]);
                mq = agg_pixel(C + p * K, outside ? NULL : Lq, mq, shift, K, P1,
                               P2, Lp);
                for (int k = 0; k < K; k++) S[p * K + k] += Lp[k];
                double *t = Lq; Lq = Lp; Lp = t;
            }
            free(Lq); free(Lp);
        }
        return;
    }
    double *Lprev = (double *)malloc(sizeof(double) * (long)W * K);
    double *Lcur = (double *)malloc(sizeof(double) * (long)W * K);
    double *mprev = (double *)malloc(sizeof(double) * W);
    double *mcur = (double *)malloc(sizeof(double) * W);
    for (int j = 0; j < H; j++) {
        int y = dy >= 0 ? j : H - 1 - j;
        int qy = y - dy;
#pragma omp parallel for schedule(static)
        for (int x = 0; x < W; x++) {
            long p = (long)y * W + x;
            int qx = x - dx;
            int outside = qx < 0 || qx >= W || qy < 0 || qy >= H;
            long shift = 0;
            const double *Lq = NULL;
            double mq = 0.0;
            if (!outside) {
                long q = (long)qy * W + qx;
                shift = (long)(base[p] - base[q]);
                Lq = Lprev + (long)qx * K;
                mq = mprev[qx];
            }
            mcur[x] = agg_pixel(C + p * K, Lq, mq, shift, K, P1, P2,
                                Lcur + (long)x * K);
            for (int k = 0; k < K; k++) S[p * K + k] += Lcur[(long)x * K + k];
        }
        double *t = Lprev; Lprev = Lcur; Lcur = t;
        t = mprev; mprev = mcur; mcur = t;
    }
    free(Lprev); free(Lcur); free(mprev); free(mcur);
}

static int base_from_disp(const double *disp0, long N, int64_t *base) {
    for (long i = 0; i < N; i++) {
        double t = disp0[i] + 0.5;
        if (!(t > -9.0e15 && t < 9.0e15)) return ORC_ERANGE;   /* NaN/inf/huge */
        int64_t v = (int64_t)t;                                /* int(): toward zero */
        base[i] = v > 0 ? v : 0;
    }
    return ORC_OK;
}

/* refine_fullres -- stereonet.py:5244-5305.  conf may be NULL. */
int orc_refine_fullres(const double *left, const double *right,
                       const double *disp0, int W, int H, int R, double P1,
                       double P2, double ad_weight, double ad_trunc, int paths,
                       double uniq, int rx, int ry, double prior_w,
                       double prior_t, double *out, double *conf) {
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
    int rc = base_from_disp(disp0, N, base);
    if (rc) { free(base); free(cl); free(cr); free(C); free(S); return rc; }
    orc_census(left, W, H, rx, ry, cl);
    orc_census(right, W, H, rx, ry, cr);
    double invalid = nbits + ad_weight * ad_trunc + prior_w * prior_t + 4.0;
    orc_band_costs(cl, cr, left, right, base, W, H, R, ad_weight, ad_trunc,
                   invalid, disp0, prior_w, prior_t, C);
    static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1},
                                   {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
    int nd = paths == 8 ? 8 : 4;
    for (int d = 0; d < nd; d++)
        orc_aggregate_path(C, base, W, H, K, P1, P2, dirs[d][0], dirs[d][1], S);
#pragma omp parallel for schedule(static)
    for (long p = 0; p < N; p++) {
        long o = p * K;
        int bk = 0;
        double bv = S[o];
        for (int k = 1; k < K; k++) {
            if (S[o + k] < bv) { bv = S[o + k]; bk = k; }
        }
        if (bk == 0 || bk == K - 1) {
            out[p] = disp0[p];
            if (conf) conf[p] = 0.0;
            continue;
        }
        double sv = 1.0e30;
        for (int k = 0; k < K; k++) {
            if (k < bk - 1 || k > bk + 1) {
                if (S[o + k] < sv) sv = S[o + k];
            }
        }
        double c = sv < 1.0e29 ? (sv - bv) / (bv + 1.0e-6) : 1.0;
        if (conf) conf[p] = c;
        if (c < uniq) { out[p] = disp0[p]; continue; }
        double a = S[o + bk - 1];
        double b = S[o + bk + 1];
        double den = a - 2.0 * bv + b;
        double off = 0.0;
        if (den > 1.0e-9) off = 0.5 * (a - b) / den;
        out[p] = (double)(base[p] - R + bk) + off;
    }
    free(base); free(cl); free(cr); free(C); free(S);
    return ORC_OK;
}

/* _mirror1 -- stereonet.py:5308-5314 */
void orc_mirror(const double *img, int W, int H, double *out) {
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            out[(long)y * W + x] = img[(long)y * W + W - 1 - x];
}

/* left_to_right -- stereonet.py:5317-5340 */
int orc_left_to_right(const double *dl, int W, int H, double *dr) {
    for (long i = 0; i < (long)W * H; i++) dr[i] = -1.0;
    for (int y = 0; y < H; y++) {
        long r = (long)y * W;
        for (int x = 0; x < W; x++) {
            double d = dl[r + x];
            double t = x - d + 0.5;
            if (!(t > -9.0e15 && t < 9.0e15)) return ORC_ERANGE;
            int64_t xr = (int64_t)t;
            if (0 <= xr && xr < W && d > dr[r + xr]) dr[r + xr] = d;
        }
        for (int x = 0; x < W; x++) {
            if (dr[r + x] < 0.0) {
                int a = x - 1;
                while (a >= 0 && dr[r + a] < 0.0) a--;
                int b = x + 1;
                while (b < W && dr[r + b] < 0.0) b++;
                double va = a >= 0 ? dr[r + a] : 1.0e9;
                double vb = b < W ? dr[r + b] : 1.0e9;
                double v = va < vb ? va : vb;
                dr[r + x] = v < 1.0e8 ? v : 0.0;
            }
        }
    }
    return ORC_OK;
}

/* lr_refine -- stereonet.py:5343-5391.  status: 0 ok, 1 occluded, 2 mismatch */
int orc_lr_refine(const double *left, const double *right, const double *disp0,
                  int W, int H, double tol, int R, double P1, double P2,
                  double ad_weight, double ad_trunc, int paths, double uniq,
                  int rx, int ry, double prior_w, double prior_t, double *out,
                  int32_t *status) {
    long N = (long)W * H;
    double *dl = (double *)malloc(sizeof(double) * N);
    double *d0r = (double *)malloc(sizeof(double) * N);
    double *m1 = (double *)malloc(sizeof(double) * N);
    double *m2 = (double *)malloc(sizeof(double) * N);
    double *m3 = (double *)malloc(sizeof(double) * N);
    double *drm = (double *)malloc(sizeof(double) * N);
    double *dr = (double *)malloc(sizeof(double) * N);
    int rc = orc_refine_fullres(left, right, disp0, W, H, R, P1, P2, ad_weight,
                                ad_trunc, paths, uniq, rx, ry, prior_w, prior_t,
                                dl, NULL);
    if (!rc) rc = orc_left_to_right(disp0, W, H, d0r);
    if (!rc) {
        orc_mirror(right, W, H, m1);
        orc_mirror(left, W, H, m2);
        orc_mirror(d0r, W, H, m3);
        rc = orc_refine_fullres(m1, m2, m3, W, H, R, P1, P2, ad_weight,
                                ad_trunc, paths, uniq, rx, ry, prior_w, prior_t,
                                drm, NULL);
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
        if (status[i] == 2) out[i] = disp0[i];
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
            out[r + x] = v < 1.0e8 ? v : disp0[r + x];
        }
    }
    free(dl); free(d0r); free(m1); free(m2); free(m3); free(drm); free(dr);
    return ORC_OK;
}

/* ----------------------------------------------------------------------
 * The rest of refine_disparity (stereonet.py:5865-5883): SLIC superpixels,
 * plane_snap (RANSAC + least-squares plane per segment) and median_filter.
 * ---------------------------------------------------------------------- */

/* slic -- stereonet.py:5394-5455.  m2 is (compactness / step) ** 2 as the
 * caller's libm pow computes it (CPython's float ** int calls pow()). */
int orc_slic(const double *rgb, int W, int H, int step, double m2, int iters,
             int32_t *lab, int *nseg) {
    if (W < 1 || H < 1 || step < 1) return ORC_EBADARG;
    int ncx = 0, ncy = 0;
    for (int x = step / 2; x < W; x += step) ncx++;
    for (int y = step / 2; y < H; y += step) ncy++;
    int nc = ncx * ncy;
    long N = (long)W * H;
    double *cs = (double *)malloc(sizeof(double) * 5 * (nc > 0 ? nc : 1));
    double *dist = (double *)malloc(sizeof(double) * N);
    double *acc = (double *)malloc(sizeof(double) * 6 * (nc > 0 ? nc : 1));
    if (!cs || !dist || !acc) { free(cs); free(dist); free(acc); return ORC_ENOMEM; }
    int k = 0;
    for (int y = step / 2; y < H; y += step)
        for (int x = step / 2; x < W; x += step) {
            long i = (long)y * W + x;
            cs[5 * k + 0] = rgb[3 * i] * 255.0;
            cs[5 * k + 1] = rgb[3 * i + 1] * 255.0;
            cs[5 * k + 2] = rgb[3 * i + 2] * 255.0;
            cs[5 * k + 3] = (double)x;
            cs[5 * k + 4] = (double)y;
            k++;
        }
    for (long i = 0; i < N; i++) lab[i] = -1;
    for (int it = 0; it < iters; it++) {
        for (long i = 0; i < N; i++) dist[i] = 1.0e30;
        for (int ci = 0; ci < nc; ci++) {
            double cr = cs[5 * ci], cg = cs[5 * ci + 1], cb = cs[5 * ci + 2];
            double cx = cs[5 * ci + 3], cy = cs[5 * ci + 4];
            int x0 = (int)cx - step, x1 = (int)cx + step;
            int y0 = (int)cy - step, y1 = (int)cy + step;
            if (x0 < 0) x0 = 0;
            if (y0 < 0) y0 = 0;
            if (x1 >= W) x1 = W - 1;
            if (y1 >= H) y1 = H - 1;
            for (int yy = y0; yy <= y1; yy++) {
                double dy = yy - cy;
                for (int xx = x0; xx <= x1; xx++) {
                    long i = (long)yy * W + xx;
                    double a = rgb[3 * i] * 255.0 - cr;
                    double b = rgb[3 * i + 1] * 255.0 - cg;
                    double c = rgb[3 * i + 2] * 255.0 - cb;
                    double dx = xx - cx;
                    double dd = a * a + b * b + c * c + m2 * (dx * dx + dy * dy);
                    if (dd < dist[i]) { dist[i] = dd; lab[i] = ci; }
                }
            }
        }
        for (int ci = 0; ci < 6 * nc; ci++) acc[ci] = 0.0;
        for (long i = 0; i < N; i++) {
            int l = lab[i];
            if (l < 0) continue;
            double *a = acc + 6 * l;
            a[0] += rgb[3 * i];
            a[1] += rgb[3 * i + 1];
            a[2] += rgb[3 * i + 2];
            a[3] += (double)(i % W);
            a[4] += (double)(i / W);
            a[5] += 1.0;
        }
        for (int ci = 0; ci < nc; ci++) {
            double *a = acc + 6 * ci;
            if (a[5] != 0.0) {
                double n = a[5];
                cs[5 * ci + 0] = a[0] / n * 255.0;
                cs[5 * ci + 1] = a[1] / n * 255.0;
                cs[5 * ci + 2] = a[2] / n * 255.0;
                cs[5 * ci + 3] = a[3] / n;
                cs[5 * ci + 4] = a[4] / n;
            }
        }
    }
    *nseg = nc;
    free(cs); free(dist); free(acc);
    return ORC_OK;
}

/* _solve3 -- stereonet.py:5458-5469; returns 0 when |det| < 1e-9. */
static int solve3(const double A[3][3], const double bv[3], double out[3]) {
    double a = A[0][0], bb = A[0][1], c = A[0][2];
    double d = A[1][0], e = A[1][1], f = A[1][2];
    double g = A[2][0], h = A[2][1], k = A[2][2];
    double det = a * (e * k - f * h) - bb * (d * k - f * g) + c * (d * h - e * g);
    if (fabs(det) < 1.0e-9) return 0;
    out[0] = (bv[0] * (e * k - f * h) - bb * (bv[1] * k - f * bv[2]) +
              c * (bv[1] * h - e * bv[2])) / det;
    out[1] = (a * (bv[1] * k - f * bv[2]) - bv[0] * (d * k - f * g) +
              c * (d * bv[2] - bv[1] * g)) / det;
    out[2] = (a * (e * bv[2] - bv[1] * h) - bb * (d * bv[2] - bv[1] * g) +
              bv[0] * (d * h - e * g)) / det;
    return 1;
}

/* _lsq_plane -- stereonet.py:5472-5502 (sequential sums in list order). */
static void lsq_plane(const long *idx, long n, const double *disp, int W, double out[3]) {
    double nn = (double)n, sx = 0.0, sy = 0.0, sd = 0.0;
    for (long j = 0; j < n; j++) sx += (double)(idx[j] % W);
    for (long j = 0; j < n; j++) sy += (double)(idx[j] / W);
    for (long j = 0; j < n; j++) sd += disp[idx[j]];
    double mx = sx / nn, my = sy / nn, md = sd / nn;
    double sxx = 0.0, sxy = 0.0, syy = 0.0, sxd = 0.0, syd = 0.0;
    for (long j = 0; j < n; j++) {
        double u = (double)(idx[j] % W) - mx;
        double v = (double)(idx[j] / W) - my;
        double w = disp[idx[j]] - md;
        sxx += u * u;
        sxy += u * v;
        syy += v * v;
        sxd += u * w;
        syd += v * w;
    }
    double det = sxx * syy - sxy * sxy;
    if (fabs(det) < 1.0e-9) { out[0] = 0.0; out[1] = 0.0; out[2] = md; return; }
    double a = (sxd * syy - syd * sxy) / det;
    double b = (syd * sxx - sxd * sxy) / det;
    out[0] = a; out[1] = b; out[2] = md - a * mx - b * my;
}

static inline uint32_t xorshift32(uint32_t s) {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return s;
}

/* plane_snap -- stereonet.py:5505-5563.  valid may be NULL. */
int orc_plane_snap(const double *disp, const double *rgb, int W, int H, const uint8_t *valid,
                   int step, double m2, double thr, double min_inl, int trials,
                   uint32_t seed, double *out) {
    long N = (long)W * H;
    int32_t *lab = (int32_t *)malloc(sizeof(int32_t) * N);
    long *order = (long *)malloc(sizeof(long) * N);
    long *pts = (long *)malloc(sizeof(long) * N);
    if (!lab || !order || !pts) { free(lab); free(order); free(pts); return ORC_ENOMEM; }
    int nseg = 0;
    int rc = orc_slic(rgb, W, H, step, m2, 5, lab, &nseg);
    if (rc) { free(lab); free(order); free(pts); return rc; }
    long *start = (long *)calloc((size_t)nseg + 1, sizeof(long));
    long *fill = (long *)calloc((size_t)nseg + 1, sizeof(long));
    for (long i = 0; i < N; i++) if (lab[i] >= 0) start[lab[i] + 1]++;
    for (int g = 0; g < nseg; g++) start[g + 1] += start[g];
    for (long i = 0; i < N; i++)
        if (lab[i] >= 0) order[start[lab[i]] + fill[lab[i]]++] = i;     /* index order */
    for (long i = 0; i < N; i++) out[i] = disp[i];
    uint32_t s = seed;
    for (int g = 0; g < nseg; g++) {
        const long *grp = order + start[g];
        long gn = start[g + 1] - start[g], n = 0;
        for (long j = 0; j < gn; j++)
            if (!valid || valid[grp[j]]) pts[n++] = grp[j];
        if (n < 12) continue;
        int have = 0;
        long bestc = -1;
        double best[3] = {0.0, 0.0, 0.0};
        for (int t = 0; t < trials; t++) {
            long tri[3];
            for (int u = 0; u < 3; u++) {
                s = xorshift32(s);
                tri[u] = pts[s % (uint32_t)n];
            }
            double A[3][3], bv[3], pl[3];
            for (int u = 0; u < 3; u++) {
                A[u][0] = (double)(tri[u] % W);
                A[u][1] = (double)(tri[u] / W);
                A[u][2] = 1.0;
                bv[u] = disp[tri[u]];
            }
            if (!solve3(A, bv, pl)) continue;
            long cnt = 0;
            for (long j = 0; j < n; j++) {
                long i = pts[j];
                if (fabs(pl[0] * (double)(i % W) + pl[1] * (double)(i / W) + pl[2] - disp[i]) <= thr)
                    cnt++;
            }
            if (cnt > bestc) {
                bestc = cnt;
                best[0] = pl[0]; best[1] = pl[1]; best[2] = pl[2];
                have = 1;
            }
        }
        if (!have || (double)bestc < min_inl * (double)n) continue;
        long ni = 0;
        for (long j = 0; j < n; j++) {
            long i = pts[j];
            if (fabs(best[0] * (double)(i % W) + best[1] * (double)(i / W) + best[2] - disp[i]) <= thr)
                pts[ni++] = i;             /* inliers, in order, compacted in place */
        }
        double pl[3];
        lsq_plane(pts, ni, disp, W, pl);
        for (long j = 0; j < gn; j++) {
            long i = grp[j];
            double v = pl[0] * (double)(i % W) + pl[1] * (double)(i / W) + pl[2];
            if (fabs(v - disp[i]) <= thr || (valid && !valid[i])) out[i] = v > 0.0 ? v : 0.0;
        }
    }
    free(lab); free(order); free(pts); free(start); free(fill);
    return ORC_OK;
}

/* median_filter -- stereonet.py:2231-2259 (upper median of the clipped window). */
int orc_median_filter(const double *disp, int W, int H, int radius, int passes, double *out) {
    long N = (long)W * H;
    int side = 2 * radius + 1;
    double *cur = (double *)malloc(sizeof(double) * N);
    double *vals = (double *)malloc(sizeof(double) * side * side);
    if (!cur || !vals) { free(cur); free(vals); return ORC_ENOMEM; }
    memcpy(cur, disp, sizeof(double) * N);
    for (int p = 0; p < passes; p++) {
        for (int y = 0; y < H; y++) {
            int y0 = y - radius > 0 ? y - radius : 0;
            int y1 = y + radius < H - 1 ? y + radius : H - 1;
            for (int x = 0; x < W; x++) {
                int x0 = x - radius > 0 ? x - radius : 0;
                int x1 = x + radius < W - 1 ? x + radius : W - 1;
                int n = 0;
                for (int yy = y0; yy <= y1; yy++)
                    for (int xx = x0; xx <= x1; xx++) vals[n++] = cur[(long)yy * W + xx];
                for (int a = 1; a < n; a++) {             /* insertion sort */
                    double v = vals[a];
                    int b = a - 1;
                    while (b >= 0 && vals[b] > v) { vals[b + 1] = vals[b]; b--; }
                    vals[b + 1] = v;
                }
                out[(long)y * W + x] = vals[n / 2];
            }
        }
        memcpy(cur, out, sizeof(double) * N);
    }
    if (passes < 1) memcpy(out, disp, sizeof(double) * N);
    free(cur); free(vals);
    return ORC_OK;
}

/* refine_disparity -- stereonet.py:5865-5883.  rgb may be NULL (no planes). */
int orc_refine_disparity(const double *left, const double *right, const double *rgb,
                         const double *disp0, int W, int H, int R, double P1, double P2,
                         int rx, int ry, double tol, int planes, int plane_step, double m2,
                         double plane_thr, double plane_min_inl, double *out,
                         int32_t *status) {
    long N = (long)W * H;
    double *d = (double *)malloc(sizeof(double) * N);
    double *e = (double *)malloc(sizeof(double) * N);
    uint8_t *valid = (uint8_t *)malloc(N);
    if (!d || !e || !valid) { free(d); free(e); free(valid); return ORC_ENOMEM; }
    int rc = orc_lr_refine(left, right, disp0, W, H, tol, R, P1, P2, 0.0, 20.0, 8, 0.0, rx, ry,
                           0.0, 4.0, d, status);
    if (!rc && planes && rgb) {
        for (long i = 0; i < N; i++) valid[i] = status[i] == 0;
        rc = orc_plane_snap(d, rgb, W, H, valid, plane_step, m2, plane_thr, plane_min_inl, 40,
                            12345u, e);
        if (!rc) memcpy(d, e, sizeof(double) * N);
    }
    if (!rc) rc = orc_median_filter(d, W, H, 1, 1, out);
    free(d); free(e); free(valid);
    return rc;
}

/* ----------------------------------------------------------------------
 * Network-level left-right consistency (stereonet.py:4974-5076).
 * ---------------------------------------------------------------------- */

/* lr_consistency -- stereonet.py:4986-5009 */
void orc_lr_consistency(const double *dl, const double *dr, int W, int H, double tol,
                        uint8_t *valid) {
    for (int y = 0; y < H; y++) {
        long row = (long)y * W;
        for (int x = 0; x < W; x++) {
            double d = dl[row + x];
            double xr = x - d;
            valid[row + x] = 1;
            if (xr < 0.0 || xr > W - 1) { valid[row + x] = 0; continue; }
            int x0 = (int)xr;
            int x1 = x0 + 1 < W ? x0 + 1 : x0;
            double f = xr - x0;
            double e = dr[row + x0] * (1.0 - f) + dr[row + x1] * f;
            double diff = d - e;
            if (diff < 0.0) diff = -diff;
            if (diff > tol) valid[row + x] = 0;
        }
    }
}

/* fill_invalid -- stereonet.py:5012-5045 */
void orc_fill_invalid(const double *disp, const uint8_t *valid, int W, int H, double *out) {
    for (long i = 0; i < (long)W * H; i++) out[i] = disp[i];
    for (int y = 0; y < H; y++) {
        long row = (long)y * W;
        int x = 0;
        while (x < W) {
            if (valid[row + x]) { x++; continue; }
            int start = x;
            while (x < W && !valid[row + x]) x++;
            int end = x;
            int hl = start > 0, hr = end < W;
            if (!hl && !hr) continue;
            double fillv;
            if (!hl) fillv = disp[row + end];
            else if (!hr) fillv = disp[row + start - 1];
            else {
                double lv = disp[row + start - 1], rv = disp[row + end];
                fillv = lv < rv ? lv : rv;
            }
            for (int i = start; i < end; i++) out[row + i] = fillv;
        }
    }
}

/* predict_consistent -- stereonet.py:5048-5076.  work_width <= 0: predict_auto
 * with the given target_peak / probe_width / max_width / passes. */
int orc_predict_consistent(const int *arch, const double *params, const double *left,
                           const double *right, int W, int H, int work_width,
                           double target_peak, int probe_width, int max_width, int passes,
                           double tol, double *out, long *kept) {
    long N = (long)W * H;
    double *dl = (double *)malloc(sizeof(double) * N), *dw = (double *)malloc(sizeof(double) * N);
    double *ml = (double *)malloc(sizeof(double) * N), *mr = (double *)malloc(sizeof(double) * N);
    double *drm = (double *)malloc(sizeof(double) * N), *dr = (double *)malloc(sizeof(double) * N);
    uint8_t *valid = (uint8_t *)malloc(N);
    int Ww = 0, Hw = 0, rc;
    if (work_width <= 0)
        rc = orc_predict_auto(arch, params, left, right, W, H, target_peak, probe_width,
                              max_width, passes, dl, dw, &Ww, &Hw, NULL);
    else
        rc = orc_predict_at_scale(arch, params, left, right, W, H, work_width, dl, dw, &Ww, &Hw);
    if (!rc) {
        orc_mirror(left, W, H, ml);
        orc_mirror(right, W, H, mr);
        rc = orc_predict_at_scale(arch, params, mr, ml, W, H, Ww, drm, dw, &Ww, &Hw);
    }
    if (!rc) {
        orc_mirror(drm, W, H, dr);
        orc_lr_consistency(dl, dr, W, H, tol, valid);
        long k = 0;
        for (long i = 0; i < N; i++) k += valid[i];
        *kept = k;
        orc_fill_invalid(dl, valid, W, H, out);
    }
    free(dl); free(dw); free(ml); free(mr); free(drm); free(dr); free(valid);
    return rc;
}
