// sv_train.cu -- StereoNet training on the GPU: train_grads
// (stereonet.py:1619-1653) over a batch of crops and Adam.step (1368-1387),
// the batch gradient being the mean of the per-sample gradients, which is
// what the reference's data-parallel harness computes with one process per
// sample (train_parallel.py:144-156).
//
// FP32 activations and gradients, FP64 parameters, Adam state and weight
// gradient sums.  The forward keeps every activation it needs (after the
// leaky ReLU only: with slope 0.2 or 0, a post-activation value is positive
// exactly when its input is, so it also gives the ReLU derivative).
// Every reduction has a fixed order, so a step is deterministic:
//   * input gradients are gathers (one thread per input element sums its
//     taps), never atomics;
//   * a weight gradient is a sum over (image, pixel) of x * gy: each CTA
//     takes a tile of outputs, stages the input patch and the output
//     gradients in shared memory, and writes per-tile partial sums for every
//     (out channel, in channel, tap) and the bias; a second kernel adds the
//     tiles in order in FP64.
// Layouts are the reference's planar ones with a leading image index; the
// siamese towers run as one batch of 2B images (the B left views, then the
// B right views).

#include <cmath>
#include <cstring>
#include <vector>

#include "sv_common.cuh"
#include "sv_network.cuh"

namespace sv {
namespace {

constexpr int kTR = 4, kTC = 32;   // 2-D tile: 4 rows x 32 columns of outputs
constexpr int kTD = 4;             // 3-D tile: 4 disparities x 1 row x 32 columns
constexpr int kMaxB = 4096;

// ------------------------------------------------------------- forward
template <int IC, int OC, int OCG, int ACT>
__global__ void __launch_bounds__(kTC *kTR)
    k_tconv2d(const float *__restrict__ x, int H, int W, int OH, int OW, int s, int dil,
              const float *__restrict__ w, const float *__restrict__ b, float *__restrict__ y,
              const float *__restrict__ resid, long resid_stride) {
    constexpr int NG = OC / OCG;
    extern __shared__ __align__(16) float tile[];
    __shared__ float sw[OCG * IC * 9];
    __shared__ float sb[OCG];
    const int img = blockIdx.z / NG, og = blockIdx.z - img * NG;
    const int tid = threadIdx.y * kTC + threadIdx.x;
    for (int i = tid; i < OCG * IC * 9; i += kTC * kTR) sw[i] = w[og * OCG * IC * 9 + i];
    if (tid < OCG) sb[tid] = b[og * OCG + tid];
    const long HW = (long)H * W;
    const float *xi = x + (long)img * IC * HW;
    const int ox0 = blockIdx.x * kTC, oy0 = blockIdx.y * kTR;
    const int ix0 = ox0 * s - dil, iy0 = oy0 * s - dil;
    const int th = (kTR - 1) * s + 2 * dil + 1, tw = (kTC - 1) * s + 2 * dil + 1;
    for (int i = tid; i < IC * th * tw; i += kTC * kTR) {
        const int c = i / (th * tw), rem = i - c * th * tw;
        const int ty = rem / tw, tx = rem - ty * tw;
        const int gy = iy0 + ty, gx = ix0 + tx;
        tile[i] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? xi[c * HW + (long)gy * W + gx] : 0.f;
    }
    __syncthreads();
    const int ox = ox0 + threadIdx.x, oy = oy0 + threadIdx.y;
    if (ox >= OW || oy >= OH) return;
    float acc[OCG];
#pragma unroll
    for (int o = 0; o < OCG; ++o) acc[o] = sb[o];
    const int by = threadIdx.y * s, bx = threadIdx.x * s;
#pragma unroll
    for (int c = 0; c < IC; ++c) {
        const float *tc = tile + c * th * tw;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
            const float *row = tc + (by + ky * dil) * tw + bx;
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                const float v = row[kx * dil];
#pragma unroll
                for (int o = 0; o < OCG; ++o)
                    acc[o] = fmaf(v, sw[(o * IC + c) * 9 + ky * 3 + kx], acc[o]);
            }
        }
    }
    const long OHW = (long)OH * OW, oi = (long)oy * OW + ox;
#pragma unroll
    for (int o = 0; o < OCG; ++o) {
        float v = acc[o];
        if (ACT == 1) v = v > 0.f ? v : v * 0.2f;
        if (ACT == 2) {                           // Refinement: relu0(disp + residual)
            v = resid[img * resid_stride + oi] + v;
            v = v > 0.f ? v : v * 0.f;
        }
        y[((long)img * OC + og * OCG + o) * OHW + oi] = v;
    }
}

size_t tconv2d_smem(int IC, int s, int dil) {
    return sizeof(float) * IC * ((kTR - 1) * s + 2 * dil + 1) * ((kTC - 1) * s + 2 * dil + 1);
}

// 3-D convolution, stride 1, same padding, leaky ReLU when ACT: a CTA is
// kTD disparities x 32 columns of one row for OCG output channels.
template <int IC, int OC, int OCG, int ACT>
__global__ void __launch_bounds__(32 * kTD)
    k_tconv3d(const float *__restrict__ x, int D, int h, int w, const float *__restrict__ wt,
              const float *__restrict__ b, float *__restrict__ y) {
    constexpr int NG = OC / OCG;
    __shared__ float sx[IC][kTD + 2][3][34];
    __shared__ float sw[OCG * IC * 27];
    __shared__ float sb[OCG];
    const int bimg = blockIdx.z / NG, og = blockIdx.z - bimg * NG;
    const int nd = (D + kTD - 1) / kTD;
    const int x0 = blockIdx.x * 32, oy = blockIdx.y / nd, d0 = (blockIdx.y - oy * nd) * kTD;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int i = tid; i < OCG * IC * 27; i += 32 * kTD) sw[i] = wt[og * OCG * IC * 27 + i];
    if (tid < OCG) sb[tid] = b[og * OCG + tid];
    const long hw = (long)h * w, total = (long)D * hw;
    const float *xb = x + (long)bimg * IC * total;
    constexpr int PLANE = (kTD + 2) * 3 * 34;
    for (int i = tid; i < IC * PLANE; i += 32 * kTD) {
        const int c = i / PLANE, rem = i - c * PLANE;
        const int dz = rem / 102, rem2 = rem - dz * 102, r = rem2 / 34, j = rem2 - r * 34;
        const int dd = d0 - 1 + dz, yy = oy - 1 + r, xx = x0 - 1 + j;
        sx[c][dz][r][j] = (dd >= 0 && dd < D && yy >= 0 && yy < h && xx >= 0 && xx < w)
                              ? xb[c * total + dd * hw + yy * w + xx]
                              : 0.f;
    }
    __syncthreads();
    const int ox = x0 + threadIdx.x, od = d0 + threadIdx.y;
    if (ox >= w || od >= D) return;
    float acc[OCG];
#pragma unroll
    for (int o = 0; o < OCG; ++o) acc[o] = sb[o];
#pragma unroll
    for (int c = 0; c < IC; ++c)
#pragma unroll
        for (int kd = 0; kd < 3; ++kd)
#pragma unroll
            for (int ky = 0; ky < 3; ++ky) {
                const float *row = &sx[c][threadIdx.y + kd][ky][threadIdx.x];
#pragma unroll
                for (int kx = 0; kx < 3; ++kx) {
                    const float v = row[kx];
#pragma unroll
                    for (int o = 0; o < OCG; ++o)
                        acc[o] = fmaf(v, sw[(o * IC + c) * 27 + kd * 9 + ky * 3 + kx], acc[o]);
                }
            }
    const long idx = (long)od * hw + (long)oy * w + ox;
#pragma unroll
    for (int o = 0; o < OCG; ++o) {
        float v = acc[o];
        if (ACT) v = v > 0.f ? v : v * 0.2f;
        y[((long)bimg * OC + og * OCG + o) * total + idx] = v;
    }
}

// CostVolume.forward (771-799): vol[b][c][d][y][x] = |fl - fr(x - d)|, 2.0
// where x - d < 0; fl is image b of f, fr image B + b.
__global__ void k_tcostvol(const float *__restrict__ f, int B, int C, int D, int h, int w,
                           float *__restrict__ vol) {
    const long hw = (long)h * w, n = (long)B * C * D * hw;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % w), y = (int)((i / w) % h), d = (int)((i / hw) % D);
        const int c = (int)((i / (hw * D)) % C), b = (int)(i / (hw * D * C));
        if (x - d < 0) {
            vol[i] = 2.0f;
            continue;
        }
        const float l = f[((long)b * C + c) * hw + (long)y * w + x];
        const float r = f[((long)(B + b) * C + c) * hw + (long)y * w + x - d];
        vol[i] = fabsf(l - r);
    }
}

// SoftArgmin.forward with CostVolume.invalid_mask (858-885, 827-840): probs
// and disparity, FP32 with max-subtraction.
__global__ void k_tsoftargmin(const float *__restrict__ cost, int B, int D, int h, int w,
                              float *__restrict__ probs, float *__restrict__ d0) {
    const long hw = (long)h * w;
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= B * hw) return;
    const int b = (int)(i / hw);
    const long p = i - b * hw;
    const int x = (int)(p % w);
    const float *cb = cost + (long)b * D * hw + p;
    float *pb = probs + (long)b * D * hw + p;
    float c[16];
    float best = -INFINITY;
    for (int d = 0; d < D; ++d) {
        c[d] = cb[d * hw] + ((d >= 1 && x < d) ? 8.0f : 0.0f);
        best = fmaxf(best, -c[d]);
    }
    float total = 0.f;
    for (int d = 0; d < D; ++d) {
        c[d] = expf(-c[d] - best);
        total += c[d];
    }
    const float inv = 1.0f / total;
    float acc = 0.f;
    for (int d = 0; d < D; ++d) {
        const float pr = c[d] * inv;
        pb[d * hw] = pr;
        acc += (float)d * pr;
    }
    d0[i] = acc;
}

// A refinement level's input [b][2][H2][W2]: 2 * bilinear(prev), guide.
__global__ void k_tupcat(const float *__restrict__ prev, int B, int h, int w, int H2, int W2,
                         const float *__restrict__ guide, float *__restrict__ rin) {
    const long n2 = (long)H2 * W2;
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= B * n2) return;
    const int b = (int)(i / n2);
    const long p = i - b * n2;
    const int oy = (int)(p / W2), ox = (int)(p - (long)oy * W2);
    const Taps t = bilinear_taps(oy, ox, h, w, H2, W2);
    const float *s = prev + (long)b * h * w;
    const float v = s[t.i00] * (float)t.w00 + s[t.i01] * (float)t.w01 + s[t.i10] * (float)t.w10 +
                    s[t.i11] * (float)t.w11;
    rin[(long)b * 2 * n2 + p] = v * 2.0f;
    rin[(long)b * 2 * n2 + n2 + p] = guide[(long)b * n2 + p];
}

// build_targets (1572-1611) one level down: disparity 0.25 * sum * 0.5,
// valid = all four, guide (optional) 0.25 * sum.
__global__ void k_tpool(const float *__restrict__ d, const uint8_t *__restrict__ v,
                        const float *__restrict__ g, int B, int H, int W, float *__restrict__ dd,
                        uint8_t *__restrict__ vv, float *__restrict__ gg) {
    const int H2 = H / 2, W2 = W / 2;
    const long n2 = (long)H2 * W2;
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= B * n2) return;
    const int b = (int)(i / n2);
    const long p = i - b * n2;
    const int y = (int)(p / W2), x = (int)(p - (long)y * W2);
    const long r0 = (long)b * H * W + (long)(2 * y) * W + 2 * x, r1 = r0 + W;
    dd[i] = 0.25f * (d[r0] + d[r0 + 1] + d[r1] + d[r1 + 1]) * 0.5f;
    vv[i] = (v[r0] && v[r0 + 1] && v[r1] && v[r1 + 1]) ? 1 : 0;
    if (g) gg[i] = 0.25f * (g[r0] + g[r0 + 1] + g[r1] + g[r1 + 1]);
}

// disparity_ce's target (1274-1323): fexp(-e^2 / (2 sigma^2)) is exactly 0
// below -700, so a pixel whose every e^2 / (2 sigma^2) exceeds 700 has
// qsum == 0 and is skipped.  Decided in FP64 as the reference does.
__device__ __forceinline__ bool ce_counted(float dg, int D) {
    const double inv2s2 = 1.0 / (2.0 * 0.8 * 0.8);
    for (int d = 0; d < D; ++d) {
        const double e = (double)d - (double)dg;
        if (!(e * e * inv2s2 > 700.0)) return true;
    }
    return false;
}

// Per-sample counts: valid pixels at 1/4, 1/2, 1/1 and the CE count.
__global__ void __launch_bounds__(256)
    k_tcounts(const uint8_t *__restrict__ vq, const uint8_t *__restrict__ vh,
              const uint8_t *__restrict__ vf, const float *__restrict__ dq, long n4, long n2,
              long n1, int D, int *__restrict__ counts) {
    __shared__ int s[4][256];
    const int b = blockIdx.x, t = threadIdx.x;
    int c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (long i = t; i < n4; i += 256) {
        if (vq[b * n4 + i]) {
            ++c0;
            if (ce_counted(dq[b * n4 + i], D)) ++c3;
        }
    }
    for (long i = t; i < n2; i += 256) c1 += vh[b * n2 + i] != 0;
    for (long i = t; i < n1; i += 256) c2 += vf[b * n1 + i] != 0;
    s[0][t] = c0; s[1][t] = c1; s[2][t] = c2; s[3][t] = c3;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (t < k)
            for (int j = 0; j < 4; ++j) s[j][t] += s[j][t + k];
        __syncthreads();
    }
    if (t < 4) counts[b * 4 + t] = s[t][0];
}

// pseudo_huber (1326-1351) of one level, weighted and averaged over the
// batch: g = wgt * (x / r) / count / B; term = r - 1 for the loss.
__global__ void k_thuber(const float *__restrict__ pred, const float *__restrict__ tgt,
                         const uint8_t *__restrict__ valid, int B, long n,
                         const int *__restrict__ counts, int lv, float wgt, float invB,
                         float *__restrict__ g, float *__restrict__ term) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= B * n) return;
    const int b = (int)(i / n);
    const int cnt = counts[b * 4 + lv];
    if (!valid[i] || cnt == 0) {
        g[i] = 0.f;
        term[i] = 0.f;
        return;
    }
    const float x = pred[i] - tgt[i];
    const float r = sqrtf(x * x + 1.0f);
    g[i] = (x / r) * (1.0f / (float)cnt) * wgt * invB;
    term[i] = r - 1.0f;
}

// SoftArgmin.backward (887-901) plus the distribution cross-entropy
// gradient (q - p) / count, weighted: gcost[b][d][p].
__global__ void k_tsoft_bwd(const float *__restrict__ probs, const float *__restrict__ d0,
                            const float *__restrict__ gd0, const float *__restrict__ dq,
                            const uint8_t *__restrict__ vq, const int *__restrict__ counts,
                            int B, int D, long hw, float ce_w, float invB,
                            float *__restrict__ gcost, float *__restrict__ term) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= B * hw) return;
    const int b = (int)(i / hw);
    const long p = i - b * hw;
    const float *pb = probs + (long)b * D * hw + p;
    float *gb = gcost + (long)b * D * hw + p;
    const float g = gd0[i], di = d0[i];
    const int cnt = counts[b * 4 + 3];
    const bool ce = vq[i] && cnt > 0 && ce_counted(dq[i], D);
    float q[16];
    if (ce) {
        const float inv2s2 = 1.0f / (2.0f * 0.8f * 0.8f);
        const float dg = dq[i];
        float xm = -INFINITY;
        for (int d = 0; d < D; ++d) {
            const float e = (float)d - dg;
            q[d] = -e * e * inv2s2;
            xm = fmaxf(xm, q[d]);
        }
        float qs = 0.f;
        for (int d = 0; d < D; ++d) {
            q[d] = q[d] < -700.f ? 0.f : expf(q[d] - xm);
            qs += q[d];
        }
        for (int d = 0; d < D; ++d) q[d] /= qs;
    }
    const float sc = ce ? ce_w / (float)cnt * invB : 0.f;
    float ce_term = 0.f;
    for (int d = 0; d < D; ++d) {
        const float pr = pb[d * hw];
        float v = g != 0.f ? g * pr * (di - (float)d) : 0.f;
        if (ce) {
            v += (q[d] - pr) * sc;
            if (pr > 1.0e-12f) ce_term -= q[d] * logf(pr);
        }
        gb[d * hw] = v;
    }
    term[i] = ce_term;
}

// Per-sample loss: 0.5 L0 + 0.7 L1 + 1.0 L2 + 2.0 CE (train_grads 1628-1649).
__global__ void __launch_bounds__(256)
    k_tloss(const float *__restrict__ t0, const float *__restrict__ t1,
            const float *__restrict__ t2, const float *__restrict__ tce, long n4, long n2,
            long n1, const int *__restrict__ counts, double *__restrict__ loss) {
    __shared__ double s[4][256];
    const int b = blockIdx.x, t = threadIdx.x;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (long i = t; i < n4; i += 256) { a0 += t0[b * n4 + i]; a3 += tce[b * n4 + i]; }
    for (long i = t; i < n2; i += 256) a1 += t1[b * n2 + i];
    for (long i = t; i < n1; i += 256) a2 += t2[b * n1 + i];
    s[0][t] = a0; s[1][t] = a1; s[2][t] = a2; s[3][t] = a3;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (t < k)
            for (int j = 0; j < 4; ++j) s[j][t] += s[j][t + k];
        __syncthreads();
    }
    if (t == 0) {
        const int *c = counts + b * 4;
        double l = 0.0;
        if (c[0]) l += 0.5 * (s[0][0] / c[0]);
        if (c[1]) l += 0.7 * (s[1][0] / c[1]);
        if (c[2]) l += 1.0 * (s[2][0] / c[2]);
        if (c[3]) l += 2.0 * (s[3][0] / c[3]);
        loss[b] = l;
    }
}

// ------------------------------------------------------------ backward
// Refinement output ReLU (slope 0): g where the output is positive.
__global__ void k_tmask0(const float *__restrict__ g, const float *__restrict__ out, long n,
                         float *__restrict__ gs) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) gs[i] = out[i] > 0.f ? g[i] : 0.f;
}

// Conv2d input gradient (528-570) as a gather: gx[img][c][iy][ix] = sum over
// o and the taps that read (iy, ix) of w * gy; times the leaky-ReLU
// derivative of the input when MASK.  Channels c < cmax are computed and
// stored with `out_ch` channels per image.
template <int IC, int OC, int MASK>
__global__ void __launch_bounds__(256)
    k_tdgrad2d(const float *__restrict__ gy, int nimg, int H, int W, int OH, int OW, int s,
               int dil, const float *__restrict__ w, const float *__restrict__ xin, int cmax,
               int out_ch, float *__restrict__ gx) {
    __shared__ float sw[OC * IC * 9];
    for (int i = threadIdx.x; i < OC * IC * 9; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
    const long HW = (long)H * W, OHW = (long)OH * OW;
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (long)nimg * cmax * HW) return;
    const int img = (int)(i / (cmax * HW));
    const long r = i - (long)img * cmax * HW;
    const int c = (int)(r / HW);
    const long p = r - (long)c * HW;
    const int iy = (int)(p / W), ix = (int)(p - (long)iy * W);
    const float *g = gy + (long)img * OC * OHW;
    float acc = 0.f;
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
        const int ny = iy + dil - ky * dil;
        if (ny < 0 || ny % s) continue;
        const int oy = ny / s;
        if (oy >= OH) continue;
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
            const int nx = ix + dil - kx * dil;
            if (nx < 0 || nx % s) continue;
            const int ox = nx / s;
            if (ox >= OW) continue;
            const float *gp = g + (long)oy * OW + ox;
#pragma unroll
            for (int o = 0; o < OC; ++o)
                acc = fmaf(sw[(o * IC + c) * 9 + ky * 3 + kx], gp[o * OHW], acc);
        }
    }
    if (MASK) acc = xin[((long)img * IC + c) * HW + p] > 0.f ? acc : acc * 0.2f;
    gx[((long)img * out_ch + c) * HW + p] = acc;
}

// The same for stride 1, tiled: the input gradient of a stride-1 3x3
// convolution is a convolution of gy with the flipped taps, so a CTA stages
// the gy tile (kTR x kTC inputs plus a dil halo, all OC channels) in shared
// memory and each thread computes ICG input channels of one pixel.
template <int IC, int OC, int ICG, int MASK>
__global__ void __launch_bounds__(kTC *kTR)
    k_tdgrad2d_s1(const float *__restrict__ gy, int H, int W, int dil,
                  const float *__restrict__ w, const float *__restrict__ xin, int cmax,
                  int out_ch, float *__restrict__ gx) {
    extern __shared__ __align__(16) float gt[];
    __shared__ float sw[OC * IC * 9];
    const int ng = (cmax + ICG - 1) / ICG;
    const int img = blockIdx.z / ng, c0 = (blockIdx.z - img * ng) * ICG;
    const int tid = threadIdx.y * kTC + threadIdx.x;
    for (int i = tid; i < OC * IC * 9; i += kTC * kTR) sw[i] = w[i];
    const long HW = (long)H * W;
    const int x0 = blockIdx.x * kTC, y0 = blockIdx.y * kTR;
    const int th = kTR + 2 * dil, tw = kTC + 2 * dil;
    const float *g = gy + (long)img * OC * HW;
    for (int i = tid; i < OC * th * tw; i += kTC * kTR) {
        const int o = i / (th * tw), r = i - o * th * tw, ty = r / tw, tx = r - ty * tw;
        const int yy = y0 - dil + ty, xx = x0 - dil + tx;
        gt[i] = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? g[o * HW + (long)yy * W + xx] : 0.f;
    }
    __syncthreads();
    const int ix = x0 + threadIdx.x, iy = y0 + threadIdx.y;
    if (ix >= W || iy >= H) return;
    float acc[ICG];
#pragma unroll
    for (int j = 0; j < ICG; ++j) acc[j] = 0.f;
#pragma unroll
    for (int o = 0; o < OC; ++o)
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
            // output row iy + dil - ky*dil sits at tile row threadIdx.y + (2 - ky) * dil
            const float *row = gt + (o * th + threadIdx.y + (2 - ky) * dil) * tw + threadIdx.x;
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                const float gv = row[(2 - kx) * dil];
#pragma unroll
                for (int j = 0; j < ICG; ++j)
                    if (c0 + j < cmax)
                        acc[j] = fmaf(sw[(o * IC + c0 + j) * 9 + ky * 3 + kx], gv, acc[j]);
            }
        }
    const long p = (long)iy * W + ix;
#pragma unroll
    for (int j = 0; j < ICG; ++j) {
        const int c = c0 + j;
        if (c >= cmax) break;
        float v = acc[j];
        if (MASK) v = xin[((long)img * IC + c) * HW + p] > 0.f ? v : v * 0.2f;
        gx[((long)img * out_ch + c) * HW + p] = v;
    }
}

// Conv3d input gradient (643-693), same form, with the leaky-ReLU
// derivative of the input when MASK.
template <int IC, int OC, int MASK>
__global__ void __launch_bounds__(256)
    k_tdgrad3d(const float *__restrict__ gy, int B, int D, int h, int w,
               const float *__restrict__ wt, const float *__restrict__ xin,
               float *__restrict__ gx) {
    __shared__ float sw[OC * IC * 27];
    for (int i = threadIdx.x; i < OC * IC * 27; i += blockDim.x) sw[i] = wt[i];
    __syncthreads();
    const long hw = (long)h * w, total = (long)D * hw;
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (long)B * IC * total) return;
    const int b = (int)(i / (IC * total));
    const long r = i - (long)b * IC * total;
    const int c = (int)(r / total);
    const long p = r - (long)c * total;
    const int dd = (int)(p / hw), yy = (int)((p / w) % h), xx = (int)(p % w);
    const float *g = gy + (long)b * OC * total;
    float acc = 0.f;
#pragma unroll
    for (int kd = 0; kd < 3; ++kd) {
        const int od = dd + 1 - kd;
        if (od < 0 || od >= D) continue;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
            const int oy = yy + 1 - ky;
            if (oy < 0 || oy >= h) continue;
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                const int ox = xx + 1 - kx;
                if (ox < 0 || ox >= w) continue;
                const float *gp = g + (long)od * hw + (long)oy * w + ox;
#pragma unroll
                for (int o = 0; o < OC; ++o)
                    acc = fmaf(sw[(o * IC + c) * 27 + kd * 9 + ky * 3 + kx], gp[o * total], acc);
            }
        }
    }
    if (MASK) acc = xin[i] > 0.f ? acc : acc * 0.2f;
    gx[i] = acc;
}

// Weight gradients, per-CTA partial sums.  A CTA walks tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... (a fixed assignment, so the sums are
// deterministic), stages each tile's input patch and output gradients in
// shared memory and accumulates, for the KPT (out of K) weight rows
// k = tid, tid + 128, ... it owns, all OC outputs in registers; at the end it
// writes partial[cta][o][k].  Rows k < K-1 are the taps, k == K-1 the bias.
constexpr int kWgCtas = 4 * 148;

// 2-D: a tile is one image's kTR x kTC outputs; taps k = c*9 + ky*3 + kx.
template <int IC, int OC>
__global__ void __launch_bounds__(128)
    k_twgrad2d(const float *__restrict__ x, const float *__restrict__ gy, int nimg, int H, int W,
               int OH, int OW, int s, int dil, float *__restrict__ partial) {
    constexpr int K = IC * 9 + 1, P = kTR * kTC, KPT = (K + 127) / 128;
    extern __shared__ __align__(16) float sm[];
    float *gyt = sm;                      // [OC][P]
    float *xt = sm + OC * P;              // [IC][th][tw]
    const int tid = threadIdx.x;
    const long HW = (long)H * W, OHW = (long)OH * OW;
    const int tx_n = (OW + kTC - 1) / kTC, ty_n = (OH + kTR - 1) / kTR;
    const long ntiles = (long)nimg * tx_n * ty_n;
    const int th = (kTR - 1) * s + 2 * dil + 1, tw = (kTC - 1) * s + 2 * dil + 1;
    float acc[KPT][OC];
#pragma unroll
    for (int j = 0; j < KPT; ++j)
#pragma unroll
        for (int o = 0; o < OC; ++o) acc[j][o] = 0.f;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int img = (int)(tile / (tx_n * ty_n));
        const int rem = (int)(tile - (long)img * tx_n * ty_n);
        const int oy0 = (rem / tx_n) * kTR, ox0 = (rem % tx_n) * kTC;
        __syncthreads();                  // the previous tile's reads are done
        for (int i = tid; i < OC * P; i += 128) {
            const int o = i / P, q = i - o * P, oy = oy0 + q / kTC, ox = ox0 + q % kTC;
            gyt[i] = (oy < OH && ox < OW)
                         ? gy[((long)img * OC + o) * OHW + (long)oy * OW + ox]
                         : 0.f;
        }
        const int ix0 = ox0 * s - dil, iy0 = oy0 * s - dil;
        for (int i = tid; i < IC * th * tw; i += 128) {
            const int c = i / (th * tw), r2 = i - c * th * tw, ty = r2 / tw, tx = r2 - ty * tw;
            const int yy = iy0 + ty, xx = ix0 + tx;
            xt[i] = (yy >= 0 && yy < H && xx >= 0 && xx < W)
                        ? x[((long)img * IC + c) * HW + (long)yy * W + xx]
                        : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const int k = tid + 128 * j;
            if (k >= K) break;
            if (k < K - 1) {
                const int c = k / 9, ky = (k % 9) / 3, kx = k % 3;
                const float *xc = xt + c * th * tw + ky * dil * tw + kx * dil;
                for (int q = 0; q < P; ++q) {
                    const float xv = xc[(q / kTC) * s * tw + (q % kTC) * s];
#pragma unroll
                    for (int o = 0; o < OC; ++o) acc[j][o] = fmaf(xv, gyt[o * P + q], acc[j][o]);
                }
            } else {
                for (int q = 0; q < P; ++q)
#pragma unroll
                    for (int o = 0; o < OC; ++o) acc[j][o] += gyt[o * P + q];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        const int k = tid + 128 * j;
        if (k < K)
#pragma unroll
            for (int o = 0; o < OC; ++o) partial[((long)blockIdx.x * OC + o) * K + k] = acc[j][o];
    }
}

size_t twgrad2d_smem(int IC, int OC, int s, int dil) {
    return sizeof(float) * (OC * kTR * kTC +
                            IC * ((kTR - 1) * s + 2 * dil + 1) * ((kTC - 1) * s + 2 * dil + 1));
}

// 3-D: a tile is one sample's kTD disparities x 1 row x 32 columns; taps
// k = c*27 + kd*9 + ky*3 + kx.
template <int IC, int OC>
__global__ void __launch_bounds__(128)
    k_twgrad3d(const float *__restrict__ x, const float *__restrict__ gy, int B, int D, int h,
               int w, float *__restrict__ partial) {
    constexpr int K = IC * 27 + 1, P = kTD * 32, KPT = (K + 127) / 128;
    __shared__ float xt[IC][kTD + 2][3][34];
    __shared__ float gyt[OC][P];
    const int tid = threadIdx.x;
    const int nd = (D + kTD - 1) / kTD, nx = (w + 31) / 32;
    const long ntiles = (long)B * h * nd * nx;
    const long hw = (long)h * w, total = (long)D * hw;
    float acc[KPT][OC];
#pragma unroll
    for (int j = 0; j < KPT; ++j)
#pragma unroll
        for (int o = 0; o < OC; ++o) acc[j][o] = 0.f;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int b = (int)(tile / ((long)h * nd * nx));
        const int rem = (int)(tile - (long)b * h * nd * nx);
        const int oy = rem / (nd * nx), r2 = rem - oy * nd * nx;
        const int d0 = (r2 / nx) * kTD, x0 = (r2 % nx) * 32;
        __syncthreads();
        for (int i = tid; i < OC * P; i += 128) {
            const int o = i / P, q = i - o * P, od = d0 + q / 32, ox = x0 + q % 32;
            gyt[o][q] = (od < D && ox < w) ? gy[((long)b * OC + o) * total + (long)od * hw +
                                                (long)oy * w + ox]
                                          : 0.f;
        }
        constexpr int PLANE = (kTD + 2) * 3 * 34;
        for (int i = tid; i < IC * PLANE; i += 128) {
            const int c = i / PLANE, r3 = i - c * PLANE;
            const int dz = r3 / 102, r4 = r3 - dz * 102, r = r4 / 34, jx = r4 - r * 34;
            const int dd = d0 - 1 + dz, yy = oy - 1 + r, xx = x0 - 1 + jx;
            xt[c][dz][r][jx] = (dd >= 0 && dd < D && yy >= 0 && yy < h && xx >= 0 && xx < w)
                                   ? x[((long)b * IC + c) * total + dd * hw + yy * w + xx]
                                   : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const int k = tid + 128 * j;
            if (k >= K) break;
            if (k < K - 1) {
                const int c = k / 27, kd = (k % 27) / 9, ky = (k % 9) / 3, kx = k % 3;
                for (int q = 0; q < P; ++q) {
                    const float xv = xt[c][q / 32 + kd][ky][q % 32 + kx];
#pragma unroll
                    for (int o = 0; o < OC; ++o) acc[j][o] = fmaf(xv, gyt[o][q], acc[j][o]);
                }
            } else {
                for (int q = 0; q < P; ++q)
#pragma unroll
                    for (int o = 0; o < OC; ++o) acc[j][o] += gyt[o][q];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        const int k = tid + 128 * j;
        if (k < K)
#pragma unroll
            for (int o = 0; o < OC; ++o) partial[((long)blockIdx.x * OC + o) * K + k] = acc[j][o];
    }
}

// CTA partials -> one layer's weight and bias gradient in FP64.  A block
// takes 32 weights (threadIdx.x); its 32 rows (threadIdx.y) add the partials
// t = y, y + 32, ... in order, and row sums are then added in row order, so
// the result does not depend on scheduling.  Parameter layout: weights
// [o][taps], then bias [o].
__global__ void __launch_bounds__(1024)
    k_treduce(const float *__restrict__ partial, long nblk, int OC, int K,
              double *__restrict__ gw, double *__restrict__ gb) {
    __shared__ double rs[32][33];
    const int j = blockIdx.x * 32 + threadIdx.x;
    const long stride = (long)OC * K;
    double s = 0.0;
    if (j < OC * K)
        for (long t = threadIdx.y; t < nblk; t += 32) s += (double)partial[t * stride + j];
    rs[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y != 0 || j >= OC * K) return;
    double tot = 0.0;
    for (int y = 0; y < 32; ++y) tot += rs[y][threadIdx.x];
    const int o = j / K, k = j - o * K;
    if (k < K - 1) gw[o * (K - 1) + k] = tot;
    else gb[o] = tot;
}

// CostVolume.backward (801-824) as a gather: gfl[c][y][x] sums over d the
// gradient times sign(fl - fr(x - d)); gfr[c][y][x] subtracts it at x + d.
__global__ void k_tcostvol_bwd(const float *__restrict__ gvol, const float *__restrict__ f,
                               int B, int C, int D, int h, int w, float *__restrict__ gf) {
    const long hw = (long)h * w, n = (long)B * C * hw;
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = (int)(i / (C * hw));
    const long r = i - (long)b * C * hw;
    const int c = (int)(r / hw);
    const long p = r - (long)c * hw;
    const int y = (int)(p / w), x = (int)(p - (long)y * w);
    const float *fl = f + ((long)b * C + c) * hw + (long)y * w;
    const float *fr = f + ((long)(B + b) * C + c) * hw + (long)y * w;
    const float *g = gvol + ((long)b * C + c) * D * hw + (long)y * w;
    float al = 0.f, ar = 0.f;
    for (int d = 0; d < D; ++d) {
        if (x - d >= 0) {
            const float v = fl[x] - fr[x - d];
            const float gg = g[d * hw + x];
            al += v < 0.f ? -gg : gg;
        }
        if (x + d < w) {
            const float v = fl[x + d] - fr[x];
            const float gg = g[d * hw + x + d];
            ar -= v < 0.f ? -gg : gg;
        }
    }
    gf[((long)b * C + c) * hw + p] = al;
    gf[((long)(B + b) * C + c) * hw + p] = ar;
}

// BilinearUpsample.backward (958-974) of `2 * (grin0 + gs)` from the
// (H2, W2) level to the (h, w) level, as a gather over the destination
// pixels whose taps touch (ys, xs); plus `add`; times (mask > 0) when a mask
// is given (the previous level's output ReLU).
__global__ void k_tup_bwd(const float *__restrict__ grin, long grin_stride,
                          const float *__restrict__ gs, int B, int H2, int W2, int h, int w,
                          int ry, int rx, const float *__restrict__ add,
                          const float *__restrict__ mask, float *__restrict__ out) {
    const long hw = (long)h * w, n2 = (long)H2 * W2;
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= B * hw) return;
    const int b = (int)(i / hw);
    const long p = i - b * hw;
    const int ys = (int)(p / w), xs = (int)(p - (long)ys * w);
    const float *g1 = grin + b * grin_stride;
    const float *g2 = gs + (long)b * n2;
    // destination rows / columns whose source taps can reach (ys, xs)
    const int cy = (int)(((double)ys + 0.5) * H2 / h), cx = (int)(((double)xs + 0.5) * W2 / w);
    float acc = 0.f;
    for (int oy = max(0, cy - ry); oy <= min(H2 - 1, cy + ry); ++oy)
        for (int ox = max(0, cx - rx); ox <= min(W2 - 1, cx + rx); ++ox) {
            const Taps t = bilinear_taps(oy, ox, h, w, H2, W2);
            float wgt = 0.f;
            if (t.i00 == p) wgt += (float)t.w00;
            if (t.i01 == p) wgt += (float)t.w01;
            if (t.i10 == p) wgt += (float)t.w10;
            if (t.i11 == p) wgt += (float)t.w11;
            if (wgt != 0.f) {
                const long q = (long)oy * W2 + ox;
                acc = fmaf((g1[q] + g2[q]) * 2.0f, wgt, acc);
            }
        }
    float v = acc + add[i];
    if (mask) v = mask[i] > 0.f ? v : 0.f;
    out[i] = v;
}

// Adam.step (1368-1387) in FP64 on the master parameters; refreshes the
// FP32 copy the kernels read.
__global__ void k_tadam(double *__restrict__ p, const double *__restrict__ g,
                        double *__restrict__ m, double *__restrict__ v, long n, double lr,
                        double c1, double c2, double clip, float *__restrict__ p32) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double b1 = 0.9, b2 = 0.999, eps = 1.0e-8;
    double gi = g[i];
    if (gi > clip) gi = clip;
    else if (gi < -clip) gi = -clip;
    const double mi = b1 * m[i] + (1.0 - b1) * gi;
    const double vi = b2 * v[i] + (1.0 - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const double pi = p[i] - lr * (mi * c1) / (sqrt(vi * c2) + eps);
    p[i] = pi;
    p32[i] = (float)pi;
}

__global__ void k_f64_to_f32(const double *__restrict__ a, long n, float *__restrict__ b) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

unsigned nblocks(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace
}  // namespace sv

using namespace sv;

// --------------------------------------------------------------- trainer
struct sv_trainer {
    int arch[13];
    int C, Cm, D, Rc, nd, dil[8];
    long np;
    long off_fw[4], off_fb[4], off_cw[3], off_cb[3], off_rw[2][9], off_rb[2][9];
    double *p64 = nullptr, *g64 = nullptr, *m = nullptr, *v = nullptr;
    float *p32 = nullptr;
    double b1t = 1.0, b2t = 1.0;
};

namespace {

long layout(sv_trainer *t) {
    long p = 0;
    const int fic[4] = {1, t->C, t->C, t->C};
    for (int i = 0; i < 4; ++i) {
        t->off_fw[i] = p; p += (long)t->C * fic[i] * 9;
        t->off_fb[i] = p; p += t->C;
    }
    const int cic[3] = {t->C, t->Cm, t->Cm}, coc[3] = {t->Cm, t->Cm, 1};
    for (int i = 0; i < 3; ++i) {
        t->off_cw[i] = p; p += (long)coc[i] * cic[i] * 27;
        t->off_cb[i] = p; p += coc[i];
    }
    for (int lv = 0; lv < 2; ++lv) {
        int prev = 2;
        for (int i = 0; i < t->nd; ++i) {
            t->off_rw[lv][i] = p; p += (long)t->Rc * prev * 9;
            t->off_rb[lv][i] = p; p += t->Rc;
            prev = t->Rc;
        }
        t->off_rw[lv][t->nd] = p; p += (long)prev * 9;
        t->off_rb[lv][t->nd] = p; p += 1;
    }
    return p;
}

struct TrainBufs {
    float *img, *a1, *a2, *a3, *f4, *vol, *b1, *b2, *cost, *probs, *d0;
    float *rin[2], *r[2][8], *out[2];
    float *dh, *gh, *dq;
    uint8_t *vh, *vq;
    int *counts;
    float *t0, *t1, *t2, *tce, *gl0, *gl1, *gl2;
    float *gs, *gs0, *gA, *gB, *grin, *gd0, *gcost, *gq2, *gq1, *gvol, *gf, *gF3, *gF4;
    float *partial;
    double *loss;
    long partial_n;
};

struct Dims {
    int B, H, W, h1, w1, h, w, H2, W2;
    long HW, HW2, hw, h1w1;
};

Dims dims(int B, int W, int H) {
    Dims d;
    d.B = B; d.H = H; d.W = W;
    d.h1 = (H - 1) / 2 + 1; d.w1 = (W - 1) / 2 + 1;
    d.h = (d.h1 - 1) / 2 + 1; d.w = (d.w1 - 1) / 2 + 1;
    d.H2 = H / 2; d.W2 = W / 2;
    d.HW = (long)H * W; d.HW2 = (long)d.H2 * d.W2; d.hw = (long)d.h * d.w;
    d.h1w1 = (long)d.h1 * d.w1;
    return d;
}

long tiles2d(int nimg, int OH, int OW) {
    return (long)nimg * ((OH + kTR - 1) / kTR) * ((OW + kTC - 1) / kTC);
}

long partial_floats(const sv_trainer *t, const Dims &d) {
    (void)d;
    // at most kWgCtas CTAs per weight-gradient launch; the widest layer
    // (OC x K) bounds the rest
    const int C = t->C, Cm = t->Cm, Rc = t->Rc;
    long m = 0;
    auto upd = [&](long v) { m = v > m ? v : m; };
    upd((long)C * (C * 9 + 1));
    upd((long)Cm * (C * 27 + 1));
    upd((long)Cm * (Cm * 27 + 1));
    upd((long)Rc * (Rc * 9 + 1));
    upd((long)Rc * (2 * 9 + 1));
    return m * kWgCtas;
}

void carve(const sv_trainer *t, const Dims &d, Carver &cv, TrainBufs &b) {
    const int B = d.B, C = t->C, Cm = t->Cm, D = t->D, Rc = t->Rc;
    const long DHW = (long)D * d.hw;
    b.img = cv.take<float>(2 * B * d.HW);
    b.a1 = cv.take<float>(2L * B * C * d.h1w1);
    b.a2 = cv.take<float>(2L * B * C * d.hw);
    b.a3 = cv.take<float>(2L * B * C * d.hw);
    b.f4 = cv.take<float>(2L * B * C * d.hw);
    b.vol = cv.take<float>((long)B * C * DHW);
    b.b1 = cv.take<float>((long)B * Cm * DHW);
    b.b2 = cv.take<float>((long)B * Cm * DHW);
    b.cost = cv.take<float>((long)B * DHW);
    b.probs = cv.take<float>((long)B * DHW);
    b.d0 = cv.take<float>((long)B * d.hw);
    const long HWl[2] = {d.HW2, d.HW};
    for (int lv = 0; lv < 2; ++lv) {
        b.rin[lv] = cv.take<float>(2L * B * HWl[lv]);
        for (int i = 0; i < t->nd; ++i) b.r[lv][i] = cv.take<float>((long)B * Rc * HWl[lv]);
        b.out[lv] = cv.take<float>((long)B * HWl[lv]);
    }
    b.dh = cv.take<float>((long)B * d.HW2);
    b.gh = cv.take<float>((long)B * d.HW2);
    b.dq = cv.take<float>((long)B * d.hw);
    b.vh = cv.take<uint8_t>((long)B * d.HW2);
    b.vq = cv.take<uint8_t>((long)B * d.hw);
    b.counts = cv.take<int>(4L * B);
    b.t0 = cv.take<float>((long)B * d.hw);
    b.t1 = cv.take<float>((long)B * d.HW2);
    b.t2 = cv.take<float>((long)B * d.HW);
    b.tce = cv.take<float>((long)B * d.hw);
    b.gl0 = cv.take<float>((long)B * d.hw);
    b.gl1 = cv.take<float>((long)B * d.HW2);
    b.gl2 = cv.take<float>((long)B * d.HW);
    b.gs = cv.take<float>((long)B * d.HW);
    b.gs0 = cv.take<float>((long)B * d.HW2);
    b.gA = cv.take<float>((long)B * Rc * d.HW);
    b.gB = cv.take<float>((long)B * Rc * d.HW);
    b.grin = cv.take<float>((long)B * d.HW);
    b.gd0 = cv.take<float>((long)B * d.hw);
    b.gcost = cv.take<float>((long)B * DHW);
    b.gq2 = cv.take<float>((long)B * Cm * DHW);
    b.gq1 = cv.take<float>((long)B * Cm * DHW);
    b.gvol = cv.take<float>((long)B * C * DHW);
    b.gf = cv.take<float>(2L * B * C * d.hw);
    b.gF3 = cv.take<float>(2L * B * C * d.h1w1);
    b.gF4 = cv.take<float>(2L * B * C * d.hw);
    b.partial_n = partial_floats(t, d);
    b.partial = cv.take<float>(b.partial_n);
    b.loss = cv.take<double>(B);
}

// 2-D conv forward launcher (the template is picked by the caller)
template <int IC, int OC, int OCG, int ACT>
int fconv2d(const float *x, int nimg, int H, int W, int OH, int OW, int s, int dil,
            const float *w, const float *b, float *y, const float *resid, long rstride,
            cudaStream_t st) {
    const size_t sm = tconv2d_smem(IC, s, dil);
    if (sm > 48 * 1024) {
        set_error("conv tile needs %zu bytes of shared memory (dilation %d too large)", sm, dil);
        return SV_ERR_SHAPE;
    }
    const dim3 g((OW + kTC - 1) / kTC, (OH + kTR - 1) / kTR, nimg * (OC / OCG));
    count_launch();
    k_tconv2d<IC, OC, OCG, ACT><<<g, dim3(kTC, kTR), sm, st>>>(x, H, W, OH, OW, s, dil, w, b, y,
                                                               resid, rstride);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <int IC, int OC, int ICG, int MASK>
int dgrad2d_s1(const float *gy, int nimg, int H, int W, int dil, const float *w,
               const float *xin, int cmax, int out_ch, float *gx, cudaStream_t st) {
    const size_t sm = sizeof(float) * OC * (kTR + 2 * dil) * (kTC + 2 * dil);
    if (sm > 48 * 1024) {
        set_error("input-gradient tile needs %zu bytes of shared memory", sm);
        return SV_ERR_SHAPE;
    }
    const dim3 g((W + kTC - 1) / kTC, (H + kTR - 1) / kTR, nimg * ((cmax + ICG - 1) / ICG));
    count_launch();
    k_tdgrad2d_s1<IC, OC, ICG, MASK><<<g, dim3(kTC, kTR), sm, st>>>(gy, H, W, dil, w, xin, cmax,
                                                                   out_ch, gx);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <int IC, int OC>
int wgrad2d(const float *x, const float *gy, int nimg, int H, int W, int OH, int OW, int s,
            int dil, float *partial, double *gw, double *gb, cudaStream_t st) {
    const size_t sm = twgrad2d_smem(IC, OC, s, dil);
    if (sm > 48 * 1024) {
        set_error("weight-gradient tile needs %zu bytes of shared memory", sm);
        return SV_ERR_SHAPE;
    }
    const long ntiles = tiles2d(nimg, OH, OW);
    const int nblk = (int)(ntiles < kWgCtas ? ntiles : kWgCtas);
    constexpr int K = IC * 9 + 1;
    count_launch();
    k_twgrad2d<IC, OC><<<nblk, 128, sm, st>>>(x, gy, nimg, H, W, OH, OW, s, dil, partial);
    count_launch();
    k_treduce<<<(OC * K + 31) / 32, dim3(32, 32), 0, st>>>(partial, nblk, OC, K, gw, gb);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <int IC, int OC>
int wgrad3d(const float *x, const float *gy, int B, int D, int h, int w, float *partial,
            double *gw, double *gb, cudaStream_t st) {
    const long ntiles = (long)B * h * ((D + kTD - 1) / kTD) * ((w + 31) / 32);
    const int nblk = (int)(ntiles < kWgCtas ? ntiles : kWgCtas);
    constexpr int K = IC * 27 + 1;
    count_launch();
    k_twgrad3d<IC, OC><<<nblk, 128, 0, st>>>(x, gy, B, D, h, w, partial);
    count_launch();
    k_treduce<<<(OC * K + 31) / 32, dim3(32, 32), 0, st>>>(partial, nblk, OC, K, gw, gb);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <int C, int CM, int RC>
int train_impl(sv_trainer *t, const float *left, const float *right, const float *disp,
               const uint8_t *valid, const Dims &d, const TrainBufs &b, float *pred,
               double *loss, cudaStream_t st) {
    const int B = d.B, D = t->D, nd = t->nd;
    const float *P = t->p32;
    double *G = t->g64;
    const long DHW = (long)D * d.hw;
    const float invB = 1.0f / (float)B;
    constexpr int FG = C % 4 == 0 ? 4 : C, CG = CM % 2 == 0 ? 2 : CM, RG = RC % 4 == 0 ? 4 : RC;
    int rc;
    // inputs: the B left views, then the B right views
    if (cudaMemcpyAsync(b.img, left, sizeof(float) * B * d.HW, cudaMemcpyDeviceToDevice, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(b.img + (long)B * d.HW, right, sizeof(float) * B * d.HW,
                        cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        set_error("input copy failed");
        return SV_ERR_CUDA;
    }
    // ---- targets (build_targets) and counts
    count_launch();
    k_tpool<<<nblocks(B * d.HW2), 256, 0, st>>>(disp, valid, left, B, d.H, d.W, b.dh, b.vh, b.gh);
    count_launch();
    k_tpool<<<nblocks(B * d.hw), 256, 0, st>>>(b.dh, b.vh, nullptr, B, d.H2, d.W2, b.dq, b.vq,
                                               nullptr);
    count_launch();
    k_tcounts<<<B, 256, 0, st>>>(b.vq, b.vh, valid, b.dq, d.hw, d.HW2, d.HW, D, b.counts);
    SV_LAUNCH_CHECK();
    // ---- forward: FeatureNet on 2B images
    if ((rc = fconv2d<1, C, FG, 1>(b.img, 2 * B, d.H, d.W, d.h1, d.w1, 2, 1, P + t->off_fw[0],
                                   P + t->off_fb[0], b.a1, nullptr, 0, st)))
        return rc;
    if ((rc = fconv2d<C, C, FG, 1>(b.a1, 2 * B, d.h1, d.w1, d.h, d.w, 2, 1, P + t->off_fw[1],
                                   P + t->off_fb[1], b.a2, nullptr, 0, st)))
        return rc;
    if ((rc = fconv2d<C, C, FG, 1>(b.a2, 2 * B, d.h, d.w, d.h, d.w, 1, 1, P + t->off_fw[2],
                                   P + t->off_fb[2], b.a3, nullptr, 0, st)))
        return rc;
    if ((rc = fconv2d<C, C, FG, 0>(b.a3, 2 * B, d.h, d.w, d.h, d.w, 1, 1, P + t->off_fw[3],
                                   P + t->off_fb[3], b.f4, nullptr, 0, st)))
        return rc;
    count_launch();
    k_tcostvol<<<nblocks((long)B * C * DHW), 256, 0, st>>>(b.f4, B, C, D, d.h, d.w, b.vol);
    const dim3 v3((d.w + 31) / 32, d.h * ((D + kTD - 1) / kTD), B * (CM / CG));
    count_launch();
    k_tconv3d<C, CM, CG, 1><<<v3, dim3(32, kTD), 0, st>>>(b.vol, D, d.h, d.w, P + t->off_cw[0],
                                                          P + t->off_cb[0], b.b1);
    count_launch();
    k_tconv3d<CM, CM, CG, 1><<<v3, dim3(32, kTD), 0, st>>>(b.b1, D, d.h, d.w, P + t->off_cw[1],
                                                           P + t->off_cb[1], b.b2);
    const dim3 v1((d.w + 31) / 32, d.h * ((D + kTD - 1) / kTD), B);
    count_launch();
    k_tconv3d<CM, 1, 1, 0><<<v1, dim3(32, kTD), 0, st>>>(b.b2, D, d.h, d.w, P + t->off_cw[2],
                                                         P + t->off_cb[2], b.cost);
    count_launch();
    k_tsoftargmin<<<nblocks(B * d.hw), 256, 0, st>>>(b.cost, B, D, d.h, d.w, b.probs, b.d0);
    SV_LAUNCH_CHECK();
    // ---- refinement levels
    const int Hs[2] = {d.H2, d.H}, Ws[2] = {d.W2, d.W};
    const long HWl[2] = {d.HW2, d.HW};
    const float *guides[2] = {b.gh, b.img};
    const float *prev = b.d0;
    int ph = d.h, pw = d.w;
    for (int lv = 0; lv < 2; ++lv) {
        const int Hl = Hs[lv], Wl = Ws[lv];
        count_launch();
        k_tupcat<<<nblocks(B * HWl[lv]), 256, 0, st>>>(prev, B, ph, pw, Hl, Wl, guides[lv],
                                                       b.rin[lv]);
        const float *cur = b.rin[lv];
        for (int i = 0; i < nd; ++i) {
            const int dl = t->dil[i];
            rc = i == 0 ? fconv2d<2, RC, RG, 1>(cur, B, Hl, Wl, Hl, Wl, 1, dl, P + t->off_rw[lv][i],
                                                P + t->off_rb[lv][i], b.r[lv][i], nullptr, 0, st)
                        : fconv2d<RC, RC, RG, 1>(cur, B, Hl, Wl, Hl, Wl, 1, dl,
                                                 P + t->off_rw[lv][i], P + t->off_rb[lv][i],
                                                 b.r[lv][i], nullptr, 0, st);
            if (rc) return rc;
            cur = b.r[lv][i];
        }
        if ((rc = fconv2d<RC, 1, 1, 2>(cur, B, Hl, Wl, Hl, Wl, 1, 1, P + t->off_rw[lv][nd],
                                       P + t->off_rb[lv][nd], b.out[lv], b.rin[lv],
                                       2 * HWl[lv], st)))
            return rc;
        prev = b.out[lv];
        ph = Hl;
        pw = Wl;
    }
    // ---- losses
    count_launch();
    k_thuber<<<nblocks(B * d.hw), 256, 0, st>>>(b.d0, b.dq, b.vq, B, d.hw, b.counts, 0, 0.5f,
                                                invB, b.gl0, b.t0);
    count_launch();
    k_thuber<<<nblocks(B * d.HW2), 256, 0, st>>>(b.out[0], b.dh, b.vh, B, d.HW2, b.counts, 1,
                                                 0.7f, invB, b.gl1, b.t1);
    count_launch();
    k_thuber<<<nblocks(B * d.HW), 256, 0, st>>>(b.out[1], disp, valid, B, d.HW, b.counts, 2,
                                                1.0f, invB, b.gl2, b.t2);
    SV_LAUNCH_CHECK();
    // ---- backward: refinement levels, fine to coarse.  gsl[lv] is the
    // gradient on level lv's output after its ReLU (Refinement.backward's g).
    float *gsl[2] = {b.gs0, b.gs};
    count_launch();
    k_tmask0<<<nblocks(B * d.HW), 256, 0, st>>>(b.gl2, b.out[1], B * d.HW, gsl[1]);
    for (int lv = 1; lv >= 0; --lv) {
        const int Hl = Hs[lv], Wl = Ws[lv];
        const float *gs = gsl[lv];
        // final conv (x = r[nd-1], gy = gs)
        if ((rc = wgrad2d<RC, 1>(b.r[lv][nd - 1], gs, B, Hl, Wl, Hl, Wl, 1, 1, b.partial,
                                 G + t->off_rw[lv][nd], G + t->off_rb[lv][nd], st)))
            return rc;
        if ((rc = dgrad2d_s1<RC, 1, RG, 1>(gs, B, Hl, Wl, 1, P + t->off_rw[lv][nd],
                                           b.r[lv][nd - 1], RC, RC, b.gA, st)))
            return rc;
        float *gcur = b.gA, *gnext = b.gB;
        for (int i = nd - 1; i >= 1; --i) {
            const int dl = t->dil[i];
            if ((rc = wgrad2d<RC, RC>(b.r[lv][i - 1], gcur, B, Hl, Wl, Hl, Wl, 1, dl, b.partial,
                                      G + t->off_rw[lv][i], G + t->off_rb[lv][i], st)))
                return rc;
            if ((rc = dgrad2d_s1<RC, RC, RG, 1>(gcur, B, Hl, Wl, dl, P + t->off_rw[lv][i],
                                                b.r[lv][i - 1], RC, RC, gnext, st)))
                return rc;
            float *tmp = gcur;
            gcur = gnext;
            gnext = tmp;
        }
        if ((rc = wgrad2d<2, RC>(b.rin[lv], gcur, B, Hl, Wl, Hl, Wl, 1, t->dil[0], b.partial,
                                 G + t->off_rw[lv][0], G + t->off_rb[lv][0], st)))
            return rc;
        // only the disparity channel of the input gradient is needed
        if ((rc = dgrad2d_s1<2, RC, 1, 0>(gcur, B, Hl, Wl, t->dil[0], P + t->off_rw[lv][0],
                                          nullptr, 1, 1, b.grin, st)))
            return rc;
        // up-sample backward of 2 * (input gradient + skip) to the previous
        // level, plus that level's loss gradient, through its output ReLU
        const int sh = lv ? d.H2 : d.h, sw = lv ? d.W2 : d.w;
        const int ry = (int)ceil(2.0 * Hl / sh) + 2, rx = (int)ceil(2.0 * Wl / sw) + 2;
        count_launch();
        k_tup_bwd<<<nblocks((long)B * sh * sw), 256, 0, st>>>(
            b.grin, HWl[lv], gs, B, Hl, Wl, sh, sw, ry, rx, lv ? b.gl1 : b.gl0,
            lv ? b.out[0] : nullptr, lv ? gsl[0] : b.gd0);
        SV_LAUNCH_CHECK();
    }
    // ---- soft-argmin + cross-entropy, cost filter, cost volume
    count_launch();
    k_tsoft_bwd<<<nblocks(B * d.hw), 256, 0, st>>>(b.probs, b.d0, b.gd0, b.dq, b.vq, b.counts, B,
                                                   D, d.hw, 2.0f, invB, b.gcost, b.tce);
    if ((rc = wgrad3d<CM, 1>(b.b2, b.gcost, B, D, d.h, d.w, b.partial, G + t->off_cw[2],
                             G + t->off_cb[2], st)))
        return rc;
    count_launch();
    k_tdgrad3d<CM, 1, 1><<<nblocks((long)B * CM * DHW), 256, 0, st>>>(
        b.gcost, B, D, d.h, d.w, P + t->off_cw[2], b.b2, b.gq2);
    if ((rc = wgrad3d<CM, CM>(b.b1, b.gq2, B, D, d.h, d.w, b.partial, G + t->off_cw[1],
                              G + t->off_cb[1], st)))
        return rc;
    count_launch();
    k_tdgrad3d<CM, CM, 1><<<nblocks((long)B * CM * DHW), 256, 0, st>>>(
        b.gq2, B, D, d.h, d.w, P + t->off_cw[1], b.b1, b.gq1);
    if ((rc = wgrad3d<C, CM>(b.vol, b.gq1, B, D, d.h, d.w, b.partial, G + t->off_cw[0],
                             G + t->off_cb[0], st)))
        return rc;
    count_launch();
    k_tdgrad3d<C, CM, 0><<<nblocks((long)B * C * DHW), 256, 0, st>>>(
        b.gq1, B, D, d.h, d.w, P + t->off_cw[0], nullptr, b.gvol);
    count_launch();
    k_tcostvol_bwd<<<nblocks((long)B * C * d.hw), 256, 0, st>>>(b.gvol, b.f4, B, C, D, d.h, d.w,
                                                                b.gf);
    SV_LAUNCH_CHECK();
    // ---- FeatureNet, both towers as one batch of 2B images
    if ((rc = wgrad2d<C, C>(b.a3, b.gf, 2 * B, d.h, d.w, d.h, d.w, 1, 1, b.partial,
                            G + t->off_fw[3], G + t->off_fb[3], st)))
        return rc;
    if ((rc = dgrad2d_s1<C, C, FG, 1>(b.gf, 2 * B, d.h, d.w, 1, P + t->off_fw[3], b.a3, C, C,
                                      b.gF4, st)))
        return rc;
    if ((rc = wgrad2d<C, C>(b.a2, b.gF4, 2 * B, d.h, d.w, d.h, d.w, 1, 1, b.partial,
                            G + t->off_fw[2], G + t->off_fb[2], st)))
        return rc;
    if ((rc = dgrad2d_s1<C, C, FG, 1>(b.gF4, 2 * B, d.h, d.w, 1, P + t->off_fw[2], b.a2, C, C,
                                      b.gf, st)))
        return rc;
    if ((rc = wgrad2d<C, C>(b.a1, b.gf, 2 * B, d.h1, d.w1, d.h, d.w, 2, 1, b.partial,
                            G + t->off_fw[1], G + t->off_fb[1], st)))
        return rc;
    count_launch();
    k_tdgrad2d<C, C, 1><<<nblocks(2L * B * C * d.h1w1), 256, 0, st>>>(
        b.gf, 2 * B, d.h1, d.w1, d.h, d.w, 2, 1, P + t->off_fw[1], b.a1, C, C, b.gF3);
    if ((rc = wgrad2d<1, C>(b.img, b.gF3, 2 * B, d.H, d.W, d.h1, d.w1, 2, 1, b.partial,
                            G + t->off_fw[0], G + t->off_fb[0], st)))
        return rc;
    // ---- per-sample loss and the prediction
    count_launch();
    k_tloss<<<B, 256, 0, st>>>(b.t0, b.t1, b.t2, b.tce, d.hw, d.HW2, d.HW, b.counts,
                               loss ? loss : b.loss);
    SV_LAUNCH_CHECK();
    if (pred && cudaMemcpyAsync(pred, b.out[1], sizeof(float) * B * d.HW,
                                cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        set_error("prediction copy failed");
        return SV_ERR_CUDA;
    }
    return SV_OK;
}

int check_dims(const sv_trainer *t, int B, int W, int H) {
    if (B < 1 || B > kMaxB) {
        set_error("batch %d outside 1..%d", B, kMaxB);
        return SV_ERR_SHAPE;
    }
    if (W % 4 || H % 4 || W < 8 || H < 8 || (long)W * H > (1l << 24)) {
        set_error("crop %dx%d: W and H must be multiples of 4 (the pyramid targets of "
                  "build_targets line up with the network's outputs only then), 8..", W, H);
        return SV_ERR_SHAPE;
    }
    if (W / 4 <= t->D - 2) {
        set_error("quarter width %d <= D-2 (the reference's invalid_mask raises there)", W / 4);
        return SV_ERR_SHAPE;
    }
    for (int i = 0; i < t->nd; ++i)
        if (t->dil[i] < 1 || t->dil[i] > 8) {
            set_error("dilation %d outside 1..8", t->dil[i]);
            return SV_ERR_NET;
        }
    return SV_OK;
}

}  // namespace

extern "C" {

int sv_trainer_create(const int *arch, int n_arch, const double *params, long n_params,
                      sv_trainer **out) {
    if (!arch || !params || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (n_arch < 6 || n_arch > 13 || arch[4] < 1 || arch[4] > 8 || n_arch != 5 + arch[4]) {
        set_error("arch vector must be {feat_C, cost_C, D, refine_C, ndil, dil...}");
        return SV_ERR_NET;
    }
    const bool ok_arch = (arch[0] == 12 && arch[1] == 6 && arch[3] == 8) ||
                         (arch[0] == 8 && arch[1] == 4 && arch[3] == 8);
    if (!ok_arch || arch[2] < 2 || arch[2] > 16) {
        set_error("trainable architectures: feat_C/cost_C/refine_C 12/6/8 or 8/4/8, D 2..16");
        return SV_ERR_NET;
    }
    sv_trainer *t = new sv_trainer();
    memcpy(t->arch, arch, sizeof(int) * n_arch);
    t->C = arch[0]; t->Cm = arch[1]; t->D = arch[2]; t->Rc = arch[3]; t->nd = arch[4];
    for (int i = 0; i < t->nd; ++i) t->dil[i] = arch[5 + i];
    t->np = layout(t);
    if (t->np != n_params) {
        set_error("checkpoint has %ld parameters, the architecture needs %ld", n_params, t->np);
        delete t;
        return SV_ERR_NET;
    }
    const size_t nb = sizeof(double) * t->np;
    cudaError_t e = cudaMalloc(&t->p64, nb);
    if (e == cudaSuccess) e = cudaMalloc(&t->g64, nb);
    if (e == cudaSuccess) e = cudaMalloc(&t->m, nb);
    if (e == cudaSuccess) e = cudaMalloc(&t->v, nb);
    if (e == cudaSuccess) e = cudaMalloc(&t->p32, sizeof(float) * t->np);
    if (e == cudaSuccess) e = cudaMemcpy(t->p64, params, nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(t->g64, 0, nb);
    if (e == cudaSuccess) e = cudaMemset(t->m, 0, nb);
    if (e == cudaSuccess) e = cudaMemset(t->v, 0, nb);
    if (e == cudaSuccess) {
        k_f64_to_f32<<<nblocks(t->np), 256>>>(t->p64, t->np, t->p32);
        e = cudaDeviceSynchronize();
    }
    if (e != cudaSuccess) {
        set_error("trainer allocation failed: %s", cudaGetErrorString(e));
        sv_trainer_destroy(t);
        return SV_ERR_CUDA;
    }
    *out = t;
    return SV_OK;
}

void sv_trainer_destroy(sv_trainer *t) {
    if (!t) return;
    cudaFree(t->p64);
    cudaFree(t->g64);
    cudaFree(t->m);
    cudaFree(t->v);
    cudaFree(t->p32);
    delete t;
}

long sv_trainer_param_count(const sv_trainer *t) { return t ? t->np : 0; }

static int copy_out(const double *src, double *dst, long n, long np) {
    if (!dst) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (n != np) { set_error("expected %ld values, got %ld", np, n); return SV_ERR_PARAM; }
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("device copy failed");
        return SV_ERR_CUDA;
    }
    return SV_OK;
}

int sv_trainer_get_params(const sv_trainer *t, double *out, long n) {
    if (!t) { set_error("NULL trainer"); return SV_ERR_NULL; }
    return copy_out(t->p64, out, n, t->np);
}

int sv_trainer_get_grads(const sv_trainer *t, double *out, long n) {
    if (!t) { set_error("NULL trainer"); return SV_ERR_NULL; }
    return copy_out(t->g64, out, n, t->np);
}

int sv_trainer_set_params(sv_trainer *t, const double *p, long n) {
    if (!t || !p) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (n != t->np) { set_error("expected %ld values, got %ld", t->np, n); return SV_ERR_PARAM; }
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(t->p64, p, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error("device copy failed");
        return SV_ERR_CUDA;
    }
    k_f64_to_f32<<<nblocks(t->np), 256>>>(t->p64, t->np, t->p32);
    if (cudaDeviceSynchronize() != cudaSuccess) { set_error("conversion failed"); return SV_ERR_CUDA; }
    return SV_OK;
}

int sv_trainer_set_grads(sv_trainer *t, const double *g, long n) {
    if (!t || !g) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (n != t->np) { set_error("expected %ld values, got %ld", t->np, n); return SV_ERR_PARAM; }
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(t->g64, g, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error("device copy failed");
        return SV_ERR_CUDA;
    }
    return SV_OK;
}

size_t sv_train_workspace_size(const sv_trainer *t, int B, int W, int H) {
    if (!t) { set_error("NULL trainer"); return 0; }
    if (check_dims(t, B, W, H) != SV_OK) return 0;
    Carver cv(nullptr);
    TrainBufs b;
    carve(t, dims(B, W, H), cv, b);
    return cv.off + 256;
}

int sv_train_grads(sv_trainer *t, const float *left, const float *right, const float *disp,
                   const uint8_t *valid, int B, int W, int H, double *loss, float *pred,
                   void *workspace, size_t workspace_bytes, void *stream) {
    if (!t || !left || !right || !disp || !valid) { set_error("NULL argument"); return SV_ERR_NULL; }
    int rc = check_dims(t, B, W, H);
    if (rc) return rc;
    const size_t need = sv_train_workspace_size(t, B, W, H);
    if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255)) {
        set_error("workspace must be 256-byte aligned and hold %zu bytes", need);
        return SV_ERR_WORKSPACE;
    }
    Carver cv(workspace);
    TrainBufs b;
    const Dims d = dims(B, W, H);
    carve(t, d, cv, b);
    cudaStream_t st = (cudaStream_t)stream;
    if (t->C == 12)
        return train_impl<12, 6, 8>(t, left, right, disp, valid, d, b, pred, loss, st);
    return train_impl<8, 4, 8>(t, left, right, disp, valid, d, b, pred, loss, st);
}

int sv_train_adam(sv_trainer *t, double lr, double clip, void *stream) {
    if (!t) { set_error("NULL trainer"); return SV_ERR_NULL; }
    if (!(lr >= 0.0) || !(clip > 0.0)) { set_error("lr must be >= 0 and clip > 0"); return SV_ERR_PARAM; }
    t->b1t *= 0.9;
    t->b2t *= 0.999;
    const double c1 = 1.0 / (1.0 - t->b1t), c2 = 1.0 / (1.0 - t->b2t);
    count_launch();
    k_tadam<<<nblocks(t->np), 256, 0, (cudaStream_t)stream>>>(t->p64, t->g64, t->m, t->v, t->np,
                                                                lr, c1, c2, clip, t->p32);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int sv_trainer_reset_adam(sv_trainer *t) {
    if (!t) { set_error("NULL trainer"); return SV_ERR_NULL; }
    t->b1t = 1.0;
    t->b2t = 1.0;
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemset(t->m, 0, sizeof(double) * t->np) != cudaSuccess ||
        cudaMemset(t->v, 0, sizeof(double) * t->np) != cudaSuccess) {
        set_error("reset failed");
        return SV_ERR_CUDA;
    }
    return SV_OK;
}

}  // extern "C"
