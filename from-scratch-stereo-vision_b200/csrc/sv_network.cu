// sv_network.cu -- StereoNet forward (stereonet.py:998-1233) and the
// resolution-selection helpers of predict_auto (3832-3961), FP32 path.
//
// Layouts are the reference's planar ones: feature maps [C][h][w], the cost
// volume and its filtered versions [C][D][h][w].  Convolutions are direct
// (one thread per output pixel computing every output channel, weights in
// shared memory, read by broadcast) with bias and activation fused:
//   * both siamese towers run in one launch (blockIdx.z picks the image);
//   * the cost volume is never stored: the first 3-D convolution computes
//     |fl - fr(x-d)| (or INVALID_COST 2.0) for each tap it reads;
//   * the last 3-D convolution, the invalid-disparity penalty and the
//     soft-argmin are one kernel, one thread per (y, x) over all D;
//   * each refinement level's bilinear x2 upsample writes the 2-channel
//     [disp*2, guide] input of its first convolution; the last convolution
//     adds the residual and applies relu (v > 0 ? v : v*0).
// Resampling positions follow BilinearUpsample (half-pixel centres, int()
// truncation) computed in FP64; image and disparity resizes blend in FP64.

#include <cmath>

#include "sv_common.cuh"
#include "sv_network.cuh"
#include "sv_netbatch.cuh"
#include "sv_select.cuh"
#include "sv_tc.cuh"

namespace sv {

// ---------------------------------------------------------------- resample

template <typename T>
__device__ __forceinline__ double gray_at(const T *img, int i);
template <>
__device__ __forceinline__ double gray_at<uint8_t>(const uint8_t *img, int i) {
    return __ddiv_rn((double)img[i], 255.0);
}
template <>
__device__ __forceinline__ double gray_at<float>(const float *img, int i) {
    return (double)img[i];
}
template <>
__device__ __forceinline__ double gray_at<double>(const double *img, int i) {
    return img[i];
}

// FP64 blend in the reference's order: ((a*w00 + b*w01) + c*w10) + d*w11.
template <typename T>
__device__ __forceinline__ double blend64(const T *x, const Taps &t) {
    double a = __dmul_rn(gray_at<T>(x, t.i00), t.w00);
    a = __dadd_rn(a, __dmul_rn(gray_at<T>(x, t.i01), t.w01));
    a = __dadd_rn(a, __dmul_rn(gray_at<T>(x, t.i10), t.w10));
    return __dadd_rn(a, __dmul_rn(gray_at<T>(x, t.i11), t.w11));
}

// resize_gray of a left/right pair (blockIdx.z) from full resolution to the
// work resolution, FP64 blend, FP32 output for the network; with gh, also
// the guide at half resolution, avgpool2 of the resized left view
// (stereonet.py:979-995), from the 2x2 blocks a 32 x 8 CTA holds in shared
// memory.
template <typename T>
__device__ __forceinline__ void resize_pair_body(int bx, int by, int bz, bool first, bool copy,
                                                 const T *__restrict__ l, const T *__restrict__ r, int W, int H, int W2, int H2,
                  float *__restrict__ lo, float *__restrict__ ro, float *__restrict__ gh,
                  SelState *sel, unsigned *sel_hist, long long sel_rank) {
    __shared__ float sv[8][33];
    if (sel && first)
        sel_init_block(sel, sel_rank, sel_hist);      // the stage's select starts here
    const T *src = bz ? r : l;
    float *dst = bz ? ro : lo;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int ox = bx * 32 + tx, oy = by * 8 + ty;
    const bool in = ox < W2 && oy < H2;
    float v = 0.f;
    if (in) {
        // copy: a native-resolution pass, which the reference runs on the
        // images themselves (predict_at_scale, stereonet.py:3941-3943)
        v = copy ? (float)gray_at<T>(src, oy * W + ox)
                 : (float)blend64<T>(src, bilinear_taps(oy, ox, H, W, H2, W2));
        dst[oy * W2 + ox] = v;
    }
    if (!gh || bz != 0) return;            // the same for the whole CTA
    sv[ty][tx] = v;
    __syncthreads();
    // a 2x2 block inside the half-resolution image lies inside the image
    // and inside this CTA (its origin is even, the CTA 32 x 8)
    if (in && !(tx & 1) && !(ty & 1) && ox / 2 < W2 / 2 && oy / 2 < H2 / 2)
        gh[(oy / 2) * (W2 / 2) + ox / 2] =
            0.25f * (((v + sv[ty][tx + 1]) + sv[ty + 1][tx]) + sv[ty + 1][tx + 1]);
}


template <typename T>
__global__ void __launch_bounds__(256)
    k_resize_pair(const T *__restrict__ l, const T *__restrict__ r, int W, int H, int W2, int H2,
                  float *__restrict__ lo, float *__restrict__ ro, float *__restrict__ gh,
                  SelState *sel, unsigned *sel_hist, long long sel_rank) {
    resize_pair_body<T>(blockIdx.x, blockIdx.y, blockIdx.z,
                        blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0, false, l, r, W,
                        H, W2, H2,
                        lo, ro, gh, sel, sel_hist, sel_rank);
}

// Batched: the pass's resample of every active pair (a 1-D grid over the
// pairs' largest tile grids, 2 images per tile); with sel, each pair's first
// CTA also starts that pair's full-resolution select.
template <typename T>
__global__ void __launch_bounds__(256)
    k_b_resize_pair(NetLaunch L, const void *const *lt, const void *const *rt, float *lo,
                    float *ro, float *gh, SelState *sel, unsigned *sel_hist) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    const int tx = (P.Ww + 31) / 32, ty = (P.Hw + 7) / 8;
    const int bz = (int)(c & 1);
    const long long t = c >> 1;
    const int bx = (int)(t % tx), by = (int)(t / tx);
    if (by >= ty) return;
    const long long rank = (long long)__dmul_rn((double)((long long)P.W * P.H), 0.95);
    resize_pair_body<T>(bx, by, bz, c == 0, P.native != 0, static_cast<const T *>(lt[p]),
                        static_cast<const T *>(rt[p]), P.W, P.H, P.Ww, P.Hw, net_slab(lo, L, p),
                        net_slab(ro, L, p), net_slab(gh, L, p), net_slab(sel, L, p),
                        net_slab(sel_hist, L, p), rank);
}

// Copy (no resample) of a pair into FP32, for predict at native resolution.
template <typename T>
__global__ void k_to_f32_pair(const T *__restrict__ l, const T *__restrict__ r, long n,
                              float *__restrict__ lo, float *__restrict__ ro) {
    const T *src = blockIdx.y ? r : l;
    float *dst = blockIdx.y ? ro : lo;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        dst[i] = (float)gray_at<T>(src, (int)i);
}

// resize of an FP64 map (sv_resize) and of the FP32 network disparity back
// to full resolution, scaled by inv (predict_at_scale, stereonet.py:3957-3959).
template <typename T>
__global__ void k_resize_scale(const T *__restrict__ x, int W, int H, int W2, int H2,
                               double inv, int scale, double *__restrict__ out) {
    int ox = blockIdx.x * blockDim.x + threadIdx.x;
    int oy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ox >= W2 || oy >= H2) return;
    Taps t = bilinear_taps(oy, ox, H, W, H2, W2);
    double v = blend64<T>(x, t);
    out[(long)oy * W2 + ox] = scale ? __dmul_rn(v, inv) : v;
}

// predict_at_scale's two outputs from the FP32 work-resolution disparity in
// one launch: the full-resolution map, bilinear and times inv
// (stereonet.py:3957-3959), and the work map itself promoted to FP64 by the
// threads that fall inside it (the work map is never larger).
// With sel, also pass 0 of the stage's full-resolution select over the
// values it writes (the select's first histogram: ghist) -- or, with wf,
// the whole width decision over them (its last CTA writes the width into
// sel->value and *mirror).  A CTA of 32 x 8 threads covers `rows` slabs of
// 8 rows (one histogram and one hand-off per CTA: fewer, larger CTAs when
// the map is large).
__device__ __forceinline__ void work_outputs_body(int bx, int by, unsigned nblk, bool copy,
                                                  const float *__restrict__ d, int Ww, int Hw, int W, int H, double inv,
                   double *__restrict__ work64, double *__restrict__ full64, SelState *sel,
                   unsigned *ghist, const WidthFuse *wf = nullptr, double *mirror = nullptr,
                   int rows = 1) {
    __shared__ unsigned hist[SEL_NB + 1];
    if (sel) {                                     // the same for every CTA
        const int nb = wf ? wf->m + 1 : SEL_NB;
        for (int i = sel_tid(); i < nb; i += sel_nt()) hist[i] = 0u;
        __syncthreads();
    }
    const int ox = bx * blockDim.x + threadIdx.x;
    for (int r = 0; r < rows; ++r) {
        const int oy = (by * rows + r) * blockDim.y + threadIdx.y;
        const bool in = ox < W && oy < H;
        double v = 0.0;
        if (in) {
            if (copy) {                  // native resolution: the network output itself
                v = (double)d[(long)oy * W + ox];
            } else {
                const Taps t = bilinear_taps(oy, ox, Hw, Ww, H, W);
                v = __dmul_rn(blend64<float>(d, t), inv);
            }
            full64[(long)oy * W + ox] = v;
            if (work64 && ox < Ww && oy < Hw)
                work64[(long)oy * Ww + ox] = (double)d[(long)oy * Ww + ox];
        }
        if (!sel) continue;
        if (wf) width_count(hist, in ? width_bin_of(*wf, v) : -1);
        else sel_count(hist, sel_key(v), in, 0ull, 0);
    }
    if (!sel) return;
    __syncthreads();
    if (wf) width_finish(*wf, sel, ghist, hist, nblk, mirror);
    else sel_pass_finish(0, sel, ghist, hist, nblk);
}


__global__ void __launch_bounds__(256)
    k_work_outputs(const float *__restrict__ d, int Ww, int Hw, int W, int H, double inv,
                   double *__restrict__ work64, double *__restrict__ full64, SelState *sel,
                   unsigned *ghist, WidthFuse wf, double *mirror) {
    work_outputs_body(blockIdx.x, blockIdx.y, gridDim.x * gridDim.y * gridDim.z, false, d, Ww,
                      Hw, W, H, inv, work64, full64, sel, ghist, wf.m >= 0 ? &wf : nullptr,
                      mirror);
}

// Batched: every active pair's full-resolution map from its work map (the
// grid covers each pair's full size exactly), with pass 0 of its select.
// With a width rule (max_width > 0), the pair's whole width decision runs
// here (sel->value: the width); else pass 0 of its value select.
__global__ void __launch_bounds__(256)
    k_b_work_outputs(NetLaunch L, const float *d, double *work64, double *full64, SelState *sel,
                     unsigned *ghist, double target, int max_width) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    const int tx = (P.W + 31) / 32;
    const unsigned nblk = (unsigned)(L.pre[p + 1] - L.pre[p]);
    WidthFuse wf{{P.W, max_width, target, 1.0}, 0, 0, (long long)((long)P.W * P.H * 0.95)};
    wf.kmax = width_rule_kmax(wf.rule);
    wf.m = wf.kmax - 48;
    work_outputs_body((int)(c % tx), (int)(c / tx), nblk, P.native != 0, net_slab(d, L, p), P.Ww,
                      P.Hw, P.W,
                      P.H, P.inv, net_slab(work64, L, p), net_slab(full64, L, p),
                      net_slab(sel, L, p), net_slab(ghist, L, p),
                      max_width > 0 ? &wf : nullptr, nullptr, kWorkRowsBatched);
}

template <typename T>
__global__ void k_promote(const T *__restrict__ x, long n, double *__restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        out[i] = (double)x[i];
}

// avgpool2, stereonet.py:979-995: 0.25 * (((a + b) + c) + d).
__global__ void k_avgpool2(const float *__restrict__ img, int H, int W,
                           float *__restrict__ out) {
    int H2 = H / 2, W2 = W / 2;
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W2 || y >= H2) return;
    const float *r0 = img + (2 * y) * W + 2 * x;
    const float *r1 = r0 + W;
    out[y * W2 + x] = 0.25f * (((r0[0] + r0[1]) + r1[0]) + r1[1]);
}

// avgpool2 in FP64 over C planes (the drop-in for the reference function).
__global__ void k_avgpool2_f64(const double *__restrict__ img, int C, int H, int W,
                               double *__restrict__ out) {
    const int H2 = H / 2, W2 = W / 2;
    const long n = (long)C * H2 * W2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i / ((long)H2 * W2));
        const int rem = (int)(i - (long)c * H2 * W2);
        const int y = rem / W2, x = rem - (rem / W2) * W2;
        const double *r0 = img + (long)c * H * W + (long)(2 * y) * W + 2 * x;
        const double *r1 = r0 + W;
        out[i] = __dmul_rn(0.25, __dadd_rn(__dadd_rn(__dadd_rn(r0[0], r0[1]), r1[0]), r1[1]));
    }
}

// ------------------------------------------------------------- conv 2d
// Shared-memory tiled 3x3 conv2d: a CTA computes a CT2_TW x CT2_TH output
// tile for OCG output channels (blockIdx.z = image * OC/OCG + group).  The
// input tile with its halo, for every input channel, is staged once in
// shared memory (zeros outside the image, which adds exactly what the
// reference's skipped taps add: nothing); weights sit as [c][tap][o] so one
// vector load feeds OCG FMAs.  With CS > 1 each output's channel sum is
// split over CS lanes (IC / CS channels each, CT2_TW x CT2_TH x CS threads)
// and a butterfly of shuffles adds the parts: a shorter dependent chain per
// thread on these small, latency-bound images.  act: 0 none, 1 leaky 0.2,
// 2 residual + relu0 (the Refinement output, v > 0 ? v : v * 0).
constexpr int CT2_TW = 32, CT2_TH = 4;

// Channel plane stride of a staged tile: th * tw, padded for CS > 1 so that
// the CS lane groups of a warp (channels CPS planes apart, 32 / CS
// consecutive columns each) start 32 / CS banks apart.
__host__ __device__ inline int conv2d_plane(int th, int tw, int CPS, int CS) {
    const int p = th * tw;
    if (CS > 1)
        for (int k = 0; k < 64; ++k)
            if ((CPS * (p + k)) % 32 == 32 / CS) return p + k;
    return p;
}

template <int IC, int OC, int OCG, int ACT, int CS>
__device__ __forceinline__ void conv2d_tiled_body(int bx, int by, int bz, const float *__restrict__ x0, const float *__restrict__ x1, int H, int W,
                   int OH, int OW, int stride, int pad, int dil, const float *__restrict__ w,
                   const float *__restrict__ b, float *y0, float *y1,
                   const float *__restrict__ resid) {
    constexpr int NG = OC / OCG, NT = CT2_TW * CT2_TH * CS, CPS = IC / CS;
    static_assert(IC % CS == 0 && (CS == 1 || CS == 2 || CS == 4), "channel split");
    extern __shared__ __align__(16) float tile[];
    __shared__ __align__(16) float sw[IC * 9 * OCG];
    __shared__ float sb[OCG];
    const int img = bz / NG, og = bz - img * NG;
    const int tid = threadIdx.x;
    for (int i = tid; i < IC * 9 * OCG; i += NT) {
        const int o = i % OCG, ct = i / OCG;          // ct = c * 9 + tap
        sw[i] = w[(og * OCG + o) * IC * 9 + ct];
    }
    if (tid < OCG) sb[tid] = b[og * OCG + tid];
    const float *x = img ? x1 : x0;
    float *y = img ? y1 : y0;
    const int ox0 = bx * CT2_TW, oy0 = by * CT2_TH;
    const int ix0 = ox0 * stride - pad, iy0 = oy0 * stride - pad;
    const int tw = (CT2_TW - 1) * stride + 2 * dil + 1;
    const int th = (CT2_TH - 1) * stride + 2 * dil + 1;
    const int plane = conv2d_plane(th, tw, CPS, CS);
    const long HW = (long)H * W;
    for (int i = tid; i < IC * th * tw; i += NT) {
        const int c = i / (th * tw);
        const int rem = i - c * th * tw;
        const int ty = rem / tw, tx = rem - ty * tw;
        const int gy = iy0 + ty, gx = ix0 + tx;
        tile[c * plane + rem] = (gy >= 0 && gy < H && gx >= 0 && gx < W)
                                    ? __ldg(x + c * HW + (long)gy * W + gx)
                                    : 0.0f;
    }
    __syncthreads();
    const int lane = tid & 31, cs = lane / (32 / CS);
    const int pos = (tid >> 5) * (32 / CS) + lane % (32 / CS);
    const int lx = pos % CT2_TW, ly = pos / CT2_TW;
    float acc[OCG];
#pragma unroll
    for (int o = 0; o < OCG; ++o) acc[o] = 0.f;
    const int sy = ly * stride, sx = lx * stride;
#pragma unroll
    for (int j = 0; j < CPS; ++j) {
        const int c = cs * CPS + j;
        const float *tc = tile + c * plane;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
            const float *row = tc + (sy + ky * dil) * tw + sx;
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                const float v = row[kx * dil];
                const float *wt = sw + (c * 9 + ky * 3 + kx) * OCG;
                if (OCG % 4 == 0) {
#pragma unroll
                    for (int o = 0; o < OCG; o += 4) {
                        const float4 w4 = *reinterpret_cast<const float4 *>(wt + o);
                        acc[o] = fmaf(v, w4.x, acc[o]);
                        acc[o + 1] = fmaf(v, w4.y, acc[o + 1]);
                        acc[o + 2] = fmaf(v, w4.z, acc[o + 2]);
                        acc[o + 3] = fmaf(v, w4.w, acc[o + 3]);
                    }
                } else {
#pragma unroll
                    for (int o = 0; o < OCG; ++o) acc[o] = fmaf(v, wt[o], acc[o]);
                }
            }
        }
    }
#pragma unroll
    for (int o = 0; o < OCG; ++o)
#pragma unroll
        for (int m = 32 / CS; m < 32; m <<= 1) acc[o] += __shfl_xor_sync(kFull, acc[o], m);
    const int ox = ox0 + lx, oy = oy0 + ly;
    if (cs != 0 || ox >= OW || oy >= OH) return;
    const long OHW = (long)OH * OW, oi = (long)oy * OW + ox;
#pragma unroll
    for (int o = 0; o < OCG; ++o) {
        float v = acc[o] + sb[o];
        if (ACT == 1) v = v > 0.f ? v : v * 0.2f;
        if (ACT == 2) {
            v = resid[oi] + v;
            v = v > 0.f ? v : v * 0.f;
        }
        y[(og * OCG + o) * OHW + oi] = v;
    }
}


template <int IC, int OC, int OCG, int ACT, int CS>
__global__ void __launch_bounds__(CT2_TW *CT2_TH *CS)
    k_conv2d_tiled(const float *__restrict__ x0, const float *__restrict__ x1, int H, int W,
                   int OH, int OW, int stride, int pad, int dil, const float *__restrict__ w,
                   const float *__restrict__ b, float *y0, float *y1,
                   const float *__restrict__ resid) {
    conv2d_tiled_body<IC, OC, OCG, ACT, CS>(blockIdx.x, blockIdx.y, blockIdx.z, x0, x1, H, W,
                                            OH, OW, stride, pad, dil, w, b, y0, y1, resid);
}

// Input and output sizes of a batched 2-D convolution, from the pass's work
// size: 0 FeatureNet c1 (work -> half), 1 c2 (half -> quarter), 2 c3/c4
// (quarter), 3 Refinement level 0 (work / 2), 4 Refinement level 1 (work).
__device__ __forceinline__ void conv_level(int lv, int Hw, int Ww, int &H, int &W, int &OH,
                                           int &OW) {
    int h1, w1, h, w;
    net_quarter(Hw, Ww, h1, w1, h, w);
    switch (lv) {
    case 0: H = Hw; W = Ww; OH = h1; OW = w1; break;
    case 1: H = h1; W = w1; OH = h; OW = w; break;
    case 2: H = OH = h; W = OW = w; break;
    case 3: H = OH = Hw / 2; W = OW = Ww / 2; break;
    default: H = OH = Hw; W = OW = Ww; break;
    }
}

template <int IC, int OC, int OCG, int ACT, int CS>
__global__ void __launch_bounds__(CT2_TW *CT2_TH *CS)
    k_b_conv2d_tiled(NetLaunch L, int lv, int Z, const float *x0, const float *x1, int stride,
                     int pad, int dil, const float *__restrict__ w, const float *__restrict__ b,
                     float *y0, float *y1, const float *resid) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    int H, W, OH, OW;
    conv_level(lv, P.Hw, P.Ww, H, W, OH, OW);
    const int tx = (OW + CT2_TW - 1) / CT2_TW, ty = (OH + CT2_TH - 1) / CT2_TH;
    const int bz = (int)(c % Z);
    const long long t = c / Z;
    const int bx = (int)(t % tx), by = (int)(t / tx);
    if (by >= ty) return;
    conv2d_tiled_body<IC, OC, OCG, ACT, CS>(bx, by, bz, net_slab(x0, L, p), net_slab(x1, L, p),
                                            H, W, OH, OW, stride, pad, dil, w, b,
                                            net_slab(y0, L, p), net_slab(y1, L, p),
                                            net_slab(resid, L, p));
}

// 3x3 convolutions (padding = dilation; stride S = 1, or 2 with dilation 1)
// with every output channel in one thread and PX pixels per thread, CTB_TW /
// PX columns apart: the register-blocked form of k_conv2d_tiled<IC, OC, *,
// ACT, CS>.  It keeps that kernel's arithmetic exactly -- each of the CS
// channel groups' partial sums is its own fmaf chain over (channel, ky, kx)
// in the same order, combined as the butterfly combines them ((s0 + s1) +
// (s2 + s3) for CS = 4, s0 + s1 for CS = 2), then the bias and the activation
// -- so its results are bit-identical to that kernel's, from one staged
// input tile for all output channels and one 16-byte weight vector per 4
// output channels, read by the whole warp at once.
constexpr int CTB_TW = 32, CTB_TH = 4;          // output tile of a CTA

template <int IC, int OC, int ACT, int CS, int PX, int S>
__device__ __forceinline__ void conv2d_wide_body(int bx, int by, const float *__restrict__ x,
                                                 int H, int W, int OH, int OW, int dil,
                                                 const float *__restrict__ w,
                                                 const float *__restrict__ b, float *y,
                                                 const float *__restrict__ resid) {
    constexpr int CPS = IC / CS, TXP = CTB_TW / PX, NT = TXP * CTB_TH;
    constexpr int OCP = (OC + 3) / 4 * 4;
    static_assert(IC % CS == 0 && (CS == 1 || CS == 2 || CS == 4) && OC <= 16, "shape");
    static_assert(CTB_TW % PX == 0 && (S == 1 || S == 2), "tile");
    extern __shared__ __align__(16) float tile[];
    __shared__ __align__(16) float sw[IC * 9 * OCP];
    __shared__ float sb[OCP];
    const int tid = threadIdx.x;
    for (int i = tid; i < IC * 9 * OCP; i += NT) {
        const int o = i % OCP, ct = i / OCP;          // ct = c * 9 + tap
        sw[i] = o < OC ? w[o * IC * 9 + ct] : 0.f;
    }
    if (tid < OCP) sb[tid] = tid < OC ? b[tid] : 0.f;
    const int ox0 = bx * CTB_TW, oy0 = by * CTB_TH;
    const int ix0 = ox0 * S - dil, iy0 = oy0 * S - dil;
    const int tw = (CTB_TW - 1) * S + 2 * dil + 1, th = (CTB_TH - 1) * S + 2 * dil + 1;
    const long HW = (long)H * W;
    for (int i = tid; i < IC * th * tw; i += NT) {
        const int c = i / (th * tw);
        const int rem = i - c * th * tw;
        const int ty = rem / tw, tx = rem - ty * tw;
        const int gy = iy0 + ty, gx = ix0 + tx;
        tile[i] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? __ldg(x + c * HW + (long)gy * W + gx)
                                                           : 0.0f;
    }
    __syncthreads();
    const int lx = tid % TXP, ly = tid / TXP;
    float acc[CS][PX][OC];
#pragma unroll
    for (int g = 0; g < CS; ++g)
#pragma unroll
        for (int q = 0; q < PX; ++q)
#pragma unroll
            for (int o = 0; o < OC; ++o) acc[g][q][o] = 0.f;
#pragma unroll
    for (int g = 0; g < CS; ++g)
#pragma unroll
        for (int j = 0; j < CPS; ++j) {
            const int c = g * CPS + j;
            const float *tc = tile + c * th * tw;
#pragma unroll
            for (int ky = 0; ky < 3; ++ky) {
                const float *row = tc + (ly * S + ky * dil) * tw + lx * S;
#pragma unroll
                for (int kx = 0; kx < 3; ++kx) {
                    float v[PX];
#pragma unroll
                    for (int q = 0; q < PX; ++q) v[q] = row[kx * dil + q * TXP * S];
                    const float *wt = sw + (c * 9 + ky * 3 + kx) * OCP;
#pragma unroll
                    for (int o4 = 0; o4 < OCP; o4 += 4) {
                        const float4 w4 = *reinterpret_cast<const float4 *>(wt + o4);
                        const float wv[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (o4 + k < OC)
#pragma unroll
                                for (int q = 0; q < PX; ++q)
                                    acc[g][q][o4 + k] = fmaf(v[q], wv[k], acc[g][q][o4 + k]);
                    }
                }
            }
        }
    const long OHW = (long)OH * OW;
#pragma unroll
    for (int q = 0; q < PX; ++q) {
        const int ox = ox0 + lx + q * TXP, oy = oy0 + ly;
        if (ox >= OW || oy >= OH) continue;
        const long oi = (long)oy * OW + ox;
#pragma unroll
        for (int o = 0; o < OC; ++o) {
            float s;
            if (CS == 4) s = (acc[0][q][o] + acc[1][q][o]) + (acc[2][q][o] + acc[3][q][o]);
            else if (CS == 2) s = acc[0][q][o] + acc[1][q][o];
            else s = acc[0][q][o];
            float v = s + sb[o];
            if (ACT == 1) v = v > 0.f ? v : v * 0.2f;
            if (ACT == 2) {
                v = resid[oi] + v;
                v = v > 0.f ? v : v * 0.f;
            }
            y[o * OHW + oi] = v;
        }
    }
}

// The network's output convolution (Refinement level 1: RC -> 1, residual
// + ReLU, k_conv2d_tiled<RC, 1, 1, 2, 4>'s arithmetic) followed by a width
// decision over the values it wrote: each CTA histograms the widths of its
// tile's outputs and the last CTA turns the totals into the width
// (predict_auto's probe: no separate decision launch).
template <int RC>
__global__ void __launch_bounds__(CT2_TW *CT2_TH * 4)
    k_conv2d_out_decide(const float *__restrict__ x, int H, int W, const float *__restrict__ w,
                        const float *__restrict__ b, float *y, const float *__restrict__ resid,
                        WidthFuse f, SelState *s, unsigned *ghist, double *mirror) {
    __shared__ unsigned hist[kWidthBins + 1];
    const int t = threadIdx.x;
    for (int i = t; i <= f.m; i += CT2_TW * CT2_TH * 4) hist[i] = 0u;
    conv2d_tiled_body<RC, 1, 1, 2, 4>(blockIdx.x, blockIdx.y, 0, x, x, H, W, H, W, 1, 1, 1, w, b,
                                      y, y, resid);
    __syncthreads();                              // the tile's outputs are written
    int bin = -1;
    if (t < CT2_TW * CT2_TH) {
        const int ox = blockIdx.x * CT2_TW + t % CT2_TW, oy = blockIdx.y * CT2_TH + t / CT2_TW;
        if (ox < W && oy < H) bin = width_bin_of(f, (double)y[(long)oy * W + ox]);
    }
    width_count(hist, bin);
    __syncthreads();
    width_finish(f, s, ghist, hist, gridDim.x * gridDim.y, mirror);
}

// The batched form: level lv of conv_level, Z images (1 or 2) per pair.
template <int IC, int OC, int ACT, int CS, int PX, int S>
__global__ void __launch_bounds__(CTB_TW / PX * CTB_TH)
    k_b_conv2d_wide(NetLaunch L, int lv, int Z, const float *x0, const float *x1, int dil,
                    const float *__restrict__ w, const float *__restrict__ b, float *y0,
                    float *y1, const float *resid) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    int H, W, OH, OW;
    conv_level(lv, P.Hw, P.Ww, H, W, OH, OW);
    const int tx = (OW + CTB_TW - 1) / CTB_TW, ty = (OH + CTB_TH - 1) / CTB_TH;
    const int img = (int)(c % Z);
    const long long t = c / Z;
    const int bx = (int)(t % tx), by = (int)(t / tx);
    if (by >= ty) return;
    conv2d_wide_body<IC, OC, ACT, CS, PX, S>(bx, by, net_slab(img ? x1 : x0, L, p), H, W, OH,
                                             OW, dil, w, b, net_slab(img ? y1 : y0, L, p),
                                             net_slab(resid, L, p));
}

static size_t conv2d_wide_bytes(int IC, int S, int dil) {
    return (size_t)IC * ((CTB_TW - 1) * S + 2 * dil + 1) * ((CTB_TH - 1) * S + 2 * dil + 1) *
           sizeof(float);
}

template <int IC, int OC, int ACT, int CS, int PX, int S>
static void b_conv2d_wide(const NetLaunch &L, unsigned ctas, int lv, int Z, const float *x0,
                          const float *x1, int dil, const float *w, const float *b, float *y0,
                          float *y1, const float *resid, cudaStream_t st) {
    const size_t smem = conv2d_wide_bytes(IC, S, dil);
    constexpr size_t kStatic = (size_t)(IC * 9 + 1) * ((OC + 3) / 4 * 4) * sizeof(float);
    if (smem + kStatic > 48 * 1024)
        cudaFuncSetAttribute(k_b_conv2d_wide<IC, OC, ACT, CS, PX, S>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_b_conv2d_wide<IC, OC, ACT, CS, PX, S><<<ctas, CTB_TW / PX * CTB_TH, smem, st>>>(
        L, lv, Z, x0, x1, dil, w, b, y0, y1, resid);
}

// A Refinement level's first convolution (2 -> RC, stride 1, dilation dil,
// leaky ReLU) with the level's input built while staging: channel 0 is
// 2 * bilinear(prev) (BilinearUpsample.forward's half-pixel taps, FP64
// weights, and StereoNet.forward's x2, stereonet.py:1224-1229) and channel 1
// the guide, computed for every tile position (halo included), 0 outside the
// image.  The CTAs of channel group 0 also store channel 0 of
// their inner tile into rin0, the residual the level's last convolution adds.
template <int RC, int OCG>
__device__ __forceinline__ void conv2d_up_body(int bx, int by, int bz, const float *__restrict__ prev, int ph, int pw, const float *__restrict__ guide,
                int H, int W, int dil, const float *__restrict__ w, const float *__restrict__ b,
                float *__restrict__ y, float *__restrict__ rin0) {
    constexpr int IC = 2, NG = RC / OCG;
    extern __shared__ __align__(16) float tile[];
    __shared__ float sw[OCG * IC * 9];
    __shared__ float sb[OCG];
    const int og = bz % NG;
    const int tid = threadIdx.y * CT2_TW + threadIdx.x;
    for (int i = tid; i < OCG * IC * 9; i += CT2_TW * CT2_TH) sw[i] = w[og * OCG * IC * 9 + i];
    if (tid < OCG) sb[tid] = b[og * OCG + tid];
    const int ox0 = bx * CT2_TW, oy0 = by * CT2_TH;
    const int ix0 = ox0 - dil, iy0 = oy0 - dil;
    const int tw = CT2_TW + 2 * dil, th = CT2_TH + 2 * dil;
    for (int i = tid; i < th * tw; i += CT2_TW * CT2_TH) {
        const int ty = i / tw, tx = i - ty * tw;
        const int gy = iy0 + ty, gx = ix0 + tx;
        float v0 = 0.f, v1 = 0.f;
        if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
            const Taps t = bilinear_taps(gy, gx, ph, pw, H, W);
            const float v = __ldg(prev + t.i00) * (float)t.w00 + __ldg(prev + t.i01) * (float)t.w01 +
                            __ldg(prev + t.i10) * (float)t.w10 + __ldg(prev + t.i11) * (float)t.w11;
            v0 = v * 2.0f;
            v1 = __ldg(guide + (long)gy * W + gx);
            if (og == 0 && ty >= dil && ty < dil + CT2_TH && tx >= dil && tx < dil + CT2_TW)
                rin0[(long)gy * W + gx] = v0;
        }
        tile[i] = v0;
        tile[th * tw + i] = v1;
    }
    __syncthreads();
    const int ox = ox0 + threadIdx.x, oy = oy0 + threadIdx.y;
    if (ox >= W || oy >= H) return;
    float acc[OCG];
#pragma unroll
    for (int o = 0; o < OCG; ++o) acc[o] = sb[o];
#pragma unroll
    for (int c = 0; c < IC; ++c) {
        const float *tc = tile + c * th * tw;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
            const float *row = tc + (threadIdx.y + ky * dil) * tw + threadIdx.x;
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
                const float v = row[kx * dil];
#pragma unroll
                for (int o = 0; o < OCG; ++o)
                    acc[o] = fmaf(v, sw[(o * IC + c) * 9 + ky * 3 + kx], acc[o]);
            }
        }
    }
    const long HW = (long)H * W, oi = (long)oy * W + ox;
#pragma unroll
    for (int o = 0; o < OCG; ++o) {
        const float v = acc[o];
        y[(og * OCG + o) * HW + oi] = v > 0.f ? v : v * 0.2f;
    }
}


template <int RC, int OCG>
__global__ void __launch_bounds__(CT2_TW *CT2_TH)
    k_conv2d_up(const float *__restrict__ prev, int ph, int pw, const float *__restrict__ guide,
                int H, int W, int dil, const float *__restrict__ w, const float *__restrict__ b,
                float *__restrict__ y, float *__restrict__ rin0) {
    conv2d_up_body<RC, OCG>(blockIdx.x, blockIdx.y, blockIdx.z, prev, ph, pw, guide, H, W, dil,
                            w, b, y, rin0);
}

// Batched: level lv (0: from the quarter-size disparity to work / 2, 1: from
// work / 2 to the work size).
template <int RC, int OCG>
__global__ void __launch_bounds__(CT2_TW *CT2_TH)
    k_b_conv2d_up(NetLaunch L, int lv, const float *prev, const float *guide, int dil,
                  const float *__restrict__ w, const float *__restrict__ b, float *y,
                  float *rin0) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    int h1, w1, h, wq;
    net_quarter(P.Hw, P.Ww, h1, w1, h, wq);
    const int ph = lv ? P.Hw / 2 : h, pw = lv ? P.Ww / 2 : wq;
    const int H = lv ? P.Hw : P.Hw / 2, W = lv ? P.Ww : P.Ww / 2;
    constexpr int Z = RC / OCG;
    const int tx = (W + CT2_TW - 1) / CT2_TW, ty = (H + CT2_TH - 1) / CT2_TH;
    const int bz = (int)(c % Z);
    const long long t = c / Z;
    const int bx = (int)(t % tx), by = (int)(t / tx);
    if (by >= ty) return;
    conv2d_up_body<RC, OCG>(bx, by, bz, net_slab(prev, L, p), ph, pw, net_slab(guide, L, p), H, W,
                            dil, w, b, net_slab(y, L, p), net_slab(rin0, L, p));
}

static size_t conv2d_tile_bytes(int IC, int stride, int dil, int CS = 1) {
    const int th = (CT2_TH - 1) * stride + 2 * dil + 1, tw = (CT2_TW - 1) * stride + 2 * dil + 1;
    return (size_t)IC * conv2d_plane(th, tw, IC / CS, CS) * sizeof(float);
}

// ------------------------------------------------------------ conv 3d
// The 3-D convolutions run on volumes of a few thousand voxels (w x h x D at
// 1/4 resolution, D <= 16), so their cost is the latency of one thread's
// chain of taps, not bandwidth or FLOPs.  A CTA stages its input tile --
// 8 columns x TD disparities x 1 row plus the 3x3x3 halo, every input
// channel -- in shared memory, zeros outside the volume (a zero tap adds
// exactly what the reference's skipped tap adds: nothing), and each output
// voxel's channel sum is split over CS lanes (C / CS channels each) that a
// butterfly of shuffles adds up.  Plane and disparity strides of the tile
// are padded so that the 32 lanes of a warp read 32 distinct banks.
constexpr int C3_TX = 8;                 // columns per CTA
constexpr int C3_RS = C3_TX + 2;         // tile row stride (halo included)

// True when the lanes of a warp (lane = position * CS + split, positions
// 8 columns wide) hit distinct shared-memory banks for plane stride P and
// disparity stride DS.
__host__ __device__ constexpr bool c3_banks_ok(int CS, int CPS, int DS, int P) {
    bool used[32] = {};
    for (int lane = 0; lane < 32; ++lane) {
        const int cs = lane % CS, pl = lane / CS;
        const int bank = (cs * CPS * P + (pl / C3_TX) * DS + pl % C3_TX) % 32;
        if (used[bank]) return false;
        used[bank] = true;
    }
    return true;
}

// The smallest conflict-free (DS, P): which = 0 gives DS, 1 gives P, -1 if
// none exists within 32 of the unpadded strides.
__host__ __device__ constexpr int c3_layout(int CS, int CPS, int TD, int which) {
    for (int ds = 3 * C3_RS; ds < 3 * C3_RS + 32; ++ds)
        for (int pl = (TD + 2) * ds; pl < (TD + 2) * ds + 32; ++pl)
            if (c3_banks_ok(CS, CPS, ds, pl)) return which == 0 ? ds : pl;
    return -1;
}

// Stages rows d0-1 .. d0+TD, y-1 .. y+1, x0-1 .. x0+8 of every channel.
// CV: the cost volume of CostVolume.forward (stereonet.py:771-799) built on
// the fly -- |fl(x) - fr(x - d)|, 2.0 where x - d < 0; else x is a C x D x h
// x w volume.  The global loads of C3_SB elements per thread are issued
// before any of them is used, so a CTA waits for about one memory latency
// per C3_SB elements instead of one per element (these small launches are
// bound by that latency).
constexpr int C3_SB = 8;

template <int C, int TD, int DS, int P, int NT, bool CV, int RS = C3_RS>
__device__ __forceinline__ void c3_stage(float *tile, const float *__restrict__ a,
                                         const float *__restrict__ bsrc, int D, int h, int w,
                                         int x0, int oy, int d0) {
    const long hw = (long)h * w;
    if constexpr (CV) {
        // The cost volume reads each left-feature value of the tile's rows
        // once per disparity and each right-feature value once per (x, d)
        // with the same x - d: stage the distinct ones (3 rows x RS left,
        // 3 rows x (RS + TD + 1) right per channel), then build the tile
        // from shared memory, lane l < 30 of a warp owning tile row l / 10,
        // column l % 10 and the warps taking the (channel, disparity)
        // slices in turn.
        constexpr int RW = RS + TD + 1, NL = C * 3 * RS, NR = C * 3 * RW;
        constexpr int NW = NT / 32, G = C * (TD + 2);
        __shared__ float sl[NL], sr[NR];
        const int xr0 = x0 - 1 - (d0 + TD);
        for (int i0 = threadIdx.x; i0 < NL + NR; i0 += NT * C3_SB) {
            float v[C3_SB];
#pragma unroll
            for (int u = 0; u < C3_SB; ++u) {
                const int i = i0 + u * NT;
                v[u] = 0.f;
                if (i < NL) {
                    const int c = i / (3 * RS), r = i - c * 3 * RS;
                    const int ry = r / RS, rx = r - ry * RS;
                    const int yy = oy - 1 + ry, xx = x0 - 1 + rx;
                    if (yy >= 0 && yy < h && xx >= 0 && xx < w)
                        v[u] = __ldg(a + c * hw + (long)yy * w + xx);
                } else if (i < NL + NR) {
                    const int j = i - NL;
                    const int c = j / (3 * RW), r = j - c * 3 * RW;
                    const int ry = r / RW, k = r - ry * RW;
                    const int yy = oy - 1 + ry, xx = xr0 + k;
                    if (yy >= 0 && yy < h && xx >= 0 && xx < w)
                        v[u] = __ldg(bsrc + c * hw + (long)yy * w + xx);
                }
            }
#pragma unroll
            for (int u = 0; u < C3_SB; ++u) {
                const int i = i0 + u * NT;
                if (i < NL) sl[i] = v[u];
                else if (i < NL + NR) sr[i - NL] = v[u];
            }
        }
        __syncthreads();
        const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
        for (int e = lane; e < 3 * RS; e += 32) {
            const int ry = e / RS, rx = e - ry * RS;
            const int yy = oy - 1 + ry, xx = x0 - 1 + rx;
            const bool pix = yy >= 0 && yy < h && xx >= 0 && xx < w;
            const float *slp = sl + e, *srp = sr + ry * RW + rx + TD + 1;
            float *tl = tile + ry * RS + rx;
#pragma unroll 4
            for (int g = wp; g < G; g += NW) {
                const int c = g / (TD + 2), dz = g - c * (TD + 2);
                const int dd = d0 - 1 + dz;
                float v = 0.f;
                if (pix && dd >= 0 && dd < D)
                    v = xx - dd < 0 ? 2.0f : fabsf(slp[c * 3 * RS] - srp[c * 3 * RW - dz]);
                tl[c * P + dz * DS] = v;
            }
        }
    } else {
        constexpr int PER_C = (TD + 2) * 3 * RS, TOTAL = C * PER_C;
        for (int i0 = threadIdx.x; i0 < TOTAL; i0 += NT * C3_SB) {
            float va[C3_SB];
            int slot[C3_SB];
#pragma unroll
            for (int u = 0; u < C3_SB; ++u) {
                const int i = i0 + u * NT;
                slot[u] = -1;
                va[u] = 0.f;
                if (i < TOTAL) {
                    const int c = i / PER_C;
                    int r = i - c * PER_C;
                    const int dz = r / (3 * RS);
                    r -= dz * 3 * RS;
                    const int ry = r / RS, rx = r - ry * RS;
                    const int dd = d0 - 1 + dz, yy = oy - 1 + ry, xx = x0 - 1 + rx;
                    slot[u] = c * P + dz * DS + ry * RS + rx;
                    if (dd >= 0 && dd < D && yy >= 0 && yy < h && xx >= 0 && xx < w)
                        va[u] = __ldg(a + (c * (long)D + dd) * hw + (long)yy * w + xx);
                }
            }
#pragma unroll
            for (int u = 0; u < C3_SB; ++u)
                if (slot[u] >= 0) tile[slot[u]] = va[u];
        }
    }
}

// One lane's share of a voxel: channels cs*CPS .. +CPS of the 27 taps, for
// OCG output channels (weights [c][tap][o] in shared memory).
template <int CPS, int OCG, int DS, int P>
__device__ __forceinline__ void c3_taps(const float *tb, const float *wb, float (&acc)[OCG]) {
#pragma unroll
    for (int j = 0; j < CPS; ++j)
#pragma unroll
        for (int kd = 0; kd < 3; ++kd)
#pragma unroll
            for (int ky = 0; ky < 3; ++ky)
#pragma unroll
                for (int kx = 0; kx < 3; ++kx) {
                    const float v = tb[j * P + kd * DS + ky * C3_RS + kx];
                    const float *wt = wb + (j * 27 + kd * 9 + ky * 3 + kx) * OCG;
                    if (OCG % 2 == 0) {
#pragma unroll
                        for (int o = 0; o < OCG; o += 2) {
                            const float2 ww = *reinterpret_cast<const float2 *>(wt + o);
                            acc[o] = fmaf(v, ww.x, acc[o]);
                            acc[o + 1] = fmaf(v, ww.y, acc[o + 1]);
                        }
                    } else {
#pragma unroll
                        for (int o = 0; o < OCG; ++o) acc[o] = fmaf(v, wt[o], acc[o]);
                    }
                }
}

template <int OCG, int CS>
__device__ __forceinline__ void c3_reduce(float (&acc)[OCG]) {
#pragma unroll
    for (int o = 0; o < OCG; ++o)
#pragma unroll
        for (int m = 1; m < CS; m <<= 1) acc[o] += __shfl_xor_sync(kFull, acc[o], m);
}

// Conv3d #1 (with the cost volume built while staging, CV) or #2 of
// CostFilter (stereonet.py:596-641, leaky ReLU 0.2): C -> OC channels, OCG
// per CTA (blockIdx.z), 128 threads = 8 columns x TD disparities x CS splits.
template <int C, int OCG, int CS, bool CV>
__device__ __forceinline__ void conv3d_split_body(int bx, int by, int bz, const float *__restrict__ a, const float *__restrict__ bsrc, int D, int h,
                   int w, const float *__restrict__ wt, const float *__restrict__ bias,
                   float *__restrict__ y) {
    constexpr int CPS = C / CS, TD = 16 / CS;
    constexpr int DS = c3_layout(CS, CPS, TD, 0), P = c3_layout(CS, CPS, TD, 1);
    static_assert(C % CS == 0 && (CS == 2 || CS == 4) && DS > 0, "tile layout");
    __shared__ float tile[C * P];
    __shared__ __align__(16) float sw[C * 27 * OCG];
    __shared__ float sb[OCG];
    const int og = bz, nd = (D + TD - 1) / TD;
    const int x0 = bx * C3_TX, oy = by / nd, d0 = (by - oy * nd) * TD;
    const int tid = threadIdx.x;
    for (int i0 = tid; i0 < C * 27 * OCG; i0 += 128 * C3_SB) {
        float v[C3_SB];
#pragma unroll
        for (int u = 0; u < C3_SB; ++u) {
            const int i = i0 + u * 128, o = i % OCG, ct = i / OCG;   // ct = c * 27 + tap
            v[u] = i < C * 27 * OCG ? __ldg(wt + (og * OCG + o) * C * 27 + ct) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < C3_SB; ++u)
            if (i0 + u * 128 < C * 27 * OCG) sw[i0 + u * 128] = v[u];
    }
    if (tid < OCG) sb[tid] = __ldg(bias + og * OCG + tid);
    c3_stage<C, TD, DS, P, 128, CV>(tile, a, bsrc, D, h, w, x0, oy, d0);
    __syncthreads();
    const int lane = tid & 31, cs = lane % CS, pos = (tid >> 5) * (32 / CS) + lane / CS;
    const int px = pos % C3_TX, pd = pos / C3_TX;
    float acc[OCG];
#pragma unroll
    for (int o = 0; o < OCG; ++o) acc[o] = 0.f;
    c3_taps<CPS, OCG, DS, P>(tile + cs * CPS * P + pd * DS + px, sw + cs * CPS * 27 * OCG, acc);
    c3_reduce<OCG, CS>(acc);
    const int ox = x0 + px, od = d0 + pd;
    if (cs != 0 || ox >= w || od >= D) return;
    const long hw = (long)h * w, total = (long)D * hw, idx = (long)od * hw + (long)oy * w + ox;
#pragma unroll
    for (int o = 0; o < OCG; ++o) {
        const float v = acc[o] + sb[o];
        y[(og * OCG + o) * total + idx] = v > 0.f ? v : v * 0.2f;
    }
}


template <int C, int OCG, int CS, bool CV>
__global__ void __launch_bounds__(128)
    k_conv3d_split(const float *__restrict__ a, const float *__restrict__ bsrc, int D, int h,
                   int w, const float *__restrict__ wt, const float *__restrict__ bias,
                   float *__restrict__ y) {
    conv3d_split_body<C, OCG, CS, CV>(blockIdx.x, blockIdx.y, blockIdx.z, a, bsrc, D, h, w, wt,
                                      bias, y);
}

// Batched CostFilter c1 (cost volume built on the fly) or c2, at the pass's
// quarter size; Z output-channel groups.
template <int C, int OCG, int CS, bool CV>
__global__ void __launch_bounds__(128)
    k_b_conv3d_split(NetLaunch L, int Z, const float *a, const float *bsrc, int D,
                     const float *__restrict__ wt, const float *__restrict__ bias, float *y) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    int h1, w1, h, w;
    net_quarter(P.Hw, P.Ww, h1, w1, h, w);
    constexpr int TD = 16 / CS;
    const int nd = (D + TD - 1) / TD;
    const int tx = (w + C3_TX - 1) / C3_TX, ty = h * nd;
    const int bz = (int)(c % Z);
    const long long t = c / Z;
    const int bx = (int)(t % tx), by = (int)(t / tx);
    if (by >= ty) return;
    conv3d_split_body<C, OCG, CS, CV>(bx, by, bz, net_slab(a, L, p), net_slab(bsrc, L, p), D, h,
                                      w, wt, bias, net_slab(y, L, p));
}

// Register-blocked CostFilter convolutions for the batch, where the launch
// is bound by throughput rather than one CTA's latency: the arithmetic of
// k_conv3d_split<C, OC, CS, CV> (each of the CS channel groups' partial
// sums an fmaf chain over (channel, kd, ky, kx) in that order, combined by
// the same xor butterfly, then bias and leaky ReLU) with every thread
// computing C3W_V neighbouring columns: the C3W_V + 2 tile values of a
// (channel, kd, ky) row are read once and feed 3 * C3W_V taps, and one
// 16-byte weight vector feeds C3W_V voxels.  A CTA covers 8 * C3W_V columns
// x TD disparities of one row (128 threads: 8 column groups x TD x CS).
// Bit-identical to k_conv3d_split.
constexpr int C3W_XP = 8, C3W_V = 2;

// Largest number of lanes of a warp that share a bank for plane stride P
// and disparity stride DS (lane = position * CS + split).
__host__ __device__ constexpr int c3w_conflicts(int CS, int CPS, int DS, int P) {
    int cnt[32] = {};
    int worst = 0;
    for (int lane = 0; lane < 32; ++lane) {
        const int cs = lane % CS, pl = lane / CS;
        const int bank = (cs * CPS * P + (pl / C3W_XP) * DS + (pl % C3W_XP) * C3W_V) % 32;
        cnt[bank] += 1;
        if (cnt[bank] > worst) worst = cnt[bank];
    }
    return worst;
}

// Disparity and plane strides (words) with the fewest bank conflicts.
__host__ __device__ constexpr int c3w_layout(int CS, int CPS, int TD, int RS, int which) {
    int best = 33, bds = 0, bp = 0;
    for (int ds = 3 * RS; ds < 3 * RS + 32; ++ds)
        for (int pl = (TD + 2) * ds; pl < (TD + 2) * ds + 32; ++pl) {
            const int c = c3w_conflicts(CS, CPS, ds, pl);
            if (c < best) {
                best = c;
                bds = ds;
                bp = pl;
            }
        }
    return which == 0 ? bds : bp;
}

template <int C, int CS>
struct C3W {
    static constexpr int CPS = C / CS, TD = 128 / (C3W_XP * CS), TX = C3W_XP * C3W_V;
    static constexpr int RS = TX + 2;
    static constexpr int DS = c3w_layout(CS, CPS, TD, RS, 0);
    static constexpr int P = c3w_layout(CS, CPS, TD, RS, 1);
};

template <int C, int OC, int CS, bool CV>
__device__ __forceinline__ void conv3d_wide_body(int bx, int by, const float *__restrict__ a,
                                                 const float *__restrict__ bsrc, int D, int h,
                                                 int w, const float *__restrict__ wt,
                                                 const float *__restrict__ bias,
                                                 float *__restrict__ y) {
    using G = C3W<C, CS>;
    constexpr int CPS = G::CPS, TD = G::TD, TX = G::TX, RS = G::RS, DS = G::DS, P = G::P;
    constexpr int OCP = (OC + 3) / 4 * 4, V = C3W_V;
    static_assert(C % CS == 0 && (CS == 2 || CS == 4) && OC <= 8, "shape");
    __shared__ float tile[C * P];
    __shared__ __align__(16) float sw[C * 27 * OCP];
    __shared__ float sb[OCP];
    const int tid = threadIdx.x;
    for (int i0 = tid; i0 < C * 27 * OCP; i0 += 128 * C3_SB) {
        float v[C3_SB];
#pragma unroll
        for (int u = 0; u < C3_SB; ++u) {
            const int i = i0 + u * 128, o = i % OCP, ct = i / OCP;   // ct = c * 27 + tap
            v[u] = (i < C * 27 * OCP && o < OC) ? __ldg(wt + o * C * 27 + ct) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < C3_SB; ++u)
            if (i0 + u * 128 < C * 27 * OCP) sw[i0 + u * 128] = v[u];
    }
    if (tid < OCP) sb[tid] = tid < OC ? __ldg(bias + tid) : 0.f;
    const int nd = (D + TD - 1) / TD;
    const int x0 = bx * TX, oy = by / nd, d0 = (by - oy * nd) * TD;
    c3_stage<C, TD, DS, P, 128, CV, RS>(tile, a, bsrc, D, h, w, x0, oy, d0);
    __syncthreads();
    const int lane = tid & 31, cs = lane % CS, pos = (tid >> 5) * (32 / CS) + lane / CS;
    const int px = pos % C3W_XP, pd = pos / C3W_XP;
    float acc[V][OC];
#pragma unroll
    for (int q = 0; q < V; ++q)
#pragma unroll
        for (int o = 0; o < OC; ++o) acc[q][o] = 0.f;
    const float *tb = tile + cs * CPS * P + pd * DS + px * V;
    const float *wb = sw + cs * CPS * 27 * OCP;
#pragma unroll
    for (int j = 0; j < CPS; ++j)
#pragma unroll
        for (int kd = 0; kd < 3; ++kd)
#pragma unroll
            for (int ky = 0; ky < 3; ++ky) {
                float r[V + 2];
#pragma unroll
                for (int i = 0; i < V + 2; ++i) r[i] = tb[j * P + kd * DS + ky * RS + i];
#pragma unroll
                for (int kx = 0; kx < 3; ++kx) {
                    const float *wp = wb + (j * 27 + kd * 9 + ky * 3 + kx) * OCP;
#pragma unroll
                    for (int o4 = 0; o4 < OCP; o4 += 4) {
                        const float4 w4 = *reinterpret_cast<const float4 *>(wp + o4);
                        const float wv[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (o4 + k < OC)
#pragma unroll
                                for (int q = 0; q < V; ++q)
                                    acc[q][o4 + k] = fmaf(r[q + kx], wv[k], acc[q][o4 + k]);
                    }
                }
            }
#pragma unroll
    for (int q = 0; q < V; ++q)
#pragma unroll
        for (int o = 0; o < OC; ++o)
#pragma unroll
            for (int m = 1; m < CS; m <<= 1) acc[q][o] += __shfl_xor_sync(kFull, acc[q][o], m);
    const int od = d0 + pd;
    if (cs != 0 || od >= D) return;
    const long hw = (long)h * w, total = (long)D * hw;
#pragma unroll
    for (int q = 0; q < V; ++q) {
        const int ox = x0 + px * V + q;
        if (ox >= w) continue;
        const long idx = (long)od * hw + (long)oy * w + ox;
#pragma unroll
        for (int o = 0; o < OC; ++o) {
            const float u = acc[q][o] + sb[o];
            y[o * total + idx] = u > 0.f ? u : u * 0.2f;
        }
    }
}

// Batched CostFilter c1 (cost volume built on the fly) or c2 at the pass's
// quarter size, register-blocked.
template <int C, int OC, int CS, bool CV>
__global__ void __launch_bounds__(128)
    k_b_conv3d_wide(NetLaunch L, const float *a, const float *bsrc, int D,
                    const float *__restrict__ wt, const float *__restrict__ bias, float *y) {
    using G = C3W<C, CS>;
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    int h1, w1, h, w;
    net_quarter(P.Hw, P.Ww, h1, w1, h, w);
    const int nd = (D + G::TD - 1) / G::TD;
    const int tx = (w + G::TX - 1) / G::TX, ty = h * nd;
    const int bx = (int)(c % tx), by = (int)(c / tx);
    if (by >= ty) return;
    conv3d_wide_body<C, OC, CS, CV>(bx, by, net_slab(a, L, p), net_slab(bsrc, L, p), D, h, w,
                                    wt, bias, net_slab(y, L, p));
}

// ----------------------------------- conv3d #3 + invalid mask + soft-argmin
// Conv3d #3 (Cm -> 1), CostVolume.invalid_mask (+8 where x < d, d >= 1,
// stereonet.py:827-840) and SoftArgmin.forward (858-885) in FP32 with
// max-subtraction: disp = sum_d d * exp(-c_d - max(-c)) / sum_d exp(...).
// A CTA is 8 columns x all D (<= 16) disparities of one row, each voxel's
// channel sum split over CS lanes as above; then 16 lanes per column reduce
// the soft-argmin over d with shuffles.
constexpr int SA_DMAX = 16;

template <int IC, int CS>
__device__ __forceinline__ void conv3d_softargmin_body(int bx, int by, const float *__restrict__ x, int D, int h, int w,
                        const float *__restrict__ wt, const float *__restrict__ b,
                        float *__restrict__ disp, float *__restrict__ spread, float *__restrict__ pmax) {
    constexpr int CPS = IC / CS, TD = SA_DMAX, NT = 128 * CS;
    constexpr int DS = c3_layout(CS, CPS, TD, 0), P = c3_layout(CS, CPS, TD, 1);
    static_assert(IC % CS == 0 && DS > 0, "tile layout");
    __shared__ float tile[IC * P];
    __shared__ float sw[IC * 27];
    __shared__ float cost[SA_DMAX][C3_TX + 1];
    const int tid = threadIdx.x;
    for (int i = tid; i < IC * 27; i += NT) sw[i] = __ldg(wt + i);
    const int x0 = bx * C3_TX, oy = by;
    c3_stage<IC, TD, DS, P, NT, false>(tile, x, nullptr, D, h, w, x0, oy, 0);
    __syncthreads();
    {
        const int lane = tid & 31, cs = lane % CS, pos = (tid >> 5) * (32 / CS) + lane / CS;
        const int px = pos % C3_TX, pd = pos / C3_TX;
        float acc[1] = {0.f};
        c3_taps<CPS, 1, DS, P>(tile + cs * CPS * P + pd * DS + px, sw + cs * CPS * 27, acc);
        c3_reduce<1, CS>(acc);
        if (cs == 0) {
            float v = acc[0] + __ldg(b);
            if (pd >= 1 && x0 + px < pd) v += 8.0f;
            cost[pd][px] = v;
        }
    }
    __syncthreads();
    if (tid >= C3_TX * SA_DMAX) return;
    // 16 lanes per column: lane d holds -cost_d
    const int px = tid / SA_DMAX, d = tid % SA_DMAX, ox = x0 + px;
    const bool live = d < D;
    const float nc = live ? -cost[d][px] : -INFINITY;
    float best = nc;
#pragma unroll
    for (int m = 1; m < SA_DMAX; m <<= 1) best = fmaxf(best, __shfl_xor_sync(kFull, best, m));
    const float e = live ? expf(nc - best) : 0.f;
    float te = e, td = (float)d * e;
#pragma unroll
    for (int m = 1; m < SA_DMAX; m <<= 1) {
        te += __shfl_xor_sync(kFull, te, m);
        td += __shfl_xor_sync(kFull, td, m);
    }
    if (d == 0 && ox < w) disp[(long)oy * w + ox] = td / te;
    if (!spread) return;                           // the same for the whole CTA
    // the distribution's spread and its peak probability (the exponent of
    // the best disparity is 1): how sure the network is of this disparity
    float t2 = (float)d * (float)d * e;
#pragma unroll
    for (int m = 1; m < SA_DMAX; m <<= 1) t2 += __shfl_xor_sync(kFull, t2, m);
    if (d == 0 && ox < w) {
        const float mu = td / te;
        spread[(long)oy * w + ox] = sqrtf(fmaxf(t2 / te - mu * mu, 0.f));
        pmax[(long)oy * w + ox] = 1.f / te;
    }
}



template <int IC, int CS>
__global__ void __launch_bounds__(128 * CS)
    k_conv3d_softargmin(const float *__restrict__ x, int D, int h, int w,
                        const float *__restrict__ wt, const float *__restrict__ b,
                        float *__restrict__ disp, float *__restrict__ spread,
                        float *__restrict__ pmax) {
    conv3d_softargmin_body<IC, CS>(blockIdx.x, blockIdx.y, x, D, h, w, wt, b, disp, spread, pmax);
}

template <int IC, int CS>
__global__ void __launch_bounds__(128 * CS)
    k_b_conv3d_softargmin(NetLaunch L, const float *x, int D, const float *__restrict__ wt,
                          const float *__restrict__ b, float *disp) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    int h1, w1, h, w;
    net_quarter(P.Hw, P.Ww, h1, w1, h, w);
    const int tx = (w + C3_TX - 1) / C3_TX;
    const int bx = (int)(c % tx), by = (int)(c / tx);
    if (by >= h) return;
    conv3d_softargmin_body<IC, CS>(bx, by, net_slab(x, L, p), D, h, w, wt, b,
                                   net_slab(disp, L, p), nullptr, nullptr);
}

// ====================================================================
// Host side
// ====================================================================

static dim3 grid2d(int W, int H, dim3 blk, int z = 1) {
    return dim3((W + blk.x - 1) / blk.x, (H + blk.y - 1) / blk.y, z);
}

int launch_resize_pair(const void *l, const void *r, int dtype, int W, int H, int W2, int H2,
                       float *lo, float *ro, cudaStream_t st, float *gh, const SelFuse *fuse) {
    SelState *ss = fuse ? fuse->state : nullptr;
    unsigned *sh = fuse ? fuse->hist : nullptr;
    const long long sr = fuse ? fuse->rank : 0;
    dim3 blk(32, 8);
    dim3 g = grid2d(W2, H2, blk, 2);
    if (W2 == W && H2 == H) {
        // a resample to the same size still runs the reference's arithmetic
    }
    switch (dtype) {
    case SV_U8: count_launch(); k_resize_pair<uint8_t><<<g, blk, 0, st>>>((const uint8_t *)l, (const uint8_t *)r, W, H, W2, H2, lo, ro, gh, ss, sh, sr); break;
    case SV_F32: count_launch(); k_resize_pair<float><<<g, blk, 0, st>>>((const float *)l, (const float *)r, W, H, W2, H2, lo, ro, gh, ss, sh, sr); break;
    case SV_F64: count_launch(); k_resize_pair<double><<<g, blk, 0, st>>>((const double *)l, (const double *)r, W, H, W2, H2, lo, ro, gh, ss, sh, sr); break;
    default: set_error("unknown dtype %d", dtype); return SV_ERR_PARAM;
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_to_f32_pair(const void *l, const void *r, int dtype, long n, float *lo, float *ro,
                       cudaStream_t st) {
    dim3 g(grid_for(n, 256), 2);
    switch (dtype) {
    case SV_U8: count_launch(); k_to_f32_pair<uint8_t><<<g, 256, 0, st>>>((const uint8_t *)l, (const uint8_t *)r, n, lo, ro); break;
    case SV_F32: count_launch(); k_to_f32_pair<float><<<g, 256, 0, st>>>((const float *)l, (const float *)r, n, lo, ro); break;
    case SV_F64: count_launch(); k_to_f32_pair<double><<<g, 256, 0, st>>>((const double *)l, (const double *)r, n, lo, ro); break;
    default: set_error("unknown dtype %d", dtype); return SV_ERR_PARAM;
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_resize_f64(const double *x, int W, int H, int W2, int H2, double *out,
                      cudaStream_t st) {
    dim3 blk(32, 8);
    count_launch(); k_resize_scale<double><<<grid2d(W2, H2, blk), blk, 0, st>>>(x, W, H, W2, H2, 1.0, 0, out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_upscale_disp(const float *dw, int Ww, int Hw, int W, int H, double inv,
                        double *out, cudaStream_t st) {
    dim3 blk(32, 8);
    count_launch(); k_resize_scale<float><<<grid2d(W, H, blk), blk, 0, st>>>(dw, Ww, Hw, W, H, inv, 1, out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_resize_f32(const float *x, int W, int H, int W2, int H2, double *out,
                      cudaStream_t st) {
    dim3 blk(32, 8);
    count_launch(); k_resize_scale<float><<<grid2d(W2, H2, blk), blk, 0, st>>>(x, W, H, W2, H2, 1.0, 0, out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_work_outputs(const float *d, int Ww, int Hw, int W, int H, double inv,
                        double *work64, double *full64, cudaStream_t st, const SelFuse *fuse) {
    if (Ww > W || Hw > H) {
        set_error("work map %dx%d larger than %dx%d", Ww, Hw, W, H);
        return SV_ERR_SHAPE;
    }
    dim3 blk(32, 8);
    count_launch();
    const WidthFuse wf = fuse && fuse->width ? *fuse->width : WidthFuse{{0, 0, 0.0, 0.0}, -1, 0, 0};
    k_work_outputs<<<grid2d(W, H, blk), blk, 0, st>>>(d, Ww, Hw, W, H, inv, work64, full64,
                                                       fuse ? fuse->state : nullptr,
                                                       fuse ? fuse->hist : nullptr, wf,
                                                       fuse ? fuse->mirror : nullptr);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_promote(const float *x, long n, double *out, cudaStream_t st) {
    count_launch(); k_promote<float><<<grid_for(n, 256), 256, 0, st>>>(x, n, out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_avgpool2_f64(const double *img, int C, int H, int W, double *out, cudaStream_t st) {
    long n = (long)C * (H / 2) * (W / 2);
    if (n > 0) {
        count_launch();
        k_avgpool2_f64<<<grid_for(n, 256), 256, 0, st>>>(img, C, H, W, out);
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_avgpool2(const float *img, int H, int W, float *out, cudaStream_t st) {
    dim3 blk(32, 8);
    count_launch(); k_avgpool2<<<grid2d(W / 2, H / 2, blk), blk, 0, st>>>(img, H, W, out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

// BF16 precision, FeatureNet and CostFilter c1/c2 on the tensor cores: the
// four feature convolutions (both images per launch), the cost volume fused
// into CostFilter c1, and CostFilter c2.  Their FP32 outputs feed the same
// CostFilter c3 + soft-argmin and Refinement kernels as the FP32 path.
static int forward_bf16_front(const NetView &n, const float *left, const float *right, int H,
                              int W, int h1, int w1, int h, int w, const FwdBufs &b,
                              cudaStream_t st) {
    SV_CUDA_TRY(cudaMemsetAsync(b.flag, 0, sizeof(int), st));
    const int C = n.C, Cm = n.Cm;
    TcConv a{};
    a.mode = 0;
    a.nd = 2;
    a.nimg = 2;
    a.D = a.OD = 1;
    a.pad = a.dil = 1;
    a.act = 1;
    a.err = b.flag;
    // c1..c4: (input, in size, out size, stride)
    const float *in[4][2] = {{left, right}, {b.fa[0], b.fa[1]}, {b.fb[0], b.fb[1]},
                             {b.fa[0], b.fa[1]}};
    float *out[4][2] = {{b.fa[0], b.fa[1]}, {b.fb[0], b.fb[1]}, {b.fa[0], b.fa[1]},
                        {b.fb[0], b.fb[1]}};
    const int ih[4] = {H, h1, h, h}, iw[4] = {W, w1, w, w};
    const int oh[4] = {h1, h, h, h}, ow[4] = {w1, w, w, w};
    for (int l = 0; l < 4; ++l) {
        a.IC = l == 0 ? 1 : C;
        a.OC = C;
        a.K = a.IC * 9;
        a.Kpad = tc_kpad(a.K);
        a.H = ih[l];
        a.W = iw[l];
        a.OH = oh[l];
        a.OW = ow[l];
        a.stride = l < 2 ? 2 : 1;
        a.act = l < 3 ? 1 : 0;
        a.x[0] = in[l][0];
        a.x[1] = in[l][1];
        a.y[0] = out[l][0];
        a.y[1] = out[l][1];
        a.wB = n.tw[l];
        a.bias = n.fb[l];
        const int rc = launch_conv_tc(a, st);
        if (rc) return rc;
    }
    // cost volume + CostFilter c1, then c2 (leaky ReLU after both)
    TcConv v{};
    v.mode = 1;
    v.nd = 3;
    v.nimg = 1;
    v.IC = C;
    v.OC = Cm;
    v.K = C * 27;
    v.Kpad = tc_kpad(v.K);
    v.D = v.OD = n.D;
    v.H = v.OH = h;
    v.W = v.OW = w;
    v.stride = v.pad = v.dil = 1;
    v.act = 1;
    v.x[0] = b.fb[0];
    v.x[1] = b.fb[1];
    v.y[0] = v.y[1] = b.v0;
    v.wB = n.tw[4];
    v.bias = n.cb[0];
    v.err = b.flag;
    int rc = launch_conv_tc(v, st);
    if (rc) return rc;
    v.mode = 0;
    v.IC = Cm;
    v.K = Cm * 27;
    v.Kpad = tc_kpad(v.K);
    v.x[0] = v.x[1] = b.v0;
    v.y[0] = v.y[1] = b.v1;
    v.wB = n.tw[5];
    v.bias = n.cb[1];
    return launch_conv_tc(v, st);
}

// The network shapes this build instantiates: the reference's shipped
// architectures (feat_C, cost_C, refine_C) = (12, 6, 8), (8, 4, 8), (8, 4, 4),
// (16, 8, 8) with D <= 16.
template <int C, int CM, int RC>
static int forward_impl(const NetView &n, const float *left, const float *right, int H, int W,
                        const float *gh, const float *gf, float *d0, float *d1, float *d2,
                        const FwdBufs &b, int precision, cudaStream_t st) {
    const int h1 = (H - 1) / 2 + 1, w1 = (W - 1) / 2 + 1;
    const int h = (h1 - 1) / 2 + 1, w = (w1 - 1) / 2 + 1;
    const int D = n.D;
    dim3 blk(32, 8);
    const dim3 tb(CT2_TW, CT2_TH);
    const int tb1 = CT2_TW * CT2_TH, tb2 = 2 * tb1, tb4 = 4 * tb1;   // k_conv2d_tiled, CS = 1/2/4
    auto tgrid = [&](int OW, int OH, int z) {
        return dim3((OW + CT2_TW - 1) / CT2_TW, (OH + CT2_TH - 1) / CT2_TH, z);
    };
    if (precision == SV_BF16) {
        const int rc = forward_bf16_front(n, left, right, H, W, h1, w1, h, w, b, st);
        if (rc) return rc;
    } else {
        // FeatureNet, both images: c1 s2 (4 output channels per thread), c2 s2,
        // c3, c4 (2 per thread: shorter chains, more CTAs -- measured faster at
        // these sizes; the arithmetic per output is the same)
        constexpr int FG = C % 4 == 0 ? 4 : C, FG2 = C % 2 == 0 ? 2 : C;
        const dim3 fg1 = tgrid(w1, h1, 2 * (C / FG)), fg = tgrid(w, h, 2 * (C / FG2));
        count_launch();
        k_conv2d_tiled<1, C, FG, 1, 1><<<fg1, tb1, conv2d_tile_bytes(1, 2, 1), st>>>(
            left, right, H, W, h1, w1, 2, 1, 1, n.fw[0], n.fb[0], b.fa[0], b.fa[1], nullptr);
        count_launch();
        k_conv2d_tiled<C, C, FG2, 1, 2><<<fg, tb2, conv2d_tile_bytes(C, 2, 1, 2), st>>>(
            b.fa[0], b.fa[1], h1, w1, h, w, 2, 1, 1, n.fw[1], n.fb[1], b.fb[0], b.fb[1],
            nullptr);
        count_launch();
        k_conv2d_tiled<C, C, FG2, 1, 2><<<fg, tb2, conv2d_tile_bytes(C, 1, 1, 2), st>>>(
            b.fb[0], b.fb[1], h, w, h, w, 1, 1, 1, n.fw[2], n.fb[2], b.fa[0], b.fa[1],
            nullptr);
        count_launch();
        k_conv2d_tiled<C, C, FG2, 0, 2><<<fg, tb2, conv2d_tile_bytes(C, 1, 1, 2), st>>>(
            b.fa[0], b.fa[1], h, w, h, w, 1, 1, 1, n.fw[3], n.fb[3], b.fb[0], b.fb[1],
            nullptr);
        SV_LAUNCH_CHECK();
        // cost volume + CostFilter c1, c2 (every output channel in each CTA,
        // so the tile is staged once)
        constexpr int CG = CM;
        constexpr int S1 = C % 4 == 0 ? 4 : 2, S2 = CM % 4 == 0 && CM > 4 ? 4 : 2;
        const dim3 vg1((w + C3_TX - 1) / C3_TX, h * ((D + 16 / S1 - 1) / (16 / S1)), CM / CG);
        const dim3 vg2((w + C3_TX - 1) / C3_TX, h * ((D + 16 / S2 - 1) / (16 / S2)), CM / CG);
        count_launch();
        k_conv3d_split<C, CG, S1, true><<<vg1, 128, 0, st>>>(b.fb[0], b.fb[1], D, h, w, n.cw[0],
                                                             n.cb[0], b.v0);
        count_launch();
        k_conv3d_split<CM, CG, S2, false><<<vg2, 128, 0, st>>>(b.v0, nullptr, D, h, w, n.cw[1],
                                                               n.cb[1], b.v1);
    }
    constexpr int S3 = CM % 2 == 0 ? 2 : 1;
    count_launch();
    k_conv3d_softargmin<CM, S3><<<dim3((w + C3_TX - 1) / C3_TX, h), 128 * S3, 0, st>>>(
        b.v1, D, h, w, n.cw[2], n.cb[2], d0, b.qspread, b.qspread ? b.qpmax : nullptr);
    SV_LAUNCH_CHECK();
    // Refinement levels
    const int Hs[2] = {H / 2, H}, Ws[2] = {W / 2, W};
    const float *guides[2] = {gh, gf};
    float *outs[2] = {d1, d2};
    const float *prev = d0;
    int ph = h, pw = w;
    for (int lv = 0; lv < 2; ++lv) {
        const int Hl = Hs[lv], Wl = Ws[lv];
        const float *cur = nullptr;
        float *bufs[2] = {b.ra, b.rb};
        constexpr int RG = RC % 4 == 0 ? 4 : RC;
        constexpr int RS = RC % 4 == 0 ? 4 : 2;     // lanes per output of the dilated convs
        for (int i = 0; i < n.ndil; ++i) {
            float *dst = bufs[i & 1];
            const int dl = n.dil[i];
            count_launch();
            if (i == 0)     // up-sample + concat built into the first convolution
                k_conv2d_up<RC, RG><<<tgrid(Wl, Hl, RC / RG), tb, conv2d_tile_bytes(2, 1, dl),
                                      st>>>(prev, ph, pw, guides[lv], Hl, Wl, dl, n.rw[lv][i],
                                            n.rb[lv][i], dst, b.rin);
            else            // every output channel per thread (measured faster)
                k_conv2d_tiled<RC, RC, RC, 1, RS><<<tgrid(Wl, Hl, 1), RS * tb1,
                                                    conv2d_tile_bytes(RC, 1, dl, RS), st>>>(
                    cur, cur, Hl, Wl, Hl, Wl, 1, dl, dl, n.rw[lv][i], n.rb[lv][i], dst, dst,
                    nullptr);
            cur = dst;
        }
        count_launch();
        if (lv == 1 && b.decide && b.decide->width)
            k_conv2d_out_decide<RC><<<tgrid(Wl, Hl, 1), tb4, conv2d_tile_bytes(RC, 1, 1, 4),
                                      st>>>(cur, Hl, Wl, n.rw[lv][n.ndil], n.rb[lv][n.ndil],
                                            outs[lv], b.rin, *b.decide->width,
                                            b.decide->state, b.decide->hist,
                                            b.decide->mirror);
        else
            k_conv2d_tiled<RC, 1, 1, 2, 4><<<tgrid(Wl, Hl, 1), tb4,
                                             conv2d_tile_bytes(RC, 1, 1, 4), st>>>(
                cur, cur, Hl, Wl, Hl, Wl, 1, 1, 1, n.rw[lv][n.ndil], n.rb[lv][n.ndil], outs[lv],
                outs[lv], b.rin);
        SV_LAUNCH_CHECK();
        prev = outs[lv];
        ph = Hl;
        pw = Wl;
    }
    return SV_OK;
}

int launch_forward(const NetView &n, const float *left, const float *right, int H, int W,
                   const float *gh, const float *gf, float *d0, float *d1, float *d2,
                   const FwdBufs &b, int precision, cudaStream_t st) {
    if (precision != SV_FP32 && precision != SV_BF16) {
        set_error("precision %d is neither SV_FP32 nor SV_BF16", precision);
        return SV_ERR_PARAM;
    }
    if (precision == SV_BF16 && (!n.tw[0] || !b.flag)) {
        set_error("BF16 forward without packed weights or an error flag");
        return SV_ERR_PARAM;
    }
    if (n.D < 1 || n.D > 16) {
        set_error("D=%d outside 1..16", n.D);
        return SV_ERR_NET;
    }
    if (n.C == 12 && n.Cm == 6 && n.Rc == 8)
        return forward_impl<12, 6, 8>(n, left, right, H, W, gh, gf, d0, d1, d2, b, precision,
                                         st);
    if (n.C == 8 && n.Cm == 4 && n.Rc == 8)
        return forward_impl<8, 4, 8>(n, left, right, H, W, gh, gf, d0, d1, d2, b, precision,
                                         st);
    if (n.C == 8 && n.Cm == 4 && n.Rc == 4)
        return forward_impl<8, 4, 4>(n, left, right, H, W, gh, gf, d0, d1, d2, b, precision,
                                         st);
    if (n.C == 16 && n.Cm == 8 && n.Rc == 8)
        return forward_impl<16, 8, 8>(n, left, right, H, W, gh, gf, d0, d1, d2, b, precision,
                                         st);
    set_error("architecture feat_C=%d cost_C=%d refine_C=%d is not instantiated", n.C, n.Cm,
              n.Rc);
    return SV_ERR_NET;
}



// ====================================================================
// Batched predict_auto passes (driven by sv_netbatch.cu)
// ====================================================================

// CTAs of each batched network kernel for one pair whose work size is at
// most Hm x Wm (the same tile shapes and channel groups as forward_impl).
template <int C, int CM, int RC>
static void stage_ctas_impl(const NetView &n, int Hm, int Wm, long long *o) {
    int h1, w1, h, w;
    net_quarter(Hm, Wm, h1, w1, h, w);
    constexpr int FG = C % 4 == 0 ? 4 : C;
    constexpr int S1 = C % 4 == 0 ? 4 : 2, S2 = CM % 4 == 0 && CM > 4 ? 4 : 2;
    constexpr int RG = RC % 4 == 0 ? 4 : RC;
    // one table serves k_b_conv2d_tiled and k_b_conv2d_wide launches alike
    static_assert(CTB_TW == CT2_TW && CTB_TH == CT2_TH, "the two 2-D tile shapes must agree");
    auto t2 = [](int OW, int OH) {
        return (long long)((OW + CT2_TW - 1) / CT2_TW) * ((OH + CT2_TH - 1) / CT2_TH);
    };
    const int D = n.D, cx = (w + C3_TX - 1) / C3_TX;
    o[NK_RESIZE] = 2LL * ((Wm + 31) / 32) * ((Hm + 7) / 8);
    o[NK_C1] = 2LL * (C / FG) * t2(w1, h1);
    o[NK_C2] = 2LL * (C / FG) * t2(w, h);
    using G1 = C3W<C, S1>;
    using G2 = C3W<CM, S2>;
    o[NK_V1] = (long long)((w + G1::TX - 1) / G1::TX) * h * ((D + G1::TD - 1) / G1::TD);
    o[NK_V2] = (long long)((w + G2::TX - 1) / G2::TX) * h * ((D + G2::TD - 1) / G2::TD);
    o[NK_SA] = (long long)cx * h;
    o[NK_R0] = (long long)(RC / RG) * t2(Wm / 2, Hm / 2);
    o[NK_R0F] = t2(Wm / 2, Hm / 2);
    o[NK_R1] = (long long)(RC / RG) * t2(Wm, Hm);
    o[NK_R1F] = t2(Wm, Hm);
    o[NK_C1W] = 2LL * t2(w1, h1);            // k_b_conv2d_wide: both images, all channels
    o[NK_C2W] = 2LL * t2(w, h);
}

int net_stage_ctas(const NetView &n, int Hm, int Wm, long long *o) {
    if (n.C == 12 && n.Cm == 6 && n.Rc == 8) stage_ctas_impl<12, 6, 8>(n, Hm, Wm, o);
    else if (n.C == 8 && n.Cm == 4 && n.Rc == 8) stage_ctas_impl<8, 4, 8>(n, Hm, Wm, o);
    else if (n.C == 8 && n.Cm == 4 && n.Rc == 4) stage_ctas_impl<8, 4, 4>(n, Hm, Wm, o);
    else if (n.C == 16 && n.Cm == 8 && n.Rc == 8) stage_ctas_impl<16, 8, 8>(n, Hm, Wm, o);
    else {
        set_error("architecture feat_C=%d cost_C=%d refine_C=%d is not instantiated", n.C, n.Cm,
                  n.Rc);
        return SV_ERR_NET;
    }
    return SV_OK;
}

static unsigned ctas_of(long long total) { return (unsigned)(total > 0 ? total : 1); }

// The FP32 forward of one stage over every active pair: forward_impl's
// kernels in their batched form, one launch each for the whole batch.
template <int C, int CM, int RC>
static int b_forward_impl(const NetView &n, const NetStageLaunch &g, const NetSlab &s,
                          cudaStream_t st) {
    const int D = n.D;
    auto L = [&](int k) { return NetLaunch{g.pre[k], g.pairs, g.n, g.slab}; };
    auto B = [&](int k) { return ctas_of(g.total[k]); };
    const int tb1 = CT2_TW * CT2_TH;
    const dim3 tb(CT2_TW, CT2_TH);
    // FeatureNet, both images: every output channel and 2 pixels per thread
    // (the arithmetic of k_conv2d_tiled<.., FG, .., 1 or 2>)
    count_launch();
    b_conv2d_wide<1, C, 1, 1, 2, 2>(L(NK_C1W), B(NK_C1W), 0, 2, s.lw, s.rw, 1, n.fw[0], n.fb[0],
                                    s.f.fa[0], s.f.fa[1], nullptr, st);
    count_launch();
    b_conv2d_wide<C, C, 1, 2, 2, 2>(L(NK_C2W), B(NK_C2W), 1, 2, s.f.fa[0], s.f.fa[1], 1,
                                    n.fw[1], n.fb[1], s.f.fb[0], s.f.fb[1], nullptr, st);
    count_launch();
    b_conv2d_wide<C, C, 1, 2, 2, 1>(L(NK_C2W), B(NK_C2W), 2, 2, s.f.fb[0], s.f.fb[1], 1,
                                    n.fw[2], n.fb[2], s.f.fa[0], s.f.fa[1], nullptr, st);
    count_launch();
    b_conv2d_wide<C, C, 0, 2, 2, 1>(L(NK_C2W), B(NK_C2W), 2, 2, s.f.fa[0], s.f.fa[1], 1,
                                    n.fw[3], n.fb[3], s.f.fb[0], s.f.fb[1], nullptr, st);
    SV_LAUNCH_CHECK();
    constexpr int S1 = C % 4 == 0 ? 4 : 2, S2 = CM % 4 == 0 && CM > 4 ? 4 : 2;
    count_launch();
    k_b_conv3d_wide<C, CM, S1, true><<<B(NK_V1), 128, 0, st>>>(
        L(NK_V1), s.f.fb[0], s.f.fb[1], D, n.cw[0], n.cb[0], s.f.v0);
    count_launch();
    k_b_conv3d_wide<CM, CM, S2, false><<<B(NK_V2), 128, 0, st>>>(
        L(NK_V2), s.f.v0, nullptr, D, n.cw[1], n.cb[1], s.f.v1);
    constexpr int S3 = CM % 2 == 0 ? 2 : 1;
    count_launch();
    k_b_conv3d_softargmin<CM, S3><<<B(NK_SA), 128 * S3, 0, st>>>(L(NK_SA), s.f.v1, D, n.cw[2],
                                                                  n.cb[2], s.d0);
    SV_LAUNCH_CHECK();
    constexpr int RG = RC % 4 == 0 ? 4 : RC;
    constexpr int RS = RC % 4 == 0 ? 4 : 2;
    const float *guides[2] = {s.gh, s.lw};
    const float *prevs[2] = {s.d0, s.d1};
    float *outs[2] = {s.d1, s.d2};
    const bool tiled = RC > 8;     // the register-blocked form holds at most 8 channels
    for (int lv = 0; lv < 2; ++lv) {
        const int kk = lv ? NK_R1 : NK_R0, kf = lv ? NK_R1F : NK_R0F;
        float *bufs[2] = {s.f.ra, s.f.rb};
        const float *cur = nullptr;
        for (int i = 0; i < n.ndil; ++i) {
            float *dst = bufs[i & 1];
            const int dl = n.dil[i];
            count_launch();
            if (i == 0)
                k_b_conv2d_up<RC, RG><<<B(kk), tb, conv2d_tile_bytes(2, 1, dl), st>>>(
                    L(kk), lv, prevs[lv], guides[lv], dl, n.rw[lv][i], n.rb[lv][i], dst, s.f.rin);
            else if (!tiled)
                b_conv2d_wide<RC, RC, 1, RS, 2, 1>(L(kf), B(kf), lv + 3, 1, cur, cur, dl,
                                                   n.rw[lv][i], n.rb[lv][i], dst, dst, nullptr,
                                                   st);
            else
                k_b_conv2d_tiled<RC, RC, RG, 1, RS><<<B(kk), RS * tb1,
                                                      conv2d_tile_bytes(RC, 1, dl, RS), st>>>(
                    L(kk), 3 + lv, RC / RG, cur, cur, 1, dl, dl, n.rw[lv][i], n.rb[lv][i], dst,
                    dst, nullptr);
            cur = dst;
        }
        count_launch();
        if (!tiled)
            b_conv2d_wide<RC, 1, 2, 4, 2, 1>(L(kf), B(kf), lv + 3, 1, cur, cur, 1,
                                             n.rw[lv][n.ndil], n.rb[lv][n.ndil], outs[lv],
                                             outs[lv], s.f.rin, st);
        else
            k_b_conv2d_tiled<RC, 1, 1, 2, 4><<<B(kf), 4 * tb1, conv2d_tile_bytes(RC, 1, 1, 4),
                                               st>>>(L(kf), 3 + lv, 1, cur, cur, 1, 1, 1,
                                                     n.rw[lv][n.ndil], n.rb[lv][n.ndil],
                                                     outs[lv], outs[lv], s.f.rin);
        SV_LAUNCH_CHECK();
    }
    return SV_OK;
}

int launch_b_forward(const NetView &n, const NetStageLaunch &g, const NetSlab &s,
                     cudaStream_t st) {
    if (n.D < 1 || n.D > 16) {
        set_error("D=%d outside 1..16", n.D);
        return SV_ERR_NET;
    }
    if (n.C == 12 && n.Cm == 6 && n.Rc == 8) return b_forward_impl<12, 6, 8>(n, g, s, st);
    if (n.C == 8 && n.Cm == 4 && n.Rc == 8) return b_forward_impl<8, 4, 8>(n, g, s, st);
    if (n.C == 8 && n.Cm == 4 && n.Rc == 4) return b_forward_impl<8, 4, 4>(n, g, s, st);
    if (n.C == 16 && n.Cm == 8 && n.Rc == 8) return b_forward_impl<16, 8, 8>(n, g, s, st);
    set_error("architecture feat_C=%d cost_C=%d refine_C=%d is not instantiated", n.C, n.Cm,
              n.Rc);
    return SV_ERR_NET;
}

int launch_b_resize(const NetStageLaunch &g, const void *const *lt, const void *const *rt,
                    int dtype, const NetSlab &s, bool with_sel, cudaStream_t st) {
    const NetLaunch L{g.pre[NK_RESIZE], g.pairs, g.n, g.slab};
    const unsigned B = ctas_of(g.total[NK_RESIZE]);
    const dim3 blk(32, 8);
    SelState *sel = with_sel ? s.sel : nullptr;
    count_launch();
    switch (dtype) {
    case SV_U8: k_b_resize_pair<uint8_t><<<B, blk, 0, st>>>(L, lt, rt, s.lw, s.rw, s.gh, sel, s.hist); break;
    case SV_F32: k_b_resize_pair<float><<<B, blk, 0, st>>>(L, lt, rt, s.lw, s.rw, s.gh, sel, s.hist); break;
    case SV_F64: k_b_resize_pair<double><<<B, blk, 0, st>>>(L, lt, rt, s.lw, s.rw, s.gh, sel, s.hist); break;
    default: set_error("unknown dtype %d", dtype); return SV_ERR_PARAM;
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_b_work_outputs(const NetLaunch &L, long long total, const NetSlab &s, bool with_sel,
                          double target, int rule_width, cudaStream_t st) {
    count_launch();
    k_b_work_outputs<<<ctas_of(total), dim3(32, 8), 0, st>>>(
        L, s.d2, nullptr, s.full, with_sel ? s.sel : nullptr, with_sel ? s.hist : nullptr,
        target, rule_width);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

}  // namespace sv
