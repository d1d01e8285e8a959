// sv_band.cu -- the learned adaptive band: features, the 4-layer band net's
// BF16 tensor-core forward / backward (sv_tc.cu), its loss, Adam, and the
// application of its output to the refinement band.
//
// Band net: 3x3 convolutions 6 -> 16 -> 16 -> 16 -> 2, dilations 1, 2, 4, 1,
// same padding, leaky ReLU 0.2 after the first three (the reference's Conv2d
// and LeakyReLU, stereonet.py:459-723).  Output channel 0 is the band-centre
// shift s = 32 o0 (px), channel 1 the log-scale rho = o1 + 1 of a Laplace
// distribution of the true shift; training minimises its negative
// log-likelihood against full-range SGM disparities.  Adam follows
// stereonet.py:1354-1387 (running-product bias correction, gradient clip).

#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "sv_common.cuh"
#include "sv_refine.cuh"
#include "sv_tc.cuh"

namespace sv {

// input planes: the six search / image features of k_band_features and the
// network's confidence (k_band_conf)
constexpr int kBandF = 8, kBandC = 16, kBandO = 2, kBandL = 4;
constexpr int kBandIC[kBandL] = {kBandF, kBandC, kBandC, kBandC};
constexpr int kBandOC[kBandL] = {kBandC, kBandC, kBandC, kBandO};
constexpr int kBandDil[kBandL] = {1, 2, 4, 1};
constexpr float kShiftScale = 32.f, kRho0 = 1.f;
constexpr float kRhoMin = -1.3862943611198906f, kRhoMax = 4.852030263919617f;
constexpr double kRhoMinD = -1.3862943611198906, kRhoMaxD = 4.852030263919617;
constexpr int kFeatRows = 4;          // output rows per feature thread
constexpr int kAggHalf = 4;           // vertical aggregation: 9 rows
constexpr int kBandInvalid = 66;

static long band_param_count() {
    long n = 0;
    for (int l = 0; l < kBandL; ++l) n += (long)kBandOC[l] * kBandIC[l] * 9 + kBandOC[l];
    return n;
}

static void band_offsets(long *ow, long *ob) {
    long o = 0;
    for (int l = 0; l < kBandL; ++l) {
        ow[l] = o;
        o += (long)kBandOC[l] * kBandIC[l] * 9;
        ob[l] = o;
        o += kBandOC[l];
    }
}

// ------------------------------------------------------------- features
template <typename T>
__device__ __forceinline__ double gray_of(const T *img, long p);
template <>
__device__ __forceinline__ double gray_of<uint8_t>(const uint8_t *img, long p) {
    return __ddiv_rn((double)img[p], 255.0);
}
template <>
__device__ __forceinline__ double gray_of<float>(const float *img, long p) {
    return (double)img[p];
}
template <>
__device__ __forceinline__ double gray_of<double>(const double *img, long p) {
    return img[p];
}

// Thread (column, 8 output rows, disparity group): the disparity range is
// split over kFeatDG groups.  For each of its d the thread forms the 16 row
// costs of its window once and slides the 9-row sum down its 8 rows, keeping
// per row the first minimum (as a packed key agg << 8 | d, so the smallest d
// wins ties), the minimum inside the +-10 band around d0 and the cost at
// round(d0); the groups combine with shared-memory atomicMin.  The right
// view's census words the block reads (its 16 rows, columns x0 - dmax ..
// x0 + 31) are staged in shared memory first.
constexpr int kFeatDG = 4, kFeatSeg = 2;
constexpr int kFeatBR = kFeatSeg * kFeatRows + 2 * kAggHalf;   // staged rows

static size_t band_features_smem(int dmax) { return (size_t)kFeatBR * (32 + dmax) * 8; }

template <typename T>
__global__ void __launch_bounds__(32 * kFeatSeg * kFeatDG)
    k_band_features(const uint64_t *__restrict__ cl, const uint64_t *__restrict__ cr,
                    const double *__restrict__ d0, const T *__restrict__ left, int W, int H,
                    int dmax, float *__restrict__ feat, int *__restrict__ err) {
    __shared__ unsigned s_best[kFeatSeg][kFeatRows][32];
    __shared__ int s_band[kFeatSeg][kFeatRows][32];
    __shared__ int s_cd0[kFeatSeg][kFeatRows][32];
    extern __shared__ uint64_t s_cr[];                 // [kFeatBR][32 + dmax]
    const int tx = threadIdx.x, ty = threadIdx.y, g = threadIdx.z;
    const int x = blockIdx.x * 32 + tx;
    const int y0 = (blockIdx.y * kFeatSeg + ty) * kFeatRows;
    const bool active = x < W && y0 < H;
    const int CW = 32 + dmax;
    {
        const int yb = blockIdx.y * kFeatSeg * kFeatRows - kAggHalf;
        const int xb = blockIdx.x * 32 - dmax;
        const int tid = (g * kFeatSeg + ty) * 32 + tx;
        for (int i = tid; i < kFeatBR * CW; i += 32 * kFeatSeg * kFeatDG) {
            const int r = i / CW, c = i - (i / CW) * CW;
            int yy = yb + r;
            yy = yy < 0 ? 0 : (yy >= H ? H - 1 : yy);
            const int gx = xb + c;
            s_cr[i] = gx >= 0 && gx < W ? __ldg(cr + (long)yy * W + gx) : 0ull;
        }
    }
    if (g == 0) {
#pragma unroll
        for (int j = 0; j < kFeatRows; ++j) {
            s_best[ty][j][tx] = 0xffffffffu;
            s_band[ty][j][tx] = 1 << 30;
            s_cd0[ty][j][tx] = 0;
        }
    }
    __syncthreads();
    if (active) {
        constexpr int NR = kFeatRows + 2 * kAggHalf;
        uint64_t clv[NR];
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            int yy = y0 - kAggHalf + i;
            yy = yy < 0 ? 0 : (yy >= H ? H - 1 : yy);
            clv[i] = __ldg(cl + (long)yy * W + x);
        }
        const uint64_t *crow = s_cr + ty * kFeatRows * CW + tx + dmax;   // column x - d at -d
        int r0[kFeatRows];
        unsigned best[kFeatRows];
        int band[kFeatRows], cd0[kFeatRows];
#pragma unroll
        for (int j = 0; j < kFeatRows; ++j) {
            const int y = y0 + j < H ? y0 + j : H - 1;
            const double t = __dadd_rn(d0[(long)y * W + x], 0.5);
            int r = 0;
            if (!(t > -9.0e15 && t < 9.0e15)) {
                if (g == 0) flag_error(err, SV_ERR_DISP);
            } else if (t >= (double)dmax) {
                r = dmax;
            } else if (t >= 1.0) {
                r = __double2int_rz(t);
            }
            r0[j] = r;
            best[j] = 0xffffffffu;
            band[j] = 1 << 30;
            cd0[j] = -1;
        }
        const int chunk = (dmax + kFeatDG) / kFeatDG;
        const int dlo = g * chunk, dhi = min(dmax, dlo + chunk - 1);
        for (int d = dlo; d <= dhi; ++d) {
            int c[NR];
            const bool in = x - d >= 0;
#pragma unroll
            for (int i = 0; i < NR; ++i)
                c[i] = in ? __popcll(clv[i] ^ crow[i * CW - d]) : kBandInvalid;
            int s = 0;
#pragma unroll
            for (int i = 0; i < 2 * kAggHalf + 1; ++i) s += c[i];
#pragma unroll
            for (int j = 0; j < kFeatRows; ++j) {
                if (j > 0) s += c[j + 2 * kAggHalf] - c[j - 1];
                best[j] = min(best[j], ((unsigned)s << 8) | (unsigned)d);
                if (abs(d - r0[j]) <= 10) band[j] = min(band[j], s);
                if (d == r0[j]) cd0[j] = s;
            }
        }
#pragma unroll
        for (int j = 0; j < kFeatRows; ++j) {
            atomicMin(&s_best[ty][j][tx], best[j]);
            atomicMin(&s_band[ty][j][tx], band[j]);
            if (cd0[j] >= 0) s_cd0[ty][j][tx] = cd0[j];     // one group owns d == r0
        }
    }
    __syncthreads();
    if (!active || g != 0) return;
    const long N = (long)W * H;
#pragma unroll
    for (int j = 0; j < kFeatRows; ++j) {
        const int y = y0 + j;
        if (y >= H) break;
        const long p = (long)y * W + x;
        const double dd = d0[p];
        const unsigned bk = s_best[ty][j][tx];
        const int dw = (int)(bk & 0xffu), aw = (int)(bk >> 8);
        feat[p] = (float)__ddiv_rn(dd, 64.0);
        feat[N + p] = (float)__ddiv_rn(__dsub_rn((double)dw, dd), 64.0);
        feat[2 * N + p] = (float)__ddiv_rn((double)aw, 558.0);
        feat[3 * N + p] = (float)__ddiv_rn((double)s_cd0[ty][j][tx], 558.0);
        feat[4 * N + p] = (float)__ddiv_rn((double)s_band[ty][j][tx], 558.0);
        feat[5 * N + p] = (float)__dsub_rn(gray_of<T>(left, p), 0.5);
    }
}

// ----------------------------------------------------------------- loss
// loss = sum over labelled pixels of (|t - 32 o0| / b + rho) / n,
// rho = clamp(o1 + 1), b = exp(rho), n = every pixel of the batch.
__global__ void __launch_bounds__(256)
    k_band_loss(const float *__restrict__ O, const float *__restrict__ target,
                const uint8_t *__restrict__ mask, long HW, long total, float inv_n,
                float *__restrict__ gO, double *__restrict__ loss) {
    double acc = 0.0;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total;
         q += (long)gridDim.x * blockDim.x) {
        const long i = q / HW, p = q - i * HW;
        const long o = i * kBandO * HW + p;
        float g0 = 0.f, g1 = 0.f;
        if (mask[q]) {
            const float s = kShiftScale * O[o];
            float rho = O[o + HW] + kRho0;
            const bool inside = rho > kRhoMin && rho < kRhoMax;
            rho = fminf(fmaxf(rho, kRhoMin), kRhoMax);
            const float b = expf(rho);
            const float e = target[q] - s;
            const float ae = fabsf(e);
            acc += (double)((ae / b + rho) * inv_n);
            const float sg = e > 0.f ? 1.f : (e < 0.f ? -1.f : 0.f);
            g0 = -sg / b * kShiftScale * inv_n;
            g1 = inside ? (1.f - ae / b) * inv_n : 0.f;
        }
        gO[o] = g0;
        gO[o + HW] = g1;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(kFull, acc, off);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, acc);
}

// ----------------------------------------------------------------- Adam
__global__ void k_band_adam(float *__restrict__ p, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, long n, float lr,
                            float b1, float b2, float eps, float clip, float c1, float c2) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = fminf(fmaxf(g[i], -clip), clip);
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// --------------------------------------------------- targets and apply
__global__ void k_band_targets(const double *__restrict__ label, const uint8_t *__restrict__ st,
                               const double *__restrict__ d0, long n, double shift_max,
                               float *__restrict__ target, uint8_t *__restrict__ mask) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t = __dsub_rn(label[i], d0[i]);
    t = t > shift_max ? shift_max : (t < -shift_max ? -shift_max : t);
    target[i] = (float)t;
    mask[i] = st[i] == 0;
}

__global__ void k_band_apply(const float *__restrict__ out, const double *__restrict__ d0,
                             long HW, double b_thr, double rad_k, int rad_min, int R,
                             double shift_max, double *__restrict__ centre,
                             uint8_t *__restrict__ rad) {
    const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (p >= HW) return;
    double rho = __dadd_rn((double)out[HW + p], 1.0);
    rho = rho < kRhoMinD ? kRhoMinD : (rho > kRhoMaxD ? kRhoMaxD : rho);
    const double b = exp(rho);
    if (b <= b_thr) {
        double s = __dmul_rn(32.0, (double)out[p]);
        s = s > shift_max ? shift_max : (s < -shift_max ? -shift_max : s);
        centre[p] = __dadd_rn(d0[p], s);
        double r = ceil(__dmul_rn(rad_k, b));
        r = r < rad_min ? rad_min : (r > R ? R : r);
        rad[p] = (uint8_t)r;
    } else {
        centre[p] = d0[p];
        rad[p] = (uint8_t)R;
    }
}

}  // namespace sv

using namespace sv;

struct sv_band {
    float *p = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    uint16_t *packs = nullptr;
    uint16_t *fwd[kBandL] = {}, *bwd[kBandL] = {};
    long n = 0;
    long ow[kBandL], ob[kBandL];
    double b1t = 1.0, b2t = 1.0;
};

namespace {

struct BandWs {
    DevFlags *flags;
    float *X[kBandL];          // X[0] unused (the features), X[l] = input of layer l
    float *O, *gO, *gA, *gB;
    double *loss;
};

size_t carve_band(void *ws, int nb, long HW, BandWs *o) {
    Carver cv(ws);
    BandWs w{};
    w.flags = cv.take<DevFlags>(1);
    for (int l = 1; l < kBandL; ++l) w.X[l] = cv.take<float>((size_t)nb * kBandC * HW);
    w.O = cv.take<float>((size_t)nb * kBandO * HW);
    w.gO = cv.take<float>((size_t)nb * kBandO * HW);
    w.gA = cv.take<float>((size_t)nb * kBandC * HW);
    w.gB = cv.take<float>((size_t)nb * kBandC * HW);
    w.loss = cv.take<double>(1);
    if (o) *o = w;
    return cv.off;
}

int band_pack(sv_band *b, cudaStream_t st) {
    for (int l = 0; l < kBandL; ++l) {
        int rc = launch_pack_weights(b->p + b->ow[l], kBandOC[l], kBandIC[l], 0, b->fwd[l], st);
        if (rc) return rc;
        if (l > 0) {
            rc = launch_pack_weights(b->p + b->ow[l], kBandOC[l], kBandIC[l], 1, b->bwd[l], st);
            if (rc) return rc;
        }
    }
    return SV_OK;
}

TcConv band_conv(int l, const float *x, float *y, const uint16_t *wB, const float *bias, int act,
                 int nb, int W, int H, int *err, bool transpose, const float *aux) {
    TcConv a{};
    a.mode = 0;
    a.nd = 2;
    a.nimg = 1;
    a.IC = transpose ? kBandOC[l] : kBandIC[l];
    a.OC = transpose ? kBandIC[l] : kBandOC[l];
    a.K = a.IC * 9;
    a.Kpad = tc_kpad(a.K);
    a.D = a.OD = 1;
    a.H = a.OH = H;
    a.W = a.OW = W;
    a.stride = 1;
    a.pad = a.dil = kBandDil[l];
    a.act = act;
    a.x[0] = a.x[1] = x;
    a.y[0] = a.y[1] = y;
    a.wB = wB;
    a.bias = bias;
    a.err = err;
    a.nb = nb;
    a.xs = (long)a.IC * H * W;
    a.ys = (long)a.OC * H * W;
    a.aux = aux;
    return a;
}

int band_forward_impl(const sv_band *b, const float *feat, int nb, int W, int H, float *out,
                      const BandWs &w, cudaStream_t st) {
    const float *in = feat;
    for (int l = 0; l < kBandL; ++l) {
        float *y = l + 1 < kBandL ? w.X[l + 1] : out;
        const TcConv a = band_conv(l, in, y, b->fwd[l], b->p + b->ob[l], l + 1 < kBandL ? 1 : 0,
                                   nb, W, H, &w.flags->status, false, nullptr);
        const int rc = launch_conv_tc(a, st);
        if (rc) return rc;
        in = y;
    }
    return SV_OK;
}

// Forward, loss and every parameter gradient into b->g.
int band_grads_impl(sv_band *b, const float *feat, const float *target, const uint8_t *mask,
                    int nb, int W, int H, const BandWs &w, cudaStream_t st) {
    const long HW = (long)W * H, total = HW * nb;
    SV_CUDA_TRY(cudaMemsetAsync(b->g, 0, sizeof(float) * b->n, st));
    SV_CUDA_TRY(cudaMemsetAsync(w.loss, 0, sizeof(double), st));
    int rc = band_forward_impl(b, feat, nb, W, H, w.O, w, st);
    if (rc) return rc;
    count_launch();
    k_band_loss<<<grid_for(total, 256, 148 * 8), 256, 0, st>>>(
        w.O, target, mask, HW, total, (float)(1.0 / (double)total), w.gO, w.loss);
    SV_LAUNCH_CHECK();
    // layer l's output gradient (w.r.t. its pre-activation) is gcur
    const float *gcur = w.gO;
    float *bufs[2] = {w.gA, w.gB};
    for (int l = kBandL - 1; l >= 0; --l) {
        TcWgrad g{};
        g.IC = kBandIC[l];
        g.OC = kBandOC[l];
        g.dil = kBandDil[l];
        g.H = H;
        g.W = W;
        g.nb = nb;
        g.xs = (long)kBandIC[l] * HW;
        g.gs = (long)kBandOC[l] * HW;
        g.x = l == 0 ? feat : w.X[l];
        g.g = gcur;
        g.gw = b->g + b->ow[l];
        g.gb = b->g + b->ob[l];
        g.err = &w.flags->status;
        rc = launch_wgrad_tc(g, st);
        if (rc) return rc;
        if (l == 0) break;
        float *dst = bufs[l & 1];
        const TcConv a = band_conv(l, gcur, dst, b->bwd[l], nullptr, 2, nb, W, H,
                                   &w.flags->status, true, w.X[l]);
        rc = launch_conv_tc(a, st);
        if (rc) return rc;
        gcur = dst;
    }
    return SV_OK;
}

int check_band_ws(void *ws, size_t bytes, int nb, int W, int H) {
    const size_t need = carve_band(nullptr, nb, (long)W * H, nullptr);
    if (!ws || ((uintptr_t)ws & 255) || bytes < need) {
        set_error("workspace needs %zu bytes, 256-aligned (have %zu)", need, bytes);
        return SV_ERR_WORKSPACE;
    }
    return SV_OK;
}

}  // namespace

#define SV_TRY(expr)                  \
    do {                              \
        int rc_ = (expr);             \
        if (rc_ != SV_OK) return rc_; \
    } while (0)

namespace sv {

// The rule centre: the network disparity moved to the wide search's first
// argmin (d0 + 64 * feature 1) wherever that argmin's 9-row cost (feature 2)
// is below tau.  The learned band refines around it.
__global__ void k_band_rule(const float *__restrict__ feat, const double *__restrict__ d0,
                            long N, double tau, double *__restrict__ centre) {
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < N;
         p += (long)gridDim.x * blockDim.x) {
        const double f1 = (double)feat[N + p], f2 = (double)feat[2 * N + p];
        centre[p] = f2 < tau ? __dadd_rn(d0[p], __dmul_rn(64.0, f1)) : d0[p];
    }
}

// Feature planes 6 and 7: the network's spread (full-resolution px / 16)
// and its peak probability - 0.5, per pixel of the last pass.
__global__ void k_band_conf(const double *__restrict__ spread, const double *__restrict__ pmax,
                            long N, float *__restrict__ feat) {
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < N;
         p += (long)gridDim.x * blockDim.x) {
        feat[6 * N + p] = (float)__ddiv_rn(spread[p], 16.0);
        feat[7 * N + p] = (float)__dsub_rn(pmax[p], 0.5);
    }
}

}  // namespace sv

extern "C" {

long sv_band_param_count(void) { return band_param_count(); }

int sv_band_create(const double *params, long n_params, sv_band **out) {
    if (!params || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (n_params != band_param_count()) {
        set_error("band net has %ld parameters, got %ld", band_param_count(), n_params);
        return SV_ERR_NET;
    }
    sv_band *b = new sv_band();
    b->n = n_params;
    band_offsets(b->ow, b->ob);
    size_t pack = 0, off_f[kBandL], off_b[kBandL];
    for (int l = 0; l < kBandL; ++l) {
        off_f[l] = pack;
        pack += tc_weight_elems(kBandIC[l] * 9);
        off_b[l] = pack;
        pack += l > 0 ? tc_weight_elems(kBandOC[l] * 9) : 0;
    }
    std::vector<float> f(n_params);
    for (long i = 0; i < n_params; ++i) f[i] = (float)params[i];
    cudaError_t e = cudaMalloc(&b->p, sizeof(float) * 4 * n_params);
    if (e == cudaSuccess) e = cudaMalloc(&b->packs, sizeof(uint16_t) * pack);
    if (e == cudaSuccess) {
        b->m = b->p + n_params;
        b->v = b->m + n_params;
        b->g = b->v + n_params;
        e = cudaMemcpy(b->p, f.data(), sizeof(float) * n_params, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(b->m, 0, sizeof(float) * 3 * n_params);
    if (e != cudaSuccess) {
        set_error("band net upload failed: %s", cudaGetErrorString(e));
        if (b->p) cudaFree(b->p);
        if (b->packs) cudaFree(b->packs);
        delete b;
        return SV_ERR_CUDA;
    }
    for (int l = 0; l < kBandL; ++l) {
        b->fwd[l] = b->packs + off_f[l];
        b->bwd[l] = l > 0 ? b->packs + off_b[l] : nullptr;
    }
    int rc = band_pack(b, nullptr);
    if (rc == SV_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) rc = SV_ERR_CUDA;
    if (rc) {
        cudaFree(b->p);
        cudaFree(b->packs);
        delete b;
        return rc;
    }
    *out = b;
    return SV_OK;
}

void sv_band_destroy(sv_band *b) {
    if (!b) return;
    if (b->p) cudaFree(b->p);
    if (b->packs) cudaFree(b->packs);
    delete b;
}

int sv_band_get_params(const sv_band *b, double *out, long n) {
    if (!b || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (n != b->n) { set_error("expected %ld parameters", b->n); return SV_ERR_PARAM; }
    std::vector<float> f(n);
    SV_CUDA_TRY(cudaDeviceSynchronize());
    SV_CUDA_TRY(cudaMemcpy(f.data(), b->p, sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (long i = 0; i < n; ++i) out[i] = f[i];
    return SV_OK;
}

size_t sv_band_features_workspace_size(int W, int H) {
    if (W < 1 || H < 1) return 0;
    Carver cv(nullptr);
    cv.take<DevFlags>(1);
    cv.take<uint64_t>((size_t)W * H);
    cv.take<uint64_t>((size_t)W * H);
    return cv.off;
}

int sv_band_rule_centre(const float *feat, const double *disp0, int W, int H, double tau,
                        double *centre, void *stream) {
    if (!feat || !disp0 || !centre) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1) { set_error("bad shape %dx%d", W, H); return SV_ERR_SHAPE; }
    if (!std::isfinite(tau)) { set_error("tau must be finite"); return SV_ERR_PARAM; }
    const long N = (long)W * H;
    count_launch();
    k_band_rule<<<grid_for(N, 256), 256, 0, (cudaStream_t)stream>>>(feat, disp0, N, tau, centre);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int sv_band_conf_features(const double *spread, const double *pmax, int W, int H, float *feat,
                          void *stream) {
    if (!spread || !pmax || !feat) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1) { set_error("bad shape %dx%d", W, H); return SV_ERR_SHAPE; }
    const long N = (long)W * H;
    count_launch();
    k_band_conf<<<grid_for(N, 256), 256, 0, (cudaStream_t)stream>>>(spread, pmax, N, feat);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int sv_band_features(const void *left, const void *right, int dtype, const double *disp0,
                     int W, int H, int dmax, float *feat, void *workspace,
                     size_t workspace_bytes, void *stream) {
    if (!left || !right || !disp0 || !feat) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1 || W > kMaxRowW) { set_error("bad shape %dx%d", W, H); return SV_ERR_SHAPE; }
    if (dmax < 0 || dmax > 255) { set_error("dmax %d outside 0..255", dmax); return SV_ERR_PARAM; }
    if (dtype != SV_U8 && dtype != SV_F32 && dtype != SV_F64) {
        set_error("dtype %d", dtype);
        return SV_ERR_PARAM;
    }
    const size_t need = sv_band_features_workspace_size(W, H);
    if (!workspace || ((uintptr_t)workspace & 255) || workspace_bytes < need) {
        set_error("workspace needs %zu bytes, 256-aligned", need);
        return SV_ERR_WORKSPACE;
    }
    Carver cv(workspace);
    DevFlags *flags = cv.take<DevFlags>(1);
    uint64_t *cl = cv.take<uint64_t>((size_t)W * H);
    uint64_t *cr = cv.take<uint64_t>((size_t)W * H);
    cudaStream_t st = (cudaStream_t)stream;
    SV_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(DevFlags), st));
    SV_TRY(launch_census(left, right, dtype, W, H, 4, 3, cl, cr, st));
    const dim3 blk(32, kFeatSeg, kFeatDG);
    const dim3 grd((W + 31) / 32, ((H + kFeatRows - 1) / kFeatRows + kFeatSeg - 1) / kFeatSeg);
    count_launch();
    if (dtype == SV_U8)
        k_band_features<uint8_t><<<grd, blk, band_features_smem(dmax), st>>>(cl, cr, disp0, (const uint8_t *)left, W, H,
                                                      dmax, feat, &flags->status);
    else if (dtype == SV_F32)
        k_band_features<float><<<grd, blk, band_features_smem(dmax), st>>>(cl, cr, disp0, (const float *)left, W, H,
                                                    dmax, feat, &flags->status);
    else
        k_band_features<double><<<grd, blk, band_features_smem(dmax), st>>>(cl, cr, disp0, (const double *)left, W, H,
                                                      dmax, feat, &flags->status);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

size_t sv_band_workspace_size(int nb, int W, int H) {
    if (nb < 1 || W < 1 || H < 1) return 0;
    return carve_band(nullptr, nb, (long)W * H, nullptr);
}

int sv_band_forward(const sv_band *b, const float *feat, int nb, int W, int H, float *out,
                    void *workspace, size_t workspace_bytes, void *stream) {
    if (!b || !feat || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (nb < 1 || W < 1 || H < 1) { set_error("bad shape"); return SV_ERR_SHAPE; }
    SV_TRY(check_band_ws(workspace, workspace_bytes, nb, W, H));
    BandWs w;
    carve_band(workspace, nb, (long)W * H, &w);
    cudaStream_t st = (cudaStream_t)stream;
    SV_CUDA_TRY(cudaMemsetAsync(w.flags, 0, sizeof(DevFlags), st));
    return band_forward_impl(b, feat, nb, W, H, out, w, st);
}

int sv_band_grads(sv_band *b, const float *feat, const float *target, const uint8_t *mask,
                  int nb, int W, int H, float *grads, double *loss, void *workspace,
                  size_t workspace_bytes, void *stream) {
    if (!b || !feat || !target || !mask) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (nb < 1 || W < 1 || H < 1) { set_error("bad shape"); return SV_ERR_SHAPE; }
    SV_TRY(check_band_ws(workspace, workspace_bytes, nb, W, H));
    BandWs w;
    carve_band(workspace, nb, (long)W * H, &w);
    cudaStream_t st = (cudaStream_t)stream;
    SV_CUDA_TRY(cudaMemsetAsync(w.flags, 0, sizeof(DevFlags), st));
    SV_TRY(band_grads_impl(b, feat, target, mask, nb, W, H, w, st));
    if (grads)
        SV_CUDA_TRY(cudaMemcpyAsync(grads, b->g, sizeof(float) * b->n, cudaMemcpyDeviceToDevice,
                                    st));
    if (loss)
        SV_CUDA_TRY(cudaMemcpyAsync(loss, w.loss, sizeof(double), cudaMemcpyDeviceToDevice, st));
    return SV_OK;
}

int sv_band_train_step(sv_band *b, const float *feat, const float *target, const uint8_t *mask,
                       int nb, int W, int H, double lr, double *loss, void *workspace,
                       size_t workspace_bytes, void *stream) {
    if (!(lr > 0.0) || !std::isfinite(lr)) { set_error("lr must be positive"); return SV_ERR_PARAM; }
    SV_TRY(sv_band_grads(b, feat, target, mask, nb, W, H, nullptr, loss, workspace,
                         workspace_bytes, stream));
    cudaStream_t st = (cudaStream_t)stream;
    const double b1 = 0.9, b2 = 0.999;
    b->b1t *= b1;
    b->b2t *= b2;
    const double c1 = 1.0 / (1.0 - b->b1t), c2 = 1.0 / (1.0 - b->b2t);
    count_launch();
    k_band_adam<<<(unsigned)((b->n + 255) / 256), 256, 0, st>>>(
        b->p, b->g, b->m, b->v, b->n, (float)lr, (float)b1, (float)b2, 1.0e-8f, 5.0f, (float)c1,
        (float)c2);
    SV_LAUNCH_CHECK();
    return band_pack(b, st);
}

int sv_band_targets(const double *label, const uint8_t *status, const double *disp0, long n,
                    double shift_max, float *target, uint8_t *mask, void *stream) {
    if (!label || !status || !disp0 || !target || !mask) {
        set_error("NULL argument");
        return SV_ERR_NULL;
    }
    if (n < 1) { set_error("bad size"); return SV_ERR_SHAPE; }
    count_launch();
    k_band_targets<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        label, status, disp0, n, shift_max, target, mask);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int sv_band_apply(const float *out, const double *disp0, int W, int H, double b_thr,
                  double rad_k, int rad_min, int R, double shift_max, double *centre,
                  uint8_t *rad, void *stream) {
    if (!out || !disp0 || !centre || !rad) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1) { set_error("bad shape"); return SV_ERR_SHAPE; }
    if (R < 0 || R > 126 || rad_min < 0 || !std::isfinite(b_thr) || !std::isfinite(rad_k) ||
        !std::isfinite(shift_max)) {
        set_error("bad band parameters");
        return SV_ERR_PARAM;
    }
    const long HW = (long)W * H;
    count_launch();
    k_band_apply<<<(unsigned)((HW + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        out, disp0, HW, b_thr, rad_k, rad_min, R, shift_max, centre, rad);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

}  // extern "C"
