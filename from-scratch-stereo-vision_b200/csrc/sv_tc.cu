// sv_tc.cu -- BF16 implicit-GEMM convolutions on the sm_100a tensor cores
// (tcgen05.mma, FP32 accumulator in tensor memory) for the network's BF16
// path: the feature tower's 2-D convolutions (FeatureNet, stereonet.py:
// 1022-1070) and the cost filter's first two 3-D convolutions (CostFilter,
// 1071-1109), the first one fused with the cost volume (CostVolume,
// 740-842).
//
// GEMM view: M = output positions (a CTA tile of 128), N = output channels
// padded to 16, K = input channels x taps padded to a multiple of 16.
//  * B (weights) is packed once at checkpoint upload into the canonical
//    K-major, no-swizzle UMMA layout (8 x 16-byte core matrices, 128
//    contiguous bytes each) and copied to shared memory once per CTA;
//  * A (the im2col tile) is gathered by the CTA's 128 threads straight into
//    that layout -- thread m owns output row m and writes 16-byte chunks of
//    8 consecutive k -- and fenced into the async proxy; a shared table maps
//    k to (channel, tap offsets);
//  * one thread issues Kpad/16 tcgen05.mma (M=128, N=16, K=16) into a
//    32-column tensor-memory accumulator and commits them to an mbarrier;
//  * each warp reads its 32 accumulator rows back with tcgen05.ld
//    (32x32b.x16) and applies bias + activation.
// CTAs are persistent over tiles.  Every mbarrier wait is bounded: on
// timeout the kernel records SV_ERR_CUDA, stops and still frees its tensor
// memory.

#include <cuda_bf16.h>

#include <mutex>

#include "sv_common.cuh"
#include "sv_tc.cuh"

namespace sv {

namespace {

constexpr int kTcM = 128, kTcN = 16, kTmemCols = 32;
constexpr int kTcMaxK = 432;                  // 16 channels x 27 taps
constexpr unsigned kWaitLimit = 1u << 24;     // polls before a wait is declared failed

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, K-major without swizzle: start address,
// leading byte offset (between the two 8-element K halves of one MMA),
// stride byte offset (between 8-row groups), all >> 4; version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// kind::f16 instruction descriptor: D F32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) |
                                ((uint32_t)(kTcN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Bounded wait for phase `parity` of the barrier; true when it completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity,
                                          unsigned limit = kWaitLimit) {
    const uint32_t a = smem_u32(bar);
    for (unsigned it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace

// ktab[k] = {channel (-1: K padding), dz, dy, dx}: mode 0 input offsets
// (input z = od + dz, y = oy * stride + dy, x = ox * stride + dx); mode 1
// cost-volume offsets (d = od + dz, y = oy + dy, x = ox + dx).
__global__ void __launch_bounds__(kTcM) k_conv_tc(TcConv a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    __shared__ int4 ktab[kTcMaxK];
    unsigned char *sA = smem;                                   // 128 x Kpad BF16
    unsigned char *sB = smem + (size_t)a.Kpad * kTcM * 2;        // 16 x Kpad BF16
    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    const uint4 *wsrc = reinterpret_cast<const uint4 *>(a.wB);
    uint4 *wdst = reinterpret_cast<uint4 *>(sB);
    for (int i = tid; i < a.Kpad * kTcN * 2 / 16; i += kTcM) wdst[i] = __ldg(wsrc + i);
    const int taps = a.nd == 3 ? 27 : 9;
    for (int k = tid; k < a.Kpad; k += kTcM) {
        int4 e = make_int4(-1, 0, 0, 0);
        if (k < a.K) {
            const int c = k / taps;
            int t = k - c * taps;
            const int kd = a.nd == 3 ? t / 9 : 1;
            if (a.nd == 3) t -= kd * 9;
            const int ky = t / 3, kx = t - (t / 3) * 3;
            if (a.mode == 0)
                e = make_int4(c, kd - 1, ky * a.dil - a.pad, kx * a.dil - a.pad);
            else
                e = make_int4(c, kd - 1, ky - 1, kx - 1);
        }
        ktab[k] = e;
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;

    const long M = (long)a.OD * a.OH * a.OW;
    const long tiles_img = (M + kTcM - 1) / kTcM;
    const int nb = a.nb > 0 ? a.nb : 1;
    const long tiles = tiles_img * (a.mode == 0 ? a.nimg : 1) * nb;
    const int ohw = a.OH * a.OW;
    const long plane = (long)a.D * a.H * a.W;     // one input channel (mode 0)
    const long fplane = (long)a.H * a.W;          // one feature channel (mode 1)
    unsigned phase = 0;
    for (long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int item = (int)(tile / tiles_img);
        const int img = item / nb, bi = item - img * nb;
        const long mi = (tile - item * tiles_img) * kTcM + tid;
        const bool row_ok = mi < M;
        int od = 0, oy = 0, ox = 0;
        if (row_ok) {
            od = (int)(mi / ohw);
            const int r = (int)(mi - (long)od * ohw);
            oy = r / a.OW;
            ox = r - oy * a.OW;
        }
        // ---- gather this thread's im2col row, 8 k at a time
        const float *x0 = (img ? a.x[1] : a.x[0]) + bi * a.xs, *x1 = a.x[1] + bi * a.xs;
        const int by = a.mode == 0 ? oy * a.stride : oy, bx = a.mode == 0 ? ox * a.stride : ox;
        for (int kg = 0; kg < a.Kpad / 8; ++kg) {
            __align__(16) __nv_bfloat16 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int4 e = ktab[kg * 8 + j];
                float f = 0.f;
                const int z = od + e.y, yy = by + e.z, xx = bx + e.w;
                if (row_ok && e.x >= 0 && z >= 0 && z < a.D && yy >= 0 && yy < a.H && xx >= 0 &&
                    xx < a.W) {
                    if (a.mode == 0) {
                        f = __ldg(x0 + e.x * plane + ((long)z * a.H + yy) * a.W + xx);
                    } else if (xx < z) {
                        f = 2.0f;
                    } else {
                        const long o = e.x * fplane + (long)yy * a.W + xx;
                        f = fabsf(__ldg(x0 + o) - __ldg(x1 + o - z));
                    }
                }
                v[j] = __float2bfloat16_rn(f);
            }
            *reinterpret_cast<uint4 *>(sA + (size_t)(kg * (kTcM / 8) + (tid >> 3)) * 128 +
                                       (tid & 7) * 16) = *reinterpret_cast<const uint4 *>(v);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0 && !failed) {
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int ks = 0; ks < a.Kpad / 16; ++ks) {
                const uint64_t da = umma_desc(a0 + ks * 2 * (kTcM / 8) * 128, (kTcM / 8) * 128, 128);
                const uint64_t db = umma_desc(b0 + ks * 2 * (kTcN / 8) * 128, (kTcN / 8) * 128, 128);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(kIdescBf16), "r"(ks));
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                ::"r"(smem_u32(&mbar))
                : "memory");
        }
        // ---- wait for the accumulator (bounded), then the epilogue
        if (!failed && !mbar_wait(&mbar, phase)) {
            failed = 1;
            flag_error(a.err, SV_ERR_TIMEOUT);
        }
        phase ^= 1u;
        __syncthreads();
        if (failed) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row_ok) {
            float *y = (img ? a.y[1] : a.y[0]) + bi * a.ys;
            const float *aux = a.aux ? a.aux + bi * a.ys : nullptr;
#pragma unroll
            for (int n = 0; n < kTcN; ++n) {
                if (n < a.OC) {
                    float v = __uint_as_float(r[n]);
                    if (a.bias) v += __ldg(a.bias + n);
                    if (a.act == 1) v = v > 0.f ? v : v * 0.2f;
                    if (a.act == 2) v = __ldg(aux + (long)n * M + mi) > 0.f ? v : v * 0.2f;
                    y[(long)n * M + mi] = v;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(kTmemCols));
}

// Element (n, k) of the 16 x Kpad operand B sits in core matrix
// (k / 8, n / 8) -- core matrices ordered k-group-major, 2 per k group --
// at row n % 8 (16 bytes per row), column k % 8.
void tc_pack_weights(const double *w, int OC, int K, uint16_t *out) {
    const int Kpad = tc_kpad(K);
    for (int n = 0; n < kTcN; ++n)
        for (int k = 0; k < Kpad; ++k) {
            const float v = (n < OC && k < K) ? (float)w[(long)n * K + k] : 0.f;
            const __nv_bfloat16 b = __float2bfloat16_rn(v);
            const size_t byte = (size_t)((k / 8) * 2 + n / 8) * 128 + (n % 8) * 16 + (k % 8) * 2;
            out[byte / 2] = *reinterpret_cast<const uint16_t *>(&b);
        }
}

// 2-D convolutions (mode 0, nd 2).  A CTA tile is 32 x 4 output pixels.
// The input patch the tile reads -- every channel, the tile's rows and
// columns scaled by the stride plus the dilated halo -- is first staged in
// shared memory as BF16 by whole warps reading rows (coalesced, all loads
// independent), and the im2col operand A is then built from shared memory:
// element (m, k) is patch[ktab[k] + base(m)].  The MMA issue, the bounded
// wait and the epilogue are those of k_conv_tc.
constexpr int kT2W = 32, kT2H = 4;
constexpr int kT2Cols = 3;              // patch columns per lane: PW <= 96

__global__ void __launch_bounds__(kTcM) k_conv2d_tc(TcConv a, int PH, int PW) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    __shared__ int ktab[kTcMaxK];                  // patch offset of k, -1 for K padding
    unsigned char *sA = smem;                                   // 128 x Kpad BF16
    unsigned char *sB = smem + (size_t)a.Kpad * kTcM * 2;        // 16 x Kpad BF16
    __nv_bfloat16 *patch = reinterpret_cast<__nv_bfloat16 *>(sB + (size_t)a.Kpad * kTcN * 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    const uint4 *wsrc = reinterpret_cast<const uint4 *>(a.wB);
    uint4 *wdst = reinterpret_cast<uint4 *>(sB);
    for (int i = tid; i < a.Kpad * kTcN * 2 / 16; i += kTcM) wdst[i] = __ldg(wsrc + i);
    const int pplane = PH * PW;
    for (int k = tid; k < a.Kpad; k += kTcM) {
        int e = -1;
        if (k < a.K) {
            const int c = k / 9, t = k - (k / 9) * 9;
            const int ky = t / 3, kx = t - (t / 3) * 3;
            e = c * pplane + ky * a.dil * PW + kx * a.dil;
        }
        ktab[k] = e;
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;

    const int tiles_x = (a.OW + kT2W - 1) / kT2W, tiles_y = (a.OH + kT2H - 1) / kT2H;
    const long tiles_img = (long)tiles_x * tiles_y;
    const int nb = a.nb > 0 ? a.nb : 1;
    const long tiles = tiles_img * a.nimg * nb;
    const long plane = (long)a.H * a.W, M = (long)a.OH * a.OW;
    const int my = tid / kT2W, mx = tid - (tid / kT2W) * kT2W;
    const int base = my * a.stride * PW + mx * a.stride;
    unsigned phase = 0;
    for (long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int item = (int)(tile / tiles_img);
        const int img = item / nb, bi = item - img * nb;
        const int t2 = (int)(tile - item * tiles_img);
        const int ty0 = (t2 / tiles_x) * kT2H, tx0 = (t2 - (t2 / tiles_x) * tiles_x) * kT2W;
        const float *x0 = (img ? a.x[1] : a.x[0]) + bi * a.xs;
        const int iy0 = ty0 * a.stride - a.pad, ix0 = tx0 * a.stride - a.pad;
        // ---- stage the patch: each warp takes 8 patch rows at a time, every
        // lane up to kT2Cols columns of each, all loads issued before the stores
        const int nrows = a.IC * PH;
        for (int r0 = warp; r0 < nrows; r0 += (kTcM / 32) * 8) {
            float v[8][kT2Cols];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int r = r0 + u * (kTcM / 32);
                const int c = r / PH, py = r - (r / PH) * PH;
                const int gy = iy0 + py;
                const bool rok = r < nrows && gy >= 0 && gy < a.H;
                const float *src = x0 + c * plane + (long)gy * a.W;
#pragma unroll
                for (int q = 0; q < kT2Cols; ++q) {
                    const int px = lane + 32 * q, gx = ix0 + px;
                    v[u][q] = rok && px < PW && gx >= 0 && gx < a.W ? __ldg(src + gx) : 0.f;
                }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int r = r0 + u * (kTcM / 32);
                if (r >= nrows) break;
#pragma unroll
                for (int q = 0; q < kT2Cols; ++q) {
                    const int px = lane + 32 * q;
                    if (px < PW) patch[(long)r * PW + px] = __float2bfloat16_rn(v[u][q]);
                }
            }
        }
        __syncthreads();
        const int oy = ty0 + my, ox = tx0 + mx;
        const bool row_ok = oy < a.OH && ox < a.OW;
        for (int kg = 0; kg < a.Kpad / 8; ++kg) {
            __align__(16) __nv_bfloat16 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int e = ktab[kg * 8 + j];
                v[j] = row_ok && e >= 0 ? patch[e + base] : __float2bfloat16_rn(0.f);
            }
            *reinterpret_cast<uint4 *>(sA + (size_t)(kg * (kTcM / 8) + (tid >> 3)) * 128 +
                                       (tid & 7) * 16) = *reinterpret_cast<const uint4 *>(v);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0 && !failed) {
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int ks = 0; ks < a.Kpad / 16; ++ks) {
                const uint64_t da = umma_desc(a0 + ks * 2 * (kTcM / 8) * 128, (kTcM / 8) * 128, 128);
                const uint64_t db = umma_desc(b0 + ks * 2 * (kTcN / 8) * 128, (kTcN / 8) * 128, 128);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(kIdescBf16), "r"(ks));
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                ::"r"(smem_u32(&mbar))
                : "memory");
        }
        if (!failed && !mbar_wait(&mbar, phase)) {
            failed = 1;
            flag_error(a.err, SV_ERR_TIMEOUT);
        }
        phase ^= 1u;
        __syncthreads();
        if (failed) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row_ok) {
            const long mi = (long)oy * a.OW + ox;
            float *y = (img ? a.y[1] : a.y[0]) + bi * a.ys;
            const float *aux = a.aux ? a.aux + bi * a.ys : nullptr;
#pragma unroll
            for (int n = 0; n < kTcN; ++n) {
                if (n < a.OC) {
                    float v = __uint_as_float(r[n]);
                    if (a.bias) v += __ldg(a.bias + n);
                    if (a.act == 1) v = v > 0.f ? v : v * 0.2f;
                    if (a.act == 2) v = __ldg(aux + (long)n * M + mi) > 0.f ? v : v * 0.2f;
                    y[(long)n * M + mi] = v;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(kTmemCols));
}

// Stride-1 2-D convolutions with at most 16 input channels, without an
// im2col operand.  A tile is 128 consecutive output pixels of one row; the
// three input rows its taps read (rows oy - pad + ky * dil) are staged in
// shared memory as BF16 in the UMMA K-major layout directly: two planes of 8
// channels each, every pixel 16 bytes, so 8 consecutive pixels form one
// 128-byte core matrix.  The A operand of tap (ky, kx) is then the same
// patch read from pixel ky * PWp + kx * dil on (start address shifted by a
// multiple of 16 bytes; LBO = one channel plane, SBO = 128 bytes), and a
// tile is 9 MMAs of K = 16 -- one per tap -- accumulating in tensor memory.
// Operand B is re-ordered on the way into shared memory from the packed
// channel-major K (k = c * 9 + t) to one 16-channel block per tap
// (k = t * 16 + c, zero for c >= IC).  The bounded wait and the epilogue
// are those of k_conv2d_tc.
constexpr int kTapW = 128;              // output pixels per tile
constexpr int kTapMaxDil = 8;

__device__ __forceinline__ int tc_b_off(int n, int k) {    // BF16 index in a packed operand B
    return (((k >> 3) * 2 + (n >> 3)) * 128 + (n & 7) * 16 + (k & 7) * 2) >> 1;
}

__global__ void __launch_bounds__(kTcM) k_conv2d_tc_tap(TcConv a, int PWp) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    unsigned char *sB = smem;                                    // 9 taps x 16 x 16 BF16
    unsigned char *patch = smem + 9 * 512;                       // [2][3][PWp] x 16 bytes
    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    {
        uint16_t *wd = reinterpret_cast<uint16_t *>(sB);
        for (int i = tid; i < 9 * 256; i += kTcM) {
            const int t = i >> 8, n = (i >> 4) & 15, c = i & 15;
            uint16_t v = 0;
            if (c < a.IC) v = a.wB[tc_b_off(n, c * 9 + t)];
            wd[tc_b_off(n, t * 16 + c)] = v;
        }
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;

    const int tiles_x = (a.OW + kTapW - 1) / kTapW;
    const long tiles_img = (long)tiles_x * a.OH;
    const int nb = a.nb > 0 ? a.nb : 1;
    const long tiles = tiles_img * a.nimg * nb;
    const long plane = (long)a.H * a.W, M = (long)a.OH * a.OW;
    const uint32_t lbo = 3u * (uint32_t)PWp * 16u;               // one 8-channel plane
    unsigned phase = 0;
    for (long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int item = (int)(tile / tiles_img);
        const int img = item / nb, bi = item - img * nb;
        const int t2 = (int)(tile - item * tiles_img);
        const int oy = t2 / tiles_x, ox0 = (t2 - oy * tiles_x) * kTapW;
        const float *x0 = (img ? a.x[1] : a.x[0]) + bi * a.xs;
        // ---- stage rows oy - pad + ky * dil: consecutive threads take
        // consecutive pixels, each 8 channels packed into one 16-byte store
        for (int e = tid; e < 2 * 3 * PWp; e += kTcM) {
            const int r = e / PWp, px = e - r * PWp;
            const int ch = r / 3, ky = r - ch * 3;
            const int iy = oy - a.pad + ky * a.dil, ix = ox0 - a.pad + px;
            const bool ok = iy >= 0 && iy < a.H && ix >= 0 && ix < a.W;
            const float *src = x0 + (long)iy * a.W + ix;
            uint32_t q[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c0 = ch * 8 + 2 * j;
                const float f0 = ok && c0 < a.IC ? __ldg(src + c0 * plane) : 0.f;
                const float f1 = ok && c0 + 1 < a.IC ? __ldg(src + (c0 + 1) * plane) : 0.f;
                const __nv_bfloat162 h2 = __floats2bfloat162_rn(f0, f1);
                q[j] = *reinterpret_cast<const uint32_t *>(&h2);
            }
            *reinterpret_cast<uint4 *>(patch + (size_t)(r * PWp + px) * 16) =
                make_uint4(q[0], q[1], q[2], q[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0 && !failed) {
            const uint32_t p0 = smem_u32(patch), b0 = smem_u32(sB);
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const int ky = t / 3, kx = t - (t / 3) * 3;
                const uint64_t da =
                    umma_desc(p0 + (uint32_t)(ky * PWp + kx * a.dil) * 16u, lbo, 128);
                const uint64_t db = umma_desc(b0 + t * 512, (kTcN / 8) * 128, 128);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(kIdescBf16), "r"(t));
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                ::"r"(smem_u32(&mbar))
                : "memory");
        }
        if (!failed && !mbar_wait(&mbar, phase)) {
            failed = 1;
            flag_error(a.err, SV_ERR_TIMEOUT);
        }
        phase ^= 1u;
        __syncthreads();
        if (failed) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int ox = ox0 + tid;
        if (ox < a.OW) {
            const long mi = (long)oy * a.OW + ox;
            float *y = (img ? a.y[1] : a.y[0]) + bi * a.ys;
            const float *aux = a.aux ? a.aux + bi * a.ys : nullptr;
#pragma unroll
            for (int n = 0; n < kTcN; ++n) {
                if (n < a.OC) {
                    float v = __uint_as_float(r[n]);
                    if (a.bias) v += __ldg(a.bias + n);
                    if (a.act == 1) v = v > 0.f ? v : v * 0.2f;
                    if (a.act == 2) v = __ldg(aux + (long)n * M + mi) > 0.f ? v : v * 0.2f;
                    y[(long)n * M + mi] = v;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(kTmemCols));
}

// Per-device launch set-up, done once: the SM count and each kernel's
// dynamic shared-memory limit (raised to kTcSmemMax; every launch checks
// its own size against it).  Launches stay free of attribute calls.
constexpr size_t kTcSmemMax = 200 * 1024;
enum { kKConv = 0, kKConv2d = 1, kKWgrad = 2, kKConv2dTap = 3, kKCount = 4 };

static int tc_setup(int which, const void *fn, int *sms) {
    static std::mutex mu;
    static int cached_sms[64];
    static bool attr_done[64][kKCount];
    int dev = 0;
    SV_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("device ordinal %d out of range", dev);
        return SV_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!cached_sms[dev])
        SV_CUDA_TRY(cudaDeviceGetAttribute(&cached_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    if (!attr_done[dev][which]) {
        SV_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmemMax));
        attr_done[dev][which] = true;
    }
    *sms = cached_sms[dev];
    return SV_OK;
}

// CTAs per SM for a kernel using `smem` bytes of dynamic shared memory.
static long tc_ctas_per_sm(size_t smem) {
    const long per = (long)((220 * 1024) / (smem + 8 * 1024));
    return per < 1 ? 1 : (per > 4 ? 4 : per);
}

static int launch_conv2d_tc(const TcConv &a, cudaStream_t st) {
    if (a.stride == 1 && a.IC <= 16 && a.dil <= kTapMaxDil && a.pad >= 0 &&
        a.K == a.IC * 9) {
        const int PWp = kTapW + 2 * a.dil;
        const size_t smem = 9 * 512 + (size_t)2 * 3 * PWp * 16;
        const long tiles = (long)((a.OW + kTapW - 1) / kTapW) * a.OH * a.nimg *
                           (a.nb > 0 ? a.nb : 1);
        if (tiles == 0) return SV_OK;
        int sms = 148;
        const int rc = tc_setup(kKConv2dTap, (const void *)k_conv2d_tc_tap, &sms);
        if (rc) return rc;
        const long cap = (long)sms * 8;               // 8 CTAs (32 TMEM columns each) per SM
        const unsigned blocks = (unsigned)(tiles < cap ? tiles : cap);
        count_launch();
        k_conv2d_tc_tap<<<blocks, kTcM, smem, st>>>(a, PWp);
        SV_LAUNCH_CHECK();
        return SV_OK;
    }
    const int PH = (kT2H - 1) * a.stride + 2 * a.dil + 1;
    const int PW = (kT2W - 1) * a.stride + 2 * a.dil + 1;
    const size_t patch = ((size_t)a.IC * PH * PW * 2 + 15) / 16 * 16;
    const size_t smem = (size_t)a.Kpad * (kTcM + kTcN) * 2 + patch;
    if (smem > kTcSmemMax || PW > 32 * kT2Cols) {
        set_error("tensor-core conv: IC=%d dil=%d stride=%d patch too large", a.IC, a.dil,
                  a.stride);
        return SV_ERR_PARAM;
    }
    const long tiles = (long)((a.OW + kT2W - 1) / kT2W) * ((a.OH + kT2H - 1) / kT2H) * a.nimg *
                       (a.nb > 0 ? a.nb : 1);
    if (tiles == 0) return SV_OK;
    int sms = 148;
    const int rc = tc_setup(kKConv2d, (const void *)k_conv2d_tc, &sms);
    if (rc) return rc;
    const long cap = (long)sms * tc_ctas_per_sm(smem);
    const unsigned blocks = (unsigned)(tiles < cap ? tiles : cap);
    count_launch();
    k_conv2d_tc<<<blocks, kTcM, smem, st>>>(a, PH, PW);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

// Self-test of the failure path every tensor-core kernel here shares: a CTA
// allocates its tensor memory, arms an mbarrier that nothing will arrive at
// (no MMA is issued), and waits with a bounded poll count.  The wait must
// give up, record SV_ERR_TIMEOUT in the flag, free the tensor memory and
// return, leaving the context usable.  done receives 1 once the CTA has
// passed its dealloc.
__global__ void __launch_bounds__(kTcM) k_selftest_wait(unsigned limit, int *flag, int *done) {
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;
    if (threadIdx.x == 0 && !mbar_wait(&mbar, 0, limit)) {
        failed = 1;
        flag_error(flag, SV_ERR_TIMEOUT);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(kTmemCols));
    __syncthreads();
    if (threadIdx.x == 0) *done = failed ? 1 : 2;
}

int launch_selftest_wait(unsigned limit, int *flag, int *done, cudaStream_t st) {
    count_launch();
    k_selftest_wait<<<1, kTcM, 0, st>>>(limit, flag, done);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_conv_tc(const TcConv &a, cudaStream_t st) {
    if (a.OC < 1 || a.OC > kTcN || a.K < 1 || a.K > kTcMaxK || a.Kpad != tc_kpad(a.K) ||
        (a.mode == 0 && (a.nimg < 1 || a.nimg > 2)) || (a.mode == 1 && a.nd != 3) ||
        !a.wB || !a.err || (a.act == 2 && !a.aux) || a.nb < 0) {
        set_error("tensor-core conv: IC=%d OC=%d K=%d outside the kernel's shapes", a.IC, a.OC,
                  a.K);
        return SV_ERR_PARAM;
    }
    if (a.mode == 0 && a.nd == 2) {
        if (a.K != a.IC * 9 || a.D != 1 || a.OD != 1 || a.stride < 1 || a.dil < 1) {
            set_error("tensor-core conv2d: inconsistent shape");
            return SV_ERR_PARAM;
        }
        return launch_conv2d_tc(a, st);
    }
    const size_t smem = (size_t)a.Kpad * (kTcM + kTcN) * 2;
    const long M = (long)a.OD * a.OH * a.OW;
    if (M == 0) return SV_OK;
    const long tiles =
        (M + kTcM - 1) / kTcM * (a.mode == 0 ? a.nimg : 1) * (a.nb > 0 ? a.nb : 1);
    int sms = 148;
    const int rc = tc_setup(kKConv, (const void *)k_conv_tc, &sms);
    if (rc) return rc;
    const long cap = (long)sms * tc_ctas_per_sm(smem);
    const unsigned blocks = (unsigned)(tiles < cap ? tiles : cap);
    count_launch();
    k_conv_tc<<<blocks, kTcM, smem, st>>>(a);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

// ------------------------------------------------------- weight gradient
// D[m][n] = sum over pixels p of A[m][p] * B[n][p] with A[m = c*9 + t][p] =
// x[c][p + tap t] (row IC*9 is all ones, giving the bias gradient) and
// B[n = o][p] = g[o][p].  M is 1 or 2 tiles of 128 rows (IC*9 + 1 <= 256),
// N = 16, K = the pixels, 64 per chunk.  CTAs stride over chunks with two
// shared-memory stages: the gather of chunk i overlaps the MMAs of chunk
// i-1, and stage reuse waits for the commit of chunk i-2.  At the end every
// CTA adds its FP32 partial sums into gw / gb.
constexpr int kWgK = 64;

__global__ void __launch_bounds__(kTcM) k_wgrad_tc(TcWgrad a, int mtiles) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int failed;
    __shared__ int4 pix[2][kWgK];                    // (item, y, x, valid)
    const size_t a_tile = (size_t)kTcM * kWgK * 2;
    const size_t stage = (size_t)mtiles * a_tile + (size_t)kTcN * kWgK * 2;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;
    const long HW = (long)a.H * a.W;
    const long P = HW * a.nb;
    const long chunks = (P + kWgK - 1) / kWgK;
    const int KR = a.IC * 9;
    // this thread's A rows, one per M tile
    int rc[2], rdy[2], rdx[2], rkind[2];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int m = mt * kTcM + tid;
        rc[mt] = 0; rdy[mt] = 0; rdx[mt] = 0;
        rkind[mt] = m < KR ? 0 : (m == KR ? 1 : 2);
        if (m < KR) {
            const int c = m / 9, t = m - (m / 9) * 9;
            rc[mt] = c;
            rdy[mt] = (t / 3 - 1) * a.dil;
            rdx[mt] = (t - (t / 3) * 3 - 1) * a.dil;
        }
    }
    int it = 0;
    for (long ch = blockIdx.x; ch < chunks; ch += gridDim.x, ++it) {
        const int s = it & 1;
        unsigned char *sA = smem + s * stage;
        unsigned char *sB = sA + (size_t)mtiles * a_tile;
        if (it >= 2 && !failed && !mbar_wait(&mbar[s], ((it - 2) >> 1) & 1)) {
            failed = 1;
            flag_error(a.err, SV_ERR_TIMEOUT);
        }
        __syncthreads();
        if (failed) break;
        if (tid < kWgK) {
            const long p = ch * kWgK + tid;
            int4 e = make_int4(0, 0, 0, 0);
            if (p < P) {
                const int item = (int)(p / HW);
                const int r = (int)(p - item * HW);
                e = make_int4(item, r / a.W, r - (r / a.W) * a.W, 1);
            }
            pix[s][tid] = e;
        }
        __syncthreads();
        {   // B: thread (n, 8 pixels)
            const int n = tid >> 3, kg = tid & 7;
            __align__(16) __nv_bfloat16 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int4 e = pix[s][kg * 8 + j];
                float f = 0.f;
                if (e.w && n < a.OC)
                    f = __ldg(a.g + e.x * a.gs + n * HW + (long)e.y * a.W + e.z);
                v[j] = __float2bfloat16_rn(f);
            }
            *reinterpret_cast<uint4 *>(sB + (size_t)(kg * 2 + (n >> 3)) * 128 + (n & 7) * 16) =
                *reinterpret_cast<const uint4 *>(v);
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {        // A: this thread's row of each M tile
            if (mt >= mtiles) break;
            unsigned char *tA = sA + (size_t)mt * a_tile;
            const float *xc = a.x + (long)rc[mt] * HW;
            for (int kg = 0; kg < kWgK / 8; ++kg) {
                __align__(16) __nv_bfloat16 v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int4 e = pix[s][kg * 8 + j];
                    float f = 0.f;
                    if (e.w) {
                        if (rkind[mt] == 0) {
                            const int yy = e.y + rdy[mt], xx = e.z + rdx[mt];
                            if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W)
                                f = __ldg(xc + e.x * a.xs + (long)yy * a.W + xx);
                        } else if (rkind[mt] == 1) {
                            f = 1.f;
                        }
                    }
                    v[j] = __float2bfloat16_rn(f);
                }
                *reinterpret_cast<uint4 *>(tA + (size_t)(kg * (kTcM / 8) + (tid >> 3)) * 128 +
                                           (tid & 7) * 16) = *reinterpret_cast<const uint4 *>(v);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0) {
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int mt = 0; mt < mtiles; ++mt) {
                for (int ks = 0; ks < kWgK / 16; ++ks) {
                    const uint64_t da = umma_desc(a0 + mt * (uint32_t)a_tile +
                                                      ks * 2 * (kTcM / 8) * 128,
                                                  (kTcM / 8) * 128, 128);
                    const uint64_t db =
                        umma_desc(b0 + ks * 2 * (kTcN / 8) * 128, (kTcN / 8) * 128, 128);
                    const uint32_t acc = (it > 0 || ks > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        ::"r"(tmem + mt * kTcN), "l"(da), "l"(db), "r"(kIdescBf16), "r"(acc));
                }
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                ::"r"(smem_u32(&mbar[s]))
                : "memory");
        }
    }
    // the last commit covers every MMA this CTA issued
    if (it > 0 && !failed && !mbar_wait(&mbar[(it - 1) & 1], ((it - 1) >> 1) & 1)) {
        failed = 1;
        flag_error(a.err, SV_ERR_TIMEOUT);
    }
    __syncthreads();
    if (it > 0 && !failed) {
        asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            if (mt >= mtiles) break;
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                  "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                  "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + mt * kTcN));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int m = mt * kTcM + tid;
#pragma unroll
            for (int n = 0; n < kTcN; ++n) {
                if (n >= a.OC) break;
                const float v = __uint_as_float(r[n]);
                if (m < KR) atomicAdd(a.gw + (long)n * KR + m, v);
                else if (m == KR) atomicAdd(a.gb + n, v);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(kTmemCols));
}

int launch_wgrad_tc(const TcWgrad &a, cudaStream_t st) {
    if (a.IC < 1 || a.OC < 1 || a.OC > kTcN || a.IC * 9 + 1 > 2 * kTcM || a.dil < 1 ||
        a.H < 1 || a.W < 1 || a.nb < 1 || !a.x || !a.g || !a.gw || !a.gb || !a.err) {
        set_error("tensor-core weight gradient: IC=%d OC=%d outside the kernel's shapes", a.IC,
                  a.OC);
        return SV_ERR_PARAM;
    }
    const int mtiles = (a.IC * 9 + 1 + kTcM - 1) / kTcM;
    const size_t smem = 2 * ((size_t)mtiles * kTcM * kWgK * 2 + (size_t)kTcN * kWgK * 2);
    const long chunks = ((long)a.H * a.W * a.nb + kWgK - 1) / kWgK;
    int sms = 148;
    const int rc = tc_setup(kKWgrad, (const void *)k_wgrad_tc, &sms);
    if (rc) return rc;
    const long cap = (long)sms * 2;
    const unsigned blocks = (unsigned)(chunks < cap ? chunks : cap);
    count_launch();
    k_wgrad_tc<<<blocks, kTcM, smem, st>>>(a, mtiles);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

__global__ void k_pack_weights(const float *__restrict__ w, int OC, int IC, int transpose,
                               int K, int Kpad, uint16_t *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kTcN * Kpad) return;
    const int n = i / Kpad, k = i - (i / Kpad) * Kpad;
    float v = 0.f;
    if (!transpose) {
        if (n < OC && k < K) v = w[n * K + k];
    } else if (n < IC && k < K) {
        const int o = k / 9, t = k - (k / 9) * 9;
        v = w[(o * IC + n) * 9 + (8 - t)];
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    out[((size_t)((k >> 3) * 2 + (n >> 3)) * 128 + (n & 7) * 16 + (k & 7) * 2) / 2] =
        *reinterpret_cast<const uint16_t *>(&b);
}

int launch_pack_weights(const float *w, int OC, int IC, int transpose, uint16_t *out,
                        cudaStream_t st) {
    const int K = (transpose ? OC : IC) * 9;
    if ((transpose ? IC : OC) > kTcN) {
        set_error("packed operand has more than 16 rows");
        return SV_ERR_PARAM;
    }
    const int Kpad = tc_kpad(K);
    count_launch();
    k_pack_weights<<<(kTcN * Kpad + 255) / 256, 256, 0, st>>>(w, OC, IC, transpose, K, Kpad,
                                                              out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

}  // namespace sv
