// sv_select.cu -- _peak (stereonet.py:3866-3869): sorted(disp)[int(n * q)],
// the 95% quantile predict_auto steers the work width with.
//
// Exact selection on order-preserving 64-bit keys of the FP64 values (signed
// zeros share one key: they compare equal in the sort, and a zero peak is
// replaced by 0.5 anyway).  Six passes over digits of 11, 11, 11, 11, 10 and
// 10 bits from the top.  Pass p: every CTA histograms digit p of the keys
// that match the prefix chosen so far into 2048 shared-memory bins
// (warp-aggregated), adds its non-zero bins into a global histogram, and the
// last CTA to finish (a device-scope counter) scans that histogram, picks the
// bin holding the rank and extends the prefix.  Passes 0 and 1 are one launch
// each; passes 2..5 run in one CTA over the few keys that still match
// (k_sel_compact); after pass 5 the prefix is the key.  Up to 16,384 values
// all six passes run in one CTA over keys kept in shared memory
// (k_sel_small); the probe's FP32 map takes four 8-bit passes over 32-bit
// keys instead (k_sel_small_f32).

#include "sv_common.cuh"
#include "sv_netbatch.cuh"
#include "sv_network.cuh"
#include "sv_select.cuh"

namespace sv {

constexpr int SEL_LB = 4;              // values a thread loads before it histograms them

__global__ void k_sel_init(SelState *s, long long rank, unsigned *hist) {
    sel_init_block(s, rank, hist);
}

__device__ __forceinline__ void sel_pass_body(long blk, long nblk, const double *__restrict__ x,
                                              long n, int pass, SelState *__restrict__ s,
                                              unsigned *__restrict__ ghist) {
    __shared__ unsigned hist[SEL_NB];
    const int t = threadIdx.x, nt = blockDim.x;
    const unsigned long long pre = pass ? s->prefix : 0ull;
    for (int i = t; i < SEL_NB; i += nt) hist[i] = 0u;
    __syncthreads();
    const long stride = nblk * nt;
    for (long b0 = blk * (long)nt; b0 < n; b0 += SEL_LB * stride) {
        double v[SEL_LB];                  // this thread's loads, all in flight at once
#pragma unroll
        for (int u = 0; u < SEL_LB; ++u) {
            const long i = b0 + u * stride + t;
            v[u] = i < n ? x[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < SEL_LB; ++u) {
            const long i = b0 + u * stride + t;
            sel_count(hist, sel_key(v[u]), i < n, pre, pass);
        }
    }
    __syncthreads();
    sel_pass_finish(pass, s, ghist, hist, (unsigned)nblk);
}

__global__ void __launch_bounds__(1024)
    k_sel_pass(const double *__restrict__ x, long n, int pass, SelState *__restrict__ s,
               unsigned *__restrict__ ghist) {
    sel_pass_body(blockIdx.x, gridDim.x, x, n, pass, s, ghist);
}

// Batched: pass `pass` of every active pair's full-resolution select (each
// pair's CTAs cover its W x H map).
__global__ void __launch_bounds__(1024)
    k_b_sel_pass(NetLaunch L, const double *x, int pass, SelState *s, unsigned *ghist) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    sel_pass_body(c, L.pre[p + 1] - L.pre[p], net_slab(x, L, p), (long)P.W * P.H, pass,
                  net_slab(s, L, p), net_slab(ghist, L, p));
}

// After pass 1 the 22 top key bits are fixed and usually only a few hundred
// keys still match.  k_sel_compact gathers them (warp-aggregated appends);
// the last CTA to finish runs passes 2..5 over them in its shared memory,
// or, when more than SEL_CAND_CAP match (a plateau of equal values), over
// all n values read again from global memory, filtered by the prefix.
constexpr int SEL_CAND_CAP = 16384;      // keys (128 KB of dynamic shared memory)

// Passes pass0..5 in one CTA over `keys` (shared memory), or, when keys is
// NULL, over sel_key(x[i]) for all n values read from global memory.
__device__ void sel_passes_cta(const unsigned long long *keys, const double *__restrict__ x,
                               long n, int pass0, unsigned long long &prefix, long long &rank,
                               unsigned *hist, unsigned *wsum, int *owner,
                               unsigned long long *owner_excl, unsigned long long *s_prefix,
                               long long *s_rank) {
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5, nt = blockDim.x;
    if (t == 0) {
        *s_prefix = prefix;
        *s_rank = rank;
    }
    __syncthreads();
    for (int pass = pass0; pass < SEL_NPASS; ++pass) {
        const int shift = sel_shift(pass), bits = sel_bits(pass), top = shift + bits;
        const unsigned mask = (1u << bits) - 1u;
        for (int i = t; i < SEL_NB; i += nt) hist[i] = 0u;
        __syncthreads();
        const unsigned long long pre = *s_prefix;
        for (long i0 = 0; i0 < n; i0 += nt) {
            const long i = i0 + t;
            unsigned digit = 0xffffffffu;
            if (i < n) {
                const unsigned long long k = keys ? keys[i] : sel_key(x[i]);
                if (top >= 64 || (k >> top) == (pre >> top)) digit = (unsigned)(k >> shift) & mask;
            }
            const unsigned same = __match_any_sync(kFull, digit);
            if (digit != 0xffffffffu && lane == __ffs(same) - 1)
                atomicAdd(&hist[digit], __popc(same));
        }
        __syncthreads();
        const int per = SEL_NB / nt;
        unsigned long long loc = 0;
        for (int j = 0; j < per; ++j) loc += hist[t * per + j];
        unsigned long long incl = loc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[wid] = (unsigned)incl;
        __syncthreads();
        if (wid == 0) {
            const int nw = nt >> 5;
            unsigned long long w = lane < nw ? wsum[lane] : 0ull, v = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(kFull, v, o);
                if (lane >= o) v += y;
            }
            if (lane < nw) wsum[lane] = (unsigned)(v - w);
        }
        __syncthreads();
        const long long rk = *s_rank;
        const long long excl = (long long)(wsum[wid] + incl - loc);
        if (rk >= excl && rk < excl + (long long)loc) {
            *owner = t;
            *owner_excl = (unsigned long long)excl;
        }
        __syncthreads();
        if (t == *owner) {
            long long rr = rk - (long long)*owner_excl;
            int b = t * per;
            for (int j = 0; j < per; ++j) {
                const long long c = hist[t * per + j];
                if (rr < c) { b = t * per + j; break; }
                rr -= c;
            }
            *s_prefix = pre | ((unsigned long long)b << shift);
            *s_rank = rr;
        }
        __syncthreads();
    }
    prefix = *s_prefix;
    rank = *s_rank;
}

__device__ __forceinline__ void sel_compact_body(long blk, long nblk, const double *__restrict__ x,
                                                 long n, SelState *__restrict__ s,
                                                 unsigned long long *__restrict__ cand,
                                                 double *mirror) {
    extern __shared__ __align__(16) unsigned long long keys[];   // SEL_CAND_CAP
    __shared__ unsigned hist[SEL_NB];
    __shared__ unsigned wsum[32];
    __shared__ int owner;
    __shared__ unsigned long long owner_excl, s_prefix;
    __shared__ long long s_rank;
    __shared__ bool last;
    const int t = threadIdx.x, lane = t & 31, nt = blockDim.x;
    const int top = sel_shift(1);                    // bits above pass 2's digit are fixed
    const unsigned long long pre = s->prefix;
    const long stride = nblk * nt;
    for (long b0 = blk * (long)nt; b0 < n; b0 += SEL_LB * stride) {
        double v[SEL_LB];
#pragma unroll
        for (int u = 0; u < SEL_LB; ++u) {
            const long i = b0 + u * stride + t;
            v[u] = i < n ? x[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < SEL_LB; ++u) {
            const long i = b0 + u * stride + t;
            unsigned long long k = 0;
            bool hit = false;
            if (i < n) {
                k = sel_key(v[u]);
                hit = (k >> top) == (pre >> top);
            }
            const unsigned m = __ballot_sync(kFull, hit);
            if (m) {
                unsigned base = 0;
                if (lane == __ffs(m) - 1) base = atomicAdd(&s->count, __popc(m));
                base = __shfl_sync(kFull, base, __ffs(m) - 1);
                const unsigned pos = base + __popc(m & ((1u << lane) - 1u));
                if (hit && pos < SEL_CAND_CAP) cand[pos] = k;
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(&s->cdone, 1u) == (unsigned)nblk - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const unsigned cnt = __ldcg(&s->count);
    const bool fits = cnt <= (unsigned)SEL_CAND_CAP;
    if (fits)
        for (unsigned i = t; i < cnt; i += nt) keys[i] = __ldcg(cand + i);
    __syncthreads();
    unsigned long long prefix = s->prefix;
    long long rank = s->rank;
    // a bucket too large for shared memory (a plateau of equal values) is
    // finished by this CTA from all n values, filtered by the prefix
    sel_passes_cta(fits ? keys : nullptr, x, fits ? (long)cnt : n, 2, prefix, rank, hist, wsum,
                   &owner, &owner_excl, &s_prefix, &s_rank);
    if (t == 0) {
        s->prefix = prefix;
        s->rank = rank;
        s->value = sel_unkey(prefix);
        if (mirror) *reinterpret_cast<volatile double *>(mirror) = s->value;
    }
}


__global__ void __launch_bounds__(1024)
    k_sel_compact(const double *__restrict__ x, long n, SelState *__restrict__ s,
                  unsigned long long *__restrict__ cand, double *mirror) {
    sel_compact_body(blockIdx.x, gridDim.x, x, n, s, cand, mirror);
}

// Batched: the compaction and passes 2..5 of every active pair's select.
// The candidates follow the pair's two global histograms.
__global__ void __launch_bounds__(1024)
    k_b_sel_compact(NetLaunch L, const double *x, SelState *s, unsigned *hist) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    unsigned *h = net_slab(hist, L, p);
    sel_compact_body(c, L.pre[p + 1] - L.pre[p], net_slab(x, L, p), (long)P.W * P.H,
                     net_slab(s, L, p), reinterpret_cast<unsigned long long *>(h + 2 * SEL_NB),
                     nullptr);
}

// Small inputs (the probe's few thousand values): one CTA keeps every key in
// shared memory and runs the six passes there, one launch instead of seven.
constexpr long SEL_SMALL_CAP = 16384;     // keys (128 KB of dynamic shared memory)

template <typename T>
__global__ void __launch_bounds__(1024)
    k_sel_small(const T *__restrict__ x, long n, long long rank0, SelState *__restrict__ s,
                double *mirror) {
    extern __shared__ __align__(16) unsigned long long keys[];
    __shared__ unsigned hist[SEL_NB];
    __shared__ unsigned wsum[32];
    __shared__ int owner;
    __shared__ unsigned long long owner_excl, s_prefix;
    __shared__ long long s_rank;
    for (long i = threadIdx.x; i < n; i += blockDim.x) keys[i] = sel_key((double)x[i]);
    __syncthreads();
    unsigned long long prefix = 0ull;
    long long rank = rank0;
    sel_passes_cta(keys, nullptr, n, 0, prefix, rank, hist, wsum, &owner, &owner_excl, &s_prefix,
                   &s_rank);
    if (threadIdx.x == 0) {
        s->prefix = prefix;
        s->rank = rank;
        s->value = sel_unkey(prefix);
        if (mirror) *reinterpret_cast<volatile double *>(mirror) = s->value;
    }
}

// The probe's FP32 map: 32-bit order keys (the order of the floats is the
// order of the FP64 values they convert to exactly; signed zeros share a
// key), four 8-bit passes in one CTA of 1024 threads.  Up to SEL32_K keys a
// thread stay in registers across the passes (loaded together, so the CTA
// waits for one memory latency); larger maps (a tall pair's probe in a
// batch) are read again each pass.  Threads 0..255 own one bin each, so a
// pass's scan is one shuffle scan and an 8-term prefix.  Same result as the
// FP64 passes, a small fraction of the instructions at probe sizes.
constexpr int SEL32_T = 1024, SEL32_K = 16;

__device__ __forceinline__ unsigned sel_key32(float f) {
    const unsigned b = __float_as_uint(f == 0.0f ? 0.0f : f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ float sel_unkey32(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__device__ __forceinline__ void sel32_count(unsigned *hist, unsigned k, bool valid, unsigned pre,
                                            int pass) {
    const int shift = 24 - 8 * pass;
    unsigned digit = 0xffffffffu;
    if (valid && (pass == 0 || (k >> (shift + 8)) == (pre >> (shift + 8))))
        digit = (k >> shift) & 255u;
    const unsigned same = __match_any_sync(kFull, digit);
    if (digit != 0xffffffffu && (threadIdx.x & 31) == __ffs(same) - 1)
        atomicAdd(&hist[digit], __popc(same));
}

// The key of rank rank0 among the n values x[0..n) (whole CTA, 1024 threads).
__device__ unsigned sel32_cta(const float *__restrict__ x, int n, unsigned rank0) {
    __shared__ unsigned hist[256];
    __shared__ unsigned wsum[8];
    __shared__ unsigned s_prefix, s_rank;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const bool inreg = n <= SEL32_T * SEL32_K;          // the same for the whole CTA
    const int nj = (n + SEL32_T - 1) / SEL32_T;
    unsigned key[SEL32_K];
    if (inreg) {
#pragma unroll
        for (int j = 0; j < SEL32_K; ++j) {
            const int i = t + j * SEL32_T;
            key[j] = i < n ? sel_key32(__ldg(x + i)) : 0u;
        }
    }
    if (t == 0) {
        s_prefix = 0u;
        s_rank = rank0;
    }
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 24 - 8 * pass;
        if (t < 256) hist[t] = 0u;
        __syncthreads();                    // bins cleared, the prefix published
        const unsigned pre = s_prefix;
        if (inreg) {
#pragma unroll
            for (int j = 0; j < SEL32_K; ++j)
                if (j < nj) sel32_count(hist, key[j], t + j * SEL32_T < n, pre, pass);
        } else {
            for (int j = 0; j < nj; ++j) {
                const int i = t + j * SEL32_T;
                sel32_count(hist, i < n ? sel_key32(__ldg(x + i)) : 0u, i < n, pre, pass);
            }
        }
        __syncthreads();
        unsigned c = 0u, incl = 0u;
        if (t < 256) {
            c = hist[t];
            incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) wsum[wid] = incl;
        }
        __syncthreads();
        unsigned excl = 0u, r = 0u;
        if (t < 256) {
            excl = incl - c;
            for (int w = 0; w < wid; ++w) excl += wsum[w];
            r = s_rank;
        }
        __syncthreads();                    // every bin owner has read the rank
        if (t < 256 && r >= excl && r < excl + c) {   // exactly one bin holds it
            s_prefix = pre | ((unsigned)t << shift);
            s_rank = r - excl;
        }
    }
    __syncthreads();
    return s_prefix;
}

__global__ void __launch_bounds__(SEL32_T)
    k_sel_small_f32(const float *__restrict__ x, int n, unsigned rank0,
                    SelState *__restrict__ s, double *mirror) {
    const unsigned k = sel32_cta(x, n, rank0);
    if (threadIdx.x == 0) {
        const double v = (double)sel_unkey32(k);
        s->prefix = sel_key(v);
        s->rank = 0;
        s->value = v;
        if (mirror) *reinterpret_cast<volatile double *>(mirror) = v;
    }
}

// Batched probe select: one CTA per pair over the probe's FP32 map (the
// pass's Ww x Hw values), rank int(0.95 n) as _peak takes it.
__global__ void __launch_bounds__(SEL32_T)
    k_b_sel_probe(NetLaunch L, const float *x0, SelState *s0) {
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    const int n = P.Ww * P.Hw;
    const unsigned k = sel32_cta(net_slab(x0, L, p), n,
                                 (unsigned)(long long)__dmul_rn((double)n, 0.95));
    if (threadIdx.x == 0) {
        SelState *s = net_slab(s0, L, p);
        const double v = (double)sel_unkey32(k);
        s->prefix = sel_key(v);
        s->rank = 0;
        s->value = v;
    }
}

// A width decision over a whole map (a full-size map no network kernel
// wrote): CTAs of 256 values, the last one finishing.
template <typename T>
__global__ void __launch_bounds__(256)
    k_width_map(const T *__restrict__ x, long n, WidthFuse f, SelState *s, unsigned *ghist,
                double *mirror) {
    __shared__ unsigned hist[kWidthBins + 1];
    const int t = threadIdx.x;
    const long i = blockIdx.x * 256L + t;
    const double v = i < n ? (double)__ldg(x + i) : 0.0;
    for (int j = t; j <= f.m; j += 256) hist[j] = 0u;
    __syncthreads();
    width_count(hist, i < n ? width_bin_of(f, v) : -1);
    __syncthreads();
    width_finish(f, s, ghist, hist, gridDim.x, mirror);
}

// The same for a small map (the probe's, at most WIDTH_SMALL_CAP values):
// one CTA, up to 16 values a thread, no state to clear.
constexpr int WIDTH_SMALL_T = 1024, WIDTH_SMALL_K = 16;
constexpr long WIDTH_SMALL_CAP = (long)WIDTH_SMALL_T * WIDTH_SMALL_K;

template <typename T>
__global__ void __launch_bounds__(WIDTH_SMALL_T)
    k_width_small(const T *__restrict__ x, int n, WidthFuse f, SelState *s, double *mirror) {
    __shared__ unsigned hist[kWidthBins + 1];
    const int t = threadIdx.x;
    T v[WIDTH_SMALL_K];
#pragma unroll
    for (int u = 0; u < WIDTH_SMALL_K; ++u) {
        const int i = t + u * WIDTH_SMALL_T;
        v[u] = i < n ? __ldg(x + i) : T(0);
    }
    for (int i = t; i <= f.m; i += WIDTH_SMALL_T) hist[i] = 0u;
    __syncthreads();
    const int nu = (n + WIDTH_SMALL_T - 1) / WIDTH_SMALL_T;   // the same for the whole CTA
#pragma unroll
    for (int u = 0; u < WIDTH_SMALL_K; ++u)
        if (u < nu) {
            const int i = t + u * WIDTH_SMALL_T;
            width_count(hist, i < n ? width_bin_of(f, (double)v[u]) : -1);
        }
    __syncthreads();
    const int width = width_from_bins<false>(f, hist);
    if (t == 0) {
        s->value = (double)width;
        if (mirror) *reinterpret_cast<volatile double *>(mirror) = (double)width;
    }
}

// Batched probe decision: one CTA per pair over its probe map (the pass's
// Ww x Hw FP32 values, read from global memory), rule scale W / pw.
__global__ void __launch_bounds__(WIDTH_SMALL_T)
    k_b_width_probe(NetLaunch L, const float *x0, SelState *s0, double target, int max_width) {
    __shared__ unsigned hist[kWidthBins + 1];
    long long c;
    const int p = net_pair(L, c);
    const NetPair &P = L.pairs[p];
    if (!P.active) return;
    const float *__restrict__ x = net_slab(x0, L, p);
    const int n = P.Ww * P.Hw, t = threadIdx.x;
    WidthFuse f{{P.W, max_width, target, (double)P.W / (double)P.pw}, 0, 0,
                (long long)__dmul_rn((double)n, 0.95)};
    f.kmax = width_rule_kmax(f.rule);
    f.m = f.kmax - 48;
    for (int i = t; i <= f.m; i += WIDTH_SMALL_T) hist[i] = 0u;
    __syncthreads();
    for (int i0 = 0; i0 < n; i0 += WIDTH_SMALL_T) {     // the same trip count for every thread
        const int i = i0 + t;
        width_count(hist, i < n ? width_bin_of(f, (double)__ldg(x + i)) : -1);
    }
    __syncthreads();
    const int width = width_from_bins<false>(f, hist);
    if (t == 0) net_slab(s0, L, p)->value = (double)width;
}

int launch_b_width_probe(const NetLaunch &L, const NetSlab &s, double target, int max_width,
                         cudaStream_t st) {
    count_launch();
    k_b_width_probe<<<(unsigned)L.n, WIDTH_SMALL_T, 0, st>>>(L, s.d2, s.sel, target, max_width);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <typename T>
int launch_width_map(const T *x, long n, const WidthFuse &f, SelState *state, unsigned *hist,
                     cudaStream_t st, double *mirror) {
    if (n < 1 || n >= (1l << 32) || f.m < 0 || f.m > kWidthBins) {
        set_error("width decision: n=%ld m=%d", n, f.m);
        return SV_ERR_PARAM;
    }
    if (n <= WIDTH_SMALL_CAP) {
        count_launch();
        k_width_small<T><<<1, WIDTH_SMALL_T, 0, st>>>(x, (int)n, f, state, mirror);
    } else {
        count_launch();
        k_sel_init<<<1, 1024, 0, st>>>(state, f.rank, hist);
        count_launch();
        k_width_map<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, n, f, state, hist, mirror);
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template int launch_width_map<float>(const float *, long, const WidthFuse &, SelState *,
                                     unsigned *, cudaStream_t, double *);
template int launch_width_map<double>(const double *, long, const WidthFuse &, SelState *,
                                      unsigned *, cudaStream_t, double *);

// The select kernels' dynamic shared-memory limits, once per device.
static int select_setup() {
    int dev = 0;
    SV_CUDA_TRY(cudaGetDevice(&dev));
    static bool ready[64] = {false};
    if (dev >= 64 || !ready[dev]) {
        SV_CUDA_TRY(cudaFuncSetAttribute(k_sel_small<double>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(SEL_SMALL_CAP * sizeof(unsigned long long))));
        SV_CUDA_TRY(cudaFuncSetAttribute(k_sel_compact,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(SEL_CAND_CAP * sizeof(unsigned long long))));
        SV_CUDA_TRY(cudaFuncSetAttribute(k_b_sel_compact,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(SEL_CAND_CAP * sizeof(unsigned long long))));
        if (dev < 64) ready[dev] = true;
    }
    return SV_OK;
}

int launch_select(const double *x, long n, long long rank, SelState *state, unsigned *hist,
                  cudaStream_t st, double *mirror) {
    if (n < 1 || n >= (1l << 32) || rank < 0 || rank >= n) {
        set_error("select: n=%ld rank=%lld", n, rank);
        return SV_ERR_PARAM;
    }
    {
        const int rc = select_setup();
        if (rc) return rc;
    }
    if (n <= SEL_SMALL_CAP) {
        count_launch();
        k_sel_small<double><<<1, 1024, (size_t)n * sizeof(unsigned long long), st>>>(
            x, n, rank, state, mirror);
        SV_LAUNCH_CHECK();
        return SV_OK;
    }
    count_launch();
    k_sel_init<<<1, 1024, 0, st>>>(state, rank, hist);       // also clears the histograms
    const int blocks = grid_for(n, 1024 * 4, 148);
    // the candidates follow the two global histograms (8-byte aligned)
    unsigned long long *cand = reinterpret_cast<unsigned long long *>(hist + 2 * SEL_NB);
    for (int p = 0; p < 2; ++p) {
        count_launch();
        k_sel_pass<<<blocks, 1024, 0, st>>>(x, n, p, state, hist + (size_t)p * SEL_NB);
    }
    count_launch();
    k_sel_compact<<<blocks, 1024, (size_t)SEL_CAND_CAP * sizeof(unsigned long long), st>>>(
        x, n, state, cand, mirror);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_select_after_pass0(const double *x, long n, SelState *state, unsigned *hist,
                              cudaStream_t st, double *mirror) {
    if (n <= SEL_SMALL_CAP || n >= (1l << 32)) {
        set_error("select after pass 0: n=%ld", n);
        return SV_ERR_PARAM;
    }
    {
        const int rc = select_setup();
        if (rc) return rc;
    }
    const int blocks = grid_for(n, 1024 * 4, 148);
    unsigned long long *cand = reinterpret_cast<unsigned long long *>(hist + 2 * SEL_NB);
    count_launch();
    k_sel_pass<<<blocks, 1024, 0, st>>>(x, n, 1, state, hist + SEL_NB);
    count_launch();
    k_sel_compact<<<blocks, 1024, (size_t)SEL_CAND_CAP * sizeof(unsigned long long), st>>>(
        x, n, state, cand, mirror);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_b_sel_probe(const NetLaunch &L, const NetSlab &s, cudaStream_t st) {
    count_launch();
    k_b_sel_probe<<<(unsigned)L.n, SEL32_T, 0, st>>>(L, s.d2, s.sel);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_b_sel_rest(const NetLaunch &L, long long total, const NetSlab &s, cudaStream_t st) {
    {
        const int rc = select_setup();
        if (rc) return rc;
    }
    const unsigned B = (unsigned)(total > 0 ? total : 1);
    count_launch();
    k_b_sel_pass<<<B, 1024, 0, st>>>(L, s.full, 1, s.sel, s.hist + SEL_NB);
    count_launch();
    k_b_sel_compact<<<B, 1024, (size_t)SEL_CAND_CAP * sizeof(unsigned long long), st>>>(
        L, s.full, s.sel, s.hist);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

// CTAs of a pair's full-resolution select passes (the single-pair grid).
long long select_ctas(long n) { return grid_for(n, 1024 * 4, 148); }

long select_small_cap() { return SEL_SMALL_CAP; }

int launch_select_small_f32(const float *x, long n, long long rank, SelState *state,
                            cudaStream_t st, double *mirror) {
    if (n < 1 || n > SEL_SMALL_CAP || rank < 0 || rank >= n) {
        set_error("select: n=%ld rank=%lld", n, rank);
        return SV_ERR_PARAM;
    }
    const int rc = select_setup();
    if (rc) return rc;
    count_launch();
    k_sel_small_f32<<<1, SEL32_T, 0, st>>>(x, (int)n, (unsigned)rank, state, mirror);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

size_t select_state_bytes() { return sizeof(SelState); }
size_t select_value_offset() { return offsetof(SelState, value); }
size_t select_hist_words() { return 2 * (size_t)SEL_NB + 2 * (size_t)SEL_CAND_CAP; }

}  // namespace sv

namespace {
__global__ void k_peak_out(const sv::SelState *s, double *out) {
    const double v = s->value;
    *out = v > 0.5 ? v : 0.5;
}
}  // namespace

extern "C" {

size_t sv_peak_workspace_size(void) {
    return sv::align256(sizeof(sv::SelState)) + sv::select_hist_words() * sizeof(unsigned) + 256;
}

// _peak (stereonet.py:3866-3869): sorted(disp)[int(len(disp) * q)], floored
// at 0.5, into *out (device FP64).
int sv_peak(const double *disp, long n, double q, double *out, void *workspace,
            size_t workspace_bytes, void *stream) {
    if (!disp || !out) { sv::set_error("NULL argument"); return SV_ERR_NULL; }
    if (!(q >= 0.0 && q < 1.0)) { sv::set_error("q=%g outside [0, 1)", q); return SV_ERR_PARAM; }
    if (!workspace || workspace_bytes < sv_peak_workspace_size() ||
        ((uintptr_t)workspace & 255)) {
        sv::set_error("workspace must be 256-byte aligned and hold %zu bytes",
                      sv_peak_workspace_size());
        return SV_ERR_WORKSPACE;
    }
    const long long rank = (long long)((double)n * q);   // Python int(): toward zero
    cudaStream_t st = (cudaStream_t)stream;
    sv::SelState *s = static_cast<sv::SelState *>(workspace);
    unsigned *hist = reinterpret_cast<unsigned *>(static_cast<char *>(workspace) +
                                                  sv::align256(sizeof(sv::SelState)));
    const int rc = sv::launch_select(disp, n, rank, s, hist, st);
    if (rc) return rc;
    sv::count_launch();
    k_peak_out<<<1, 1, 0, st>>>(s, out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int sv_work_width(const double *map, long n, int W, double target_peak, int max_width,
                  double scale, int *width, void *workspace, size_t workspace_bytes,
                  void *stream) {
    if (!map || !width) { sv::set_error("NULL argument"); return SV_ERR_NULL; }
    if (n < 1 || n >= (1l << 32) || W < 1 || max_width < 1 || !std::isfinite(target_peak) ||
        !std::isfinite(scale) || !(scale > 0.0)) {
        sv::set_error("bad arguments");
        return SV_ERR_PARAM;
    }
    const sv::WidthRule r{W, max_width, target_peak, scale};
    const int kmax = sv::width_rule_kmax(r), m = kmax - 48;
    if (m > sv::kWidthBins) {
        sv::set_error("%d possible widths (at most %d)", m + 1, sv::kWidthBins + 1);
        return SV_ERR_PARAM;
    }
    if (!workspace || ((uintptr_t)workspace & 255) ||
        workspace_bytes < sv_peak_workspace_size()) {
        sv::set_error("workspace needs %zu bytes, 256-aligned", sv_peak_workspace_size());
        return SV_ERR_WORKSPACE;
    }
    auto *s = static_cast<sv::SelState *>(workspace);
    auto *hist = reinterpret_cast<unsigned *>(static_cast<char *>(workspace) +
                                              sv::align256(sizeof(sv::SelState)));
    cudaStream_t st = (cudaStream_t)stream;
    const sv::WidthFuse f{r, m, kmax, (long long)(n * 0.95)};
    const int rc = sv::launch_width_map<double>(map, n, f, s, hist, st, nullptr);
    if (rc) return rc;
    double v = 0.0;
    SV_CUDA_TRY(cudaMemcpyAsync(&v, reinterpret_cast<const char *>(s) + offsetof(sv::SelState, value),
                                sizeof(double), cudaMemcpyDeviceToHost, st));
    SV_CUDA_TRY(cudaStreamSynchronize(st));
    *width = (int)v;
    return SV_OK;
}

}  // extern "C"
