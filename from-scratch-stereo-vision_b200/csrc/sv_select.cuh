// sv_select.cuh -- the device parts of the exact radix select (_peak,
// stereonet.py:3866-3869) that other kernels share: the order keys, the
// per-pass digit histogram and the last-CTA prefix extension.  A network
// stage that ends with a full-resolution select runs pass 0 inside its own
// kernels (the first clears the state, the kernel that writes the FP64 map
// histograms the values it writes); sv_select.cu holds the select kernels.
#pragma once

#include "sv_common.cuh"

namespace sv {

constexpr int SEL_NPASS = 6;
constexpr int SEL_NB = 2048;

// Digits of 11, 11, 11, 11, 10 and 10 bits from the top of the 64-bit key.
__host__ __device__ constexpr int sel_bits(int pass) { return pass < 4 ? 11 : 10; }
__host__ __device__ constexpr int sel_shift(int pass) {
    return pass < 4 ? 53 - 11 * pass : (pass == 4 ? 10 : 0);
}

struct SelState {
    unsigned long long prefix;
    long long rank;
    double value;
    unsigned done[SEL_NPASS];          // CTAs finished per pass
    unsigned cdone;                    // CTAs finished in the compaction
    unsigned count;                    // keys left after pass 1
};

// Order key of an FP64 value (signed zeros share one key: they compare
// equal in the sort).
__device__ __forceinline__ unsigned long long sel_key(double d) {
    return ordkey(d == 0.0 ? 0.0 : d);
}

__device__ __forceinline__ double sel_unkey(unsigned long long k) {
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

__device__ __forceinline__ int sel_tid() { return threadIdx.y * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int sel_nt() { return blockDim.x * blockDim.y; }

// A selection of `rank` starts here: the state and both global pass
// histograms cleared, by one whole CTA.
__device__ __forceinline__ void sel_init_block(SelState *s, long long rank, unsigned *hist) {
    const int t = sel_tid(), nt = sel_nt();
    for (int i = t; i < 2 * SEL_NB; i += nt) hist[i] = 0u;
    if (t) return;
    s->prefix = 0ull;
    s->rank = rank;
    s->value = 0.0;
    for (int p = 0; p < SEL_NPASS; ++p) s->done[p] = 0u;
    s->cdone = 0u;
    s->count = 0u;
}

// Adds key k's digit of `pass` to the shared histogram when k is valid and
// matches the prefix chosen so far (warp-aggregated); all 32 lanes call it.
__device__ __forceinline__ void sel_count(unsigned *hist, unsigned long long k, bool valid,
                                          unsigned long long pre, int pass) {
    const int shift = sel_shift(pass), top = shift + sel_bits(pass);
    const unsigned mask = (1u << sel_bits(pass)) - 1u;
    unsigned digit = 0xffffffffu;
    if (valid && (top >= 64 || (k >> top) == (pre >> top))) digit = (unsigned)(k >> shift) & mask;
    const unsigned same = __match_any_sync(kFull, digit);
    if (digit != 0xffffffffu && (sel_tid() & 31) == __ffs(same) - 1)
        atomicAdd(&hist[digit], __popc(same));
}

// The end of pass `pass`, called by every thread of every CTA once its
// counts are in the shared `hist`: the non-zero bins go into ghist, and the
// last of the nblk CTAs working on this select to finish (counted in
// s->done[pass]) finds the bin holding s->rank and extends the prefix.
// Block sizes that divide SEL_NB, >= 64.
__device__ __forceinline__ void sel_pass_finish(int pass, SelState *s, unsigned *ghist,
                                                const unsigned *hist, unsigned nblk) {
    __shared__ unsigned wsum[32];
    __shared__ int owner;
    __shared__ unsigned long long owner_excl;
    __shared__ bool last;
    const int t = sel_tid(), nt = sel_nt(), lane = t & 31, wid = t >> 5;
    const int shift = sel_shift(pass);
    for (int i = t; i < SEL_NB; i += nt)
        if (hist[i]) atomicAdd(&ghist[i], hist[i]);
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(&s->done[pass], 1u) == nblk - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last CTA: each thread sums `per` bins, a block scan finds the owner
    const int per = SEL_NB / nt;
    unsigned long long loc = 0;
    for (int j = 0; j < per; ++j) loc += __ldcg(ghist + t * per + j);
    unsigned long long incl = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[wid] = (unsigned)incl;    // at most n < 2^32 keys
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
    const long long rank = s->rank;
    const long long excl = (long long)(wsum[wid] + incl - loc);
    if (rank >= excl && rank < excl + (long long)loc) {
        owner = t;
        owner_excl = (unsigned long long)excl;
    }
    __syncthreads();
    if (t == owner) {
        long long r = rank - (long long)owner_excl;
        int b = t * per;
        for (int j = 0; j < per; ++j) {
            const long long c = __ldcg(ghist + t * per + j);
            if (r < c) {
                b = t * per + j;
                break;
            }
            r -= c;
        }
        s->prefix |= (unsigned long long)b << shift;
        s->rank = r;
        if (pass == SEL_NPASS - 1) s->value = sel_unkey(s->prefix);
    }
}

// ------------------------------------------------------------------
// predict_auto's next work width straight from a map, without the value.
//
// predict_auto only needs the width that its rule (width_for,
// stereonet.py:3915-3919) gives for the map's 95% quantile v*:
//   width(v) = clamp(int(W * target / max(g(v), 1e-6) + 0.5), 48, min(W, max_width)),
//   g(v) = max(v, 0.5) * scale   (scale = W / probe width for the probe, else 1).
// width() is monotone non-increasing in the values' order, so listing the
// map's widths in the order of its values lists them from the widest down,
// and width(v*) is the width at position rank of that list: a histogram of
// the map's widths (one pass, fused into the kernel that writes the map)
// gives it exactly, for every map.  Bin b holds width kmax - b.  NaN values
// count as the largest values, as the order keys of positive NaNs sort
// (bin m, width 48).
struct WidthRule {
    int W, max_width;
    double target, scale;
};

__host__ __device__ inline int width_rule_kmax(const WidthRule &r) {
    const int k = r.W < r.max_width ? r.W : r.max_width;
    return k > 48 ? k : 48;
}

// width_for of the floored (and scaled) value, in FP64 with every operation
// rounded as the host rounds it.
__device__ __forceinline__ int width_rule_of(const WidthRule &r, double v) {
    const double pk = v > 0.5 ? v : 0.5;
    const double peak = __dmul_rn(pk, r.scale);
    const double m = peak > 1.0e-6 ? peak : 1.0e-6;
    const double q = __dadd_rn(__ddiv_rn(__dmul_rn((double)r.W, r.target), m), 0.5);
    int w = q < 2147483647.0 ? (q > -2147483648.0 ? (int)q : -2147483647 - 1) : 2147483647;
    if (w > r.W) w = r.W;
    if (w > r.max_width) w = r.max_width;
    if (w < 48) w = 48;
    return w;
}

// What a fused or standalone width decision needs.
struct WidthFuse {
    WidthRule rule;
    int m, kmax;            // m + 1 bins: widths kmax .. kmax - m (= 48)
    long long rank;         // position of the quantile in the map
};

constexpr int kWidthBins = 2048;         // bins a decision can hold (widths up to 2095)

__device__ __forceinline__ int width_bin_of(const WidthFuse &f, double v) {
    return v != v ? f.m : f.kmax - width_rule_of(f.rule, v);
}

// Adds bin b (b < 0: nothing) to the shared histogram, warp-aggregated; all
// 32 lanes call it.
__device__ __forceinline__ void width_count(unsigned *hist, int b) {
    const unsigned same = __match_any_sync(kFull, (unsigned)b);
    if (b >= 0 && (sel_tid() & 31) == __ffs(same) - 1) atomicAdd(&hist[b], __popc(same));
}

// The width from the decision's totals h[0..m] (whole CTA): the number of
// j < m whose prefix h[0] + .. + h[j] is <= rank, subtracted from kmax.
// G: h in global memory, written by other CTAs (read around L1).
template <bool G>
__device__ __forceinline__ int width_from_bins(const WidthFuse &f, const unsigned *h) {
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned wcnt[32];
    const int t = sel_tid(), nt = sel_nt(), lane = t & 31, wid = t >> 5, nw = nt >> 5;
    const int per = (f.m + nt - 1) / nt, j0 = t * per;
    const int j1 = j0 + per < f.m ? j0 + per : f.m;
    unsigned long long loc = 0;
    for (int j = j0; j < j1; ++j) loc += G ? __ldcg(h + j) : h[j];
    unsigned long long incl = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const unsigned long long v0 = lane < nw ? wsum[lane] : 0ull;
        unsigned long long v = v0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, v, o);
            if (lane >= o) v += y;
        }
        if (lane < nw) wsum[lane] = v - v0;
    }
    __syncthreads();
    unsigned long long run = wsum[wid] + incl - loc;
    unsigned cnt = 0;
    for (int j = j0; j < j1; ++j) {
        run += G ? __ldcg(h + j) : h[j];
        if ((long long)run <= f.rank) ++cnt;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(kFull, cnt, o);
    if (lane == 0) wcnt[wid] = cnt;
    __syncthreads();
    unsigned total = 0;
    for (int w = 0; w < nw; ++w) total += wcnt[w];
    return f.kmax - (int)total;
}

// The end of a CTA's share of a decision: its bins (hist, m + 1 of them) go
// into ghist, and the last of the nblk CTAs turns the totals into the width
// (into s->value, and *mirror when given).  ghist and s->done[0] start at 0.
__device__ __forceinline__ void width_finish(const WidthFuse &f, SelState *s, unsigned *ghist,
                                             const unsigned *hist, unsigned nblk,
                                             double *mirror) {
    __shared__ bool last;
    const int t = sel_tid(), nt = sel_nt();
    for (int i = t; i <= f.m; i += nt)
        if (hist[i]) atomicAdd(&ghist[i], hist[i]);
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(&s->done[0], 1u) == nblk - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int width = width_from_bins<true>(f, ghist);
    if (t == 0) {
        s->value = (double)width;
        if (mirror) *reinterpret_cast<volatile double *>(mirror) = (double)width;
    }
}

}  // namespace sv
