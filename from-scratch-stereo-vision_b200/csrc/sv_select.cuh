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

}  // namespace sv
