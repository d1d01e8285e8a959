// sv_select.cu -- _peak (stereonet.py:3866-3869): sorted(disp)[int(n * q)],
// the 95% quantile predict_auto steers the work width with.
//
// Exact selection on order-preserving 64-bit keys of the FP64 values (signed
// zeros share one key: they compare equal in the sort, and a zero peak is
// replaced by 0.5 anyway).
//  Four passes over 16-bit digits from the top.  Pass p is a
//  histogram of digit p over the keys that match the prefix chosen so far
//  (warp-aggregated atomics into a 65536-bin global histogram), followed by
//  a one-CTA parallel scan that picks the bin holding the rank and extends
//  the prefix.  After pass 3 the prefix is the key.

#include "sv_common.cuh"
#include "sv_network.cuh"

namespace sv {

constexpr int SEL_DIGIT = 16;
constexpr int SEL_NB = 1 << SEL_DIGIT;
constexpr int SEL_NPASS = 4;

struct SelState {
    unsigned long long prefix;
    long long rank;
    double value;
};

__device__ __forceinline__ unsigned long long sel_key(double d) {
    return ordkey(d == 0.0 ? 0.0 : d);
}

__device__ __forceinline__ double sel_unkey(unsigned long long k) {
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

// ---------------------------------------------------- large: 16-bit radix
__global__ void k_sel_init(SelState *s, long long rank) {
    s->prefix = 0ull;
    s->rank = rank;
    s->value = 0.0;
}

__global__ void __launch_bounds__(256)
    k_sel_hist16(const double *__restrict__ x, long n, int pass, const SelState *__restrict__ s,
                 unsigned *__restrict__ hist) {
    const int shift = 64 - SEL_DIGIT * (pass + 1);
    const int top = shift + SEL_DIGIT;
    const unsigned long long pre = s->prefix;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i0 = blockIdx.x * (long)blockDim.x; i0 < n; i0 += stride) {
        const long i = i0 + threadIdx.x;
        unsigned digit = 0xffffffffu;
        if (i < n) {
            const unsigned long long k = sel_key(x[i]);
            if (top >= 64 || (k >> top) == (pre >> top))
                digit = (unsigned)(k >> shift) & (SEL_NB - 1);
        }
        const unsigned same = __match_any_sync(kFull, digit);
        if (digit != 0xffffffffu && (threadIdx.x & 31) == __ffs(same) - 1)
            atomicAdd(&hist[digit], (unsigned)__popc(same));
    }
}

// One CTA of 1024 threads, 64 bins each: find the bin holding s->rank.
__global__ void __launch_bounds__(1024)
    k_sel_pick16(const unsigned *__restrict__ hist, int pass, SelState *__restrict__ s) {
    __shared__ unsigned long long warp_tot[32];
    __shared__ long long found[2];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const uint4 *h4 = reinterpret_cast<const uint4 *>(hist) + t * 16;
    unsigned long long loc = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const uint4 v = h4[i];
        loc += (unsigned long long)v.x + v.y + v.z + v.w;
    }
    unsigned long long x = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned long long w = warp_tot[lane], v = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, v, o);
            if (lane >= o) v += y;
        }
        warp_tot[lane] = v - w;                     // exclusive
    }
    __syncthreads();
    const long long rank = s->rank;
    const long long excl = (long long)(warp_tot[wid] + x - loc);
    if (rank >= excl && rank < excl + (long long)loc) {        // exactly one thread
        found[0] = t;
        found[1] = rank - excl;
    }
    __syncthreads();
    // warp 0 finds the bin inside the owner's 64 (two per lane)
    if (wid == 0) {
        const int owner = (int)found[0];
        const long long r = found[1];
        const uint2 c2 = reinterpret_cast<const uint2 *>(hist)[owner * 32 + lane];
        const unsigned long long c = (unsigned long long)c2.x + c2.y;
        unsigned long long inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, inc, o);
            if (lane >= o) inc += y;
        }
        const long long ex = (long long)(inc - c);
        if (r >= ex && r < ex + (long long)c) {
            const long long rr = r - ex;
            const int b = owner * 64 + lane * 2 + (rr < (long long)c2.x ? 0 : 1);
            const int shift = 64 - SEL_DIGIT * (pass + 1);
            s->prefix |= (unsigned long long)b << shift;
            s->rank = rr < (long long)c2.x ? rr : rr - c2.x;
            if (pass == SEL_NPASS - 1) s->value = sel_unkey(s->prefix);
        }
    }
}

int launch_select(const double *x, long n, long long rank, SelState *state, unsigned *hist,
                  cudaStream_t st) {
    SV_CUDA_TRY(cudaMemsetAsync(hist, 0, (size_t)SEL_NPASS * SEL_NB * sizeof(unsigned), st));
    count_launch();
    k_sel_init<<<1, 1, 0, st>>>(state, rank);
    const int blocks = grid_for(n, 256 * 4, 148 * 2);
    for (int p = 0; p < SEL_NPASS; ++p) {
        count_launch();
        k_sel_hist16<<<blocks, 256, 0, st>>>(x, n, p, state, hist + (size_t)p * SEL_NB);
        count_launch();
        k_sel_pick16<<<1, 1024, 0, st>>>(hist + (size_t)p * SEL_NB, p, state);
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

size_t select_state_bytes() { return sizeof(SelState); }
size_t select_value_offset() { return offsetof(SelState, value); }
size_t select_hist_words() { return (size_t)SEL_NPASS * SEL_NB; }

}  // namespace sv
