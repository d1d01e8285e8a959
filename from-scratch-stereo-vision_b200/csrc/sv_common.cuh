// sv_common.cuh -- shared helpers for the sm_100a kernels and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>
#include <cstddef>

#include "sv_b200.h"

namespace sv {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kInf = 1 << 29;        // "no candidate" in the integer SGM recurrence
constexpr int kMaxRowW = 16384;      // row kernels keep one image row in shared memory
constexpr int kMaxK = 253;           // band width limit (R <= 126): k fits 8 bits of a WTA key
constexpr int kMaxPenalty = 4096;    // P1, P2 bound: 8 paths x (68 + P2) stays below 2^16

// Thread-local error detail for sv_last_error().
void set_error(const char *fmt, ...);

// Process-wide count of kernels this library has launched (sv_launch_count);
// a relaxed atomic increment per launch, read only for reporting.
void count_launch();
void count_launches(unsigned long long n);     // a graph replay's kernels
void uncount_launches(unsigned long long n);   // kernels recorded, not yet run
unsigned long long launch_count_now();

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Bump allocator over a caller workspace.  With base == nullptr it only
// measures, so sizing and carving share one code path.
struct Carver {
    char *base;
    size_t off = 0;
    explicit Carver(void *b) : base(static_cast<char *>(b)) {}
    template <typename T>
    T *take(size_t count) {
        size_t o = off;
        off = align256(off + count * sizeof(T));
        return base ? reinterpret_cast<T *>(base + o) : nullptr;
    }
};

// Device-side data errors (first error wins), kept at the workspace start.
struct DevFlags {
    int status;
    int pad[63];
};

#define SV_CUDA_TRY(expr)                                                        \
    do {                                                                         \
        cudaError_t e_ = (expr);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            ::sv::set_error("%s failed: %s", #expr, cudaGetErrorString(e_));     \
            return SV_ERR_CUDA;                                                  \
        }                                                                        \
    } while (0)

#define SV_LAUNCH_CHECK()                                                        \
    do {                                                                         \
        cudaError_t e_ = cudaGetLastError();                                     \
        if (e_ != cudaSuccess) {                                                 \
            ::sv::set_error("kernel launch failed: %s", cudaGetErrorString(e_)); \
            return SV_ERR_CUDA;                                                  \
        }                                                                        \
    } while (0)

inline int grid_for(long n, int block, int max_blocks = 148 * 16) {
    long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (int)g;
}

// ---------------------------------------------------------------- device
__device__ __forceinline__ void flag_error(int *flag, int code) {
    atomicCAS(flag, 0, code);
}

// Order-preserving map of a double to uint64 (NaN excluded by the caller).
__device__ __forceinline__ unsigned long long ordkey(double d) {
    long long b = __double_as_longlong(d);
    return b >= 0 ? ((unsigned long long)b | 0x8000000000000000ull)
                  : ~(unsigned long long)b;
}

// Exclusive prefix max over the threads of a block (v from thread t;
// returns max over threads < t, or `ident`).  sbuf: 32 ints of shared memory.
__device__ __forceinline__ int block_excl_max(int v, int ident, int *sbuf) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x = max(x, y);
    }
    if (lane == 31) sbuf[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = lane < nw ? sbuf[lane] : ident;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w = max(w, y);
        }
        sbuf[lane] = w;
    }
    __syncthreads();
    int prefix = wid > 0 ? sbuf[wid - 1] : ident;
    int incl = max(prefix, x);
    int excl = __shfl_up_sync(kFull, incl, 1);
    if (lane == 0) excl = prefix;
    __syncthreads();
    return excl;
}

// Exclusive suffix min over the threads of a block (min over threads > t).
__device__ __forceinline__ int block_excl_min_suffix(int v, int ident, int *sbuf) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_down_sync(kFull, x, o);
        if (lane + o < 32) x = min(x, y);
    }
    if (lane == 0) sbuf[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = lane < nw ? sbuf[lane] : ident;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_down_sync(kFull, w, o);
            if (lane + o < 32) w = min(w, y);
        }
        sbuf[lane] = w;
    }
    __syncthreads();
    int suffix = wid + 1 < nw ? sbuf[wid + 1] : ident;
    int incl = min(suffix, x);
    int excl = __shfl_down_sync(kFull, incl, 1);
    if (lane == 31) excl = suffix;
    __syncthreads();
    return excl;
}

}  // namespace sv
