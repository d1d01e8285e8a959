// sv_netbatch.cuh -- predict_auto over many pairs without host round trips.
//
// Every pair of a batch carries a NetPair record in device memory.  Its full
// resolution and probe size are fixed; the work size of the next network
// pass is written on the device by the decide kernel of the pass before
// (predict_auto's width rule, stereonet.py:3872-3929), so a whole batch --
// probe, up to `passes` passes, the peaks between them -- is one fixed
// sequence of launches that a CUDA graph can hold.
//
// A batched launch covers the CTAs of every pair back to back: block b
// belongs to pair p when pre[p] <= b < pre[p+1], where pre is a host-built
// prefix of each pair's largest CTA count for that kernel (from its largest
// possible work size).  A CTA reads its pair's current sizes, maps its local
// index onto the tile grid of those sizes and leaves when it falls outside
// (or when the pass does not run for the pair).  Per-pair scratch sits in
// equal slabs `slab` bytes apart, so a kernel is given pair 0's pointers.
#pragma once

#include "sv_common.cuh"
#include "sv_refine.cuh"

namespace sv {

constexpr int kNetTrace = 8;

struct NetPair {
    int W, H;            // full resolution
    int pw, ph;          // probe size
    int Wm, Hm;          // largest work size any pass may use
    int active;          // the current pass runs for this pair
    int work;            // requested work width of the current pass
    int Ww, Hw;          // work size of the current pass
    int native;          // the pass runs at full resolution (no resample either way)
    double inv;          // full / work scale of the current pass (1.0 at native size)
    int ntrace;          // widths chosen so far (predict_auto's trace)
    int trace[kNetTrace];
    double peak;         // the last peak the pair's selects produced
};

struct NetLaunch {
    const long long *pre;     // [n+1] CTA prefix of this launch
    const NetPair *pairs;     // [n]
    int n;
    long long slab;           // bytes between the pairs' scratch slabs
};

// The pair this block belongs to, and the block's index within the pair.
__device__ __forceinline__ int net_pair(const NetLaunch &L, long long &c) {
    const long long b = blockIdx.x;
    const int p = batch_find(L.pre, L.n, b);
    c = b - L.pre[p];
    return p;
}

template <typename T>
__device__ __forceinline__ T *net_slab(T *p0, const NetLaunch &L, int p) {
    if (!p0) return nullptr;
    return reinterpret_cast<T *>(reinterpret_cast<uintptr_t>(p0) + (uintptr_t)((long long)p * L.slab));
}

// FeatureNet's stride-2 output sizes for a work size (conv out = (x-1)/2+1).
__host__ __device__ inline void net_quarter(int Hw, int Ww, int &h1, int &w1, int &h, int &w) {
    h1 = (Hw - 1) / 2 + 1;
    w1 = (Ww - 1) / 2 + 1;
    h = (h1 - 1) / 2 + 1;
    w = (w1 - 1) / 2 + 1;
}

}  // namespace sv
