// sv_refine.cu -- full-resolution refinement kernels (sm_100a).
//
// The reference (stereonet.py:5115-5391) refines a network disparity with a
// census transform, Hamming costs in a band of K = 2R+1 disparities around
// round(disp0), 8-path SGM, winner-take-all with a parabola fit, and a
// left-right check.  Everything up to the parabola is integer arithmetic on
// integer-valued doubles in the reference; here it is integer arithmetic
// (uint64 census, uint8 costs, int32 recurrence, uint8/uint16 path costs),
// which is exact.  The parabola, the left-right test and the fills run in
// IEEE FP64 with the reference's operation order (no contraction: the
// explicit __d*_rn intrinsics), so every output bit matches.
//
// Right view.  lr_refine (stereonet.py:5353-5356) refines the mirrored pair.
// Census of a mirrored image is a fixed bit permutation of the unmirrored
// census, the same for both images, so Hamming distances are unchanged; the
// 8 SGM directions map onto themselves under mirroring and S is an integer
// sum.  The right view is therefore computed in place: at right-image pixel x
// the candidate d matches left column x + d, and no mirrored copy is made.

#include "sv_common.cuh"
#include "sv_refine.cuh"

namespace sv {

__constant__ int c_dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1},
                                 {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};

// ------------------------------------------------------------------ base
// base = max(0, int(disp0 + 0.5)), stereonet.py:5256-5259.  Python's int()
// truncates toward zero: __double2int_rz.
__global__ void k_base(const double *__restrict__ disp0, long N,
                       int32_t *__restrict__ base, int *flag) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N;
         i += (long)gridDim.x * blockDim.x) {
        double d = disp0[i];
        int b = 0;
        if (!(fabs(d) < 1073741824.0)) {          // NaN fails too
            flag_error(flag, SV_ERR_DISP);
        } else {
            int v = __double2int_rz(__dadd_rn(d, 0.5));
            b = v > 0 ? v : 0;
        }
        base[i] = b;
    }
}

// ---------------------------------------------------------------- census
// stereonet.py:5115-5142.  One CTA computes a CT_W x CT_H tile from a shared
// copy of the tile plus its clamped halo.  Offsets run dy-major, dx-minor,
// centre skipped; s = 2s + (neighbour < centre), so the first offset lands in
// the top bit, exactly as the reference builds its Python int.
constexpr int CT_W = 32, CT_H = 8;

// The census word of the pixel at ctr (in a tile of CT_W + 2 RX columns)
// with the window fixed at compile time: every offset's bit position is a
// constant, so each neighbour costs a compare and an OR.
template <typename T, int RX, int RY>
__device__ __forceinline__ uint64_t census_bits(const T *ctr) {
    constexpr int SW = CT_W + 2 * RX, WX = 2 * RX + 1;
    constexpr int CENTRE = RY * WX + RX, NB = (2 * RY + 1) * WX - 1;
    const T c = *ctr;
    unsigned half[2] = {0u, 0u};
#pragma unroll
    for (int dy = -RY; dy <= RY; ++dy)
#pragma unroll
        for (int dx = -RX; dx <= RX; ++dx) {
            const int lin = (dy + RY) * WX + dx + RX;
            if (lin == CENTRE) continue;
            const int bit = NB - 1 - (lin > CENTRE ? lin - 1 : lin);
            half[bit >> 5] |= (unsigned)(ctr[dy * SW + dx] < c) << (bit & 31);
        }
    return ((uint64_t)half[1] << 32) | half[0];
}

// One CT_W x CT_H tile starting at (tx0, ty0), called by a whole CTA.
template <typename T>
__device__ __forceinline__ void census_tile(const T *__restrict__ img, int W, int H, int rx,
                                            int ry, uint64_t *__restrict__ out, int tx0,
                                            int ty0, T *tile) {
    const int sw = CT_W + 2 * rx, sh = CT_H + 2 * ry;
    const int tid = threadIdx.y * CT_W + threadIdx.x;
    for (int i = tid; i < sw * sh; i += CT_W * CT_H) {
        int sy = i / sw, sx = i - sy * sw;
        int gy = min(max(ty0 + sy - ry, 0), H - 1);
        int gx = min(max(tx0 + sx - rx, 0), W - 1);
        tile[i] = img[(long)gy * W + gx];
    }
    __syncthreads();
    const int x = tx0 + threadIdx.x, y = ty0 + threadIdx.y;
    if (x >= W || y >= H) return;
    const T *ctr = tile + (threadIdx.y + ry) * sw + threadIdx.x + rx;
    if (rx == 4 && ry == 3) {       // the 9 x 7 window of refine_disparity
        out[(long)y * W + x] = census_bits<T, 4, 3>(ctr);
        return;
    }
    const T c = *ctr;
    uint64_t s = 0;
    for (int dy = -ry; dy <= ry; ++dy) {
        const T *row = ctr + dy * sw;
        for (int dx = -rx; dx <= rx; ++dx) {
            if (dx == 0 && dy == 0) continue;
            s = (s << 1) | (uint64_t)(row[dx] < c);
        }
    }
    out[(long)y * W + x] = s;
}

template <typename T>
__global__ void __launch_bounds__(CT_W *CT_H)
    k_census(const T *__restrict__ img0, const T *__restrict__ img1, int W, int H,
             int rx, int ry, uint64_t *__restrict__ out0, uint64_t *__restrict__ out1) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    census_tile<T>(blockIdx.z ? img1 : img0, W, H, rx, ry, blockIdx.z ? out1 : out0,
                   blockIdx.x * CT_W, blockIdx.y * CT_H, reinterpret_cast<T *>(smem_raw));
}

// ------------------------------------------------------------ band costs
// stereonet.py:5156-5189 with ad_weight = prior_w = 0.  View 0 (left
// reference): candidate d = base[p]-R+k matches right column x-d.  View 1
// (right reference, unmirrored): candidate d matches left column x+d.
__global__ void k_band_costs(const uint64_t *__restrict__ cl,
                             const uint64_t *__restrict__ cr,
                             const int32_t *__restrict__ base0,
                             const int32_t *__restrict__ base1, int W, long N,
                             int R, int K, int invalid, uint8_t *__restrict__ C0,
                             uint8_t *__restrict__ C1) {
    const int view = blockIdx.y;
    const uint64_t *ref = view ? cr : cl;
    const uint64_t *oth = view ? cl : cr;
    const int32_t *base = view ? base1 : base0;
    uint8_t *C = view ? C1 : C0;
    const long total = N * K;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
         i += (long)gridDim.x * blockDim.x) {
        long p = i / K;
        int k = (int)(i - p * K);
        int x = (int)(p % W);
        int d = base[p] - R + k;
        int c = invalid;
        if (view == 0) {
            if (d >= 0 && x - d >= 0) c = __popcll(ref[p] ^ oth[p - d]);
        } else {
            if (d >= 0 && x + d <= W - 1) c = __popcll(ref[p] ^ oth[p + d]);
        }
        C[i] = (uint8_t)c;
    }
}

// ------------------------------------------------------------------- SGM
// stereonet.py:5192-5241.  One warp sweeps one scanline of one direction of
// one view.  Band index k lives at flat position i = lane*V + j + 1 (so
// position 0 stands for k = -1 and position K+1 for k = K); V values per lane
// cover K + 2 <= 32V.  Per pixel:
//   t(k)   = min(Lq(k), Lq(k-1)+P1, Lq(k+1)+P1)        (INF outside 0..K-1)
//   best(k)= min(t(k + shift), mq + P2),  shift = base[p] - base[q]
//   L(k)   = C(k) + best(k) - mq,         mq = min_k Lq(k)
// which is the reference's candidate set: mq+P2 always, the other three only
// where kq, kq-1, kq+1 fall inside the band.  shift is warp-uniform, so the
// re-centring is one warp shuffle (V of them) and only where it is nonzero.
// The path minimum is one redux.sync.
constexpr int SGM_G = 4;   // pixels per prefetch group

template <int V>
__device__ __forceinline__ int pick(const int (&a)[V], int sel) {
    int v = a[0];
#pragma unroll
    for (int u = 1; u < V; ++u) v = (sel == u) ? a[u] : v;
    return v;
}

template <int V>
__device__ __forceinline__ void shift_band(const int (&t)[V], int (&o)[V], int s,
                                           int lane) {
    s = max(-64 * V, min(64 * V, s));
    int qs = s >= 0 ? s / V : -((-s + V - 1) / V);   // floor(s / V)
    int rs = s - qs * V;                              // 0 <= rs < V
#pragma unroll
    for (int j = 0; j < V; ++j) {
        int sel = j + rs, off = qs;
        if (sel >= V) { sel -= V; off += 1; }
        int v = pick<V>(t, sel);
        int src = lane + off;
        int got = __shfl_sync(kFull, v, src & 31);
        o[j] = (src >= 0 && src < 32) ? got : kInf;
    }
}

template <int V, typename LT, bool ADD_S>
__global__ void __launch_bounds__(256)
    k_sgm(const uint8_t *__restrict__ C0, const uint8_t *__restrict__ C1,
          const int32_t *__restrict__ base0, const int32_t *__restrict__ base1,
          int W, int H, int K, int P1, int P2, LT *__restrict__ Lout, int npaths,
          SgmTasks tasks) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
    if (gw >= tasks.start[tasks.nseg]) return;
    int sg = 0;
    while (gw >= tasks.start[sg + 1]) ++sg;
    const int j0 = gw - tasks.start[sg];
    const int view = tasks.view[sg], dir = tasks.dir[sg];
    const int dx = c_dirs[dir][0], dy = c_dirs[dir][1];

    int x0, y0, n;
    if (dy == 0) {
        y0 = j0; x0 = dx > 0 ? 0 : W - 1; n = W;
    } else if (dx == 0) {
        x0 = j0; y0 = dy > 0 ? 0 : H - 1; n = H;
    } else {
        if (j0 < W) {
            x0 = j0; y0 = dy > 0 ? 0 : H - 1;
        } else {
            int i = j0 - W + 1;
            x0 = dx > 0 ? 0 : W - 1;
            y0 = dy > 0 ? i : H - 1 - i;
        }
        int nx = dx > 0 ? W - x0 : x0 + 1;
        int ny = dy > 0 ? H - y0 : y0 + 1;
        n = min(nx, ny);
    }
    const uint8_t *__restrict__ C = view ? C1 : C0;
    const int32_t *__restrict__ base = view ? base1 : base0;
    const long N = (long)W * H;
    LT *__restrict__ Lo = ADD_S ? Lout : Lout + (long)(view * npaths + dir) * N * K;
    const long step = (long)dy * W + dx;
    const long p0 = (long)y0 * W + x0;

    int kk[V];
    bool kv[V];
#pragma unroll
    for (int j = 0; j < V; ++j) {
        kk[j] = lane * V + j - 1;
        kv[j] = (unsigned)kk[j] < (unsigned)K;
    }

    int ca[SGM_G][V], cb2[SGM_G][V], ba[SGM_G], bb[SGM_G];
    auto load = [&](int g, int (&cg)[SGM_G][V], int (&bg)[SGM_G]) {
#pragma unroll
        for (int u = 0; u < SGM_G; ++u) {
            int t = g * SGM_G + u;
            if (t < n) {
                long pp = p0 + t * step;
                bg[u] = __ldg(base + pp);
#pragma unroll
                for (int j = 0; j < V; ++j)
                    cg[u][j] = kv[j] ? (int)__ldg(C + pp * K + kk[j]) : 0;
            }
        }
    };

    int t_[V];
    int mq = 0, bprev = 0;
    auto process = [&](int g, const int (&cg)[SGM_G][V], const int (&bg)[SGM_G]) {
#pragma unroll
        for (int u = 0; u < SGM_G; ++u) {
            const int t = g * SGM_G + u;
            if (t >= n) break;
            const long pp = p0 + t * step;
            int L[V];
            int lmin = kInf;
            if (t == 0) {
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    L[j] = kv[j] ? cg[u][j] : kInf;
                    lmin = min(lmin, L[j]);
                }
            } else {
                const int s = bg[u] - bprev;
                int ts[V];
                if (s == 0) {
#pragma unroll
                    for (int j = 0; j < V; ++j) ts[j] = t_[j];
                } else {
                    shift_band<V>(t_, ts, s, lane);
                }
                const int cap = mq + P2;
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    int best = min(ts[j], cap);
                    L[j] = kv[j] ? cg[u][j] + best - mq : kInf;
                    lmin = min(lmin, L[j]);
                }
            }
            bprev = bg[u];
            mq = (int)__reduce_min_sync(kFull, (unsigned)lmin);
#pragma unroll
            for (int j = 0; j < V; ++j) {
                if (kv[j]) {
                    if (ADD_S) {
                        Lo[pp * K + kk[j]] = (LT)(Lo[pp * K + kk[j]] + L[j]);
                    } else {
                        Lo[pp * K + kk[j]] = (LT)L[j];
                    }
                }
            }
            int up = __shfl_up_sync(kFull, L[V - 1], 1);
            int dn = __shfl_down_sync(kFull, L[0], 1);
            if (lane == 0) up = kInf;
            if (lane == 31) dn = kInf;
#pragma unroll
            for (int j = 0; j < V; ++j) {
                int ln = j > 0 ? L[j - 1] : up;
                int rn = j < V - 1 ? L[j + 1] : dn;
                t_[j] = min(L[j], min(ln, rn) + P1);
            }
        }
    };

    const int ng = (n + SGM_G - 1) / SGM_G;
    load(0, ca, ba);
    for (int g = 0; g < ng; g += 2) {
        if (g + 1 < ng) load(g + 1, cb2, bb);
        process(g, ca, ba);
        if (g + 1 >= ng) break;
        if (g + 2 < ng) load(g + 2, ca, ba);
        process(g + 1, cb2, bb);
    }
}

// --------------------------------------------------------- left_to_right
// stereonet.py:5317-5340, one CTA per row.  Forward warp: the reference keeps
// the first x (in scan order) whose d is the largest value landing on a
// column, with a strict > against the initial -1.0; that is reproduced with
// an atomicMax on the value (signed zeros folded) and an atomicMin on x among
// the maxima, so signed zeros and ties come out bit-identical.  Holes
// (value < 0) take min(nearest filled left, nearest filled right), 1e9
// sentinels, 0.0 when neither exists; within a run of holes the reference's
// in-place update gives every hole that same value.  base of the result is
// written too (the right view's band centre).
// One row, called by a whole CTA; smem_raw holds 13*W bytes, sbuf 32 ints.
__device__ __forceinline__ void l2r_row(const double *__restrict__ row, int W,
                                        double *__restrict__ dr_row,
                                        int32_t *__restrict__ base_row,
                                        unsigned char *smem_raw, int *sbuf,
                                        int32_t *__restrict__ base_l = nullptr,
                                        int *flag = nullptr) {
    unsigned long long *key = reinterpret_cast<unsigned long long *>(smem_raw);
    int *win = reinterpret_cast<int *>(key + W);
    unsigned char *hole = reinterpret_cast<unsigned char *>(win + W);
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        key[x] = 0ull;
        win[x] = INT_MAX;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        double d = row[x];
        int xr = __double2int_rz(__dadd_rn(__dsub_rn((double)x, d), 0.5));
        if (xr >= 0 && xr < W && d > -1.0) atomicMax(&key[xr], ordkey(d == 0.0 ? 0.0 : d));
        if (base_l) {                             // k_base's value for this pixel
            int b = 0;
            if (!(fabs(d) < 1073741824.0)) {
                flag_error(flag, SV_ERR_DISP);
            } else {
                const int v = __double2int_rz(__dadd_rn(d, 0.5));
                b = v > 0 ? v : 0;
            }
            base_l[x] = b;
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        double d = row[x];
        int xr = __double2int_rz(__dadd_rn(__dsub_rn((double)x, d), 0.5));
        if (xr >= 0 && xr < W && d > -1.0 && ordkey(d == 0.0 ? 0.0 : d) == key[xr])
            atomicMin(&win[xr], x);
    }
    __syncthreads();
    double *val = reinterpret_cast<double *>(key);   // reuse: key[x] is dead after this
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        double v = win[x] != INT_MAX ? row[win[x]] : -1.0;
        val[x] = v;
        hole[x] = v < 0.0;
    }
    __syncthreads();
    // nearest non-hole to the left / right of each position
    const int chunk = (W + blockDim.x - 1) / blockDim.x;
    const int xb = min(W, (int)threadIdx.x * chunk), xe = min(W, xb + chunk);
    int lastv = -1, firstv = W;
    for (int x = xb; x < xe; ++x)
        if (!hole[x]) { lastv = x; if (firstv == W) firstv = x; }
    const int carryL = block_excl_max(lastv, -1, sbuf);
    const int carryR = block_excl_min_suffix(firstv, W, sbuf);
    int *nxt = win;   // reuse: win[] is dead after val[]
    __syncthreads();
    int nv = carryR;
    for (int x = xe - 1; x >= xb; --x) {
        nxt[x] = nv;
        if (!hole[x]) nv = x;
    }
    int pv = carryL;
    for (int x = xb; x < xe; ++x) {
        double v = val[x];
        if (hole[x]) {
            double va = pv >= 0 ? val[pv] : 1.0e9;
            double vb = nxt[x] < W ? val[nxt[x]] : 1.0e9;
            double m = va < vb ? va : vb;
            v = m < 1.0e8 ? m : 0.0;
        } else {
            pv = x;
        }
        dr_row[x] = v;
        if (base_row) {
            int b = __double2int_rz(__dadd_rn(v, 0.5));
            base_row[x] = b > 0 ? b : 0;
        }
    }
}

// With base_l, also k_base over the left disparity (the rows it reads).
__global__ void __launch_bounds__(256)
    k_left_to_right(const double *__restrict__ dl, int W, double *__restrict__ dr,
                    int32_t *__restrict__ base_r, int32_t *__restrict__ base_l, int *flag) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int sbuf[32];
    const long r = (long)blockIdx.x * W;
    l2r_row(dl + r, W, dr + r, base_r ? base_r + r : nullptr, smem_raw, sbuf,
            base_l ? base_l + r : nullptr, flag);
}

// ------------------------------------------------------------- LR check
// stereonet.py:5357-5390, one CTA per row.  status from the FP64 values;
// mismatches (2) take disp0; occlusions (1) take min(out of the nearest
// non-occluded pixel left / right), 1e9 sentinels, disp0 when neither exists.
// The fill reads only non-occluded pixels, so order does not matter.
// One row (all pointers at the row start), called by a whole CTA; smem_raw
// holds 13*W bytes, sbuf 32 ints.
__device__ __forceinline__ void lr_row(const double *__restrict__ dl,
                                       const double *__restrict__ drr,
                                       const double *__restrict__ disp0, int W, double tol,
                                       double *__restrict__ out, uint8_t *__restrict__ status,
                                       unsigned char *smem_raw, int *sbuf) {
    double *val = reinterpret_cast<double *>(smem_raw);
    int *nxt = reinterpret_cast<int *>(val + W);
    unsigned char *st = reinterpret_cast<unsigned char *>(nxt + W);
    const long r = 0;
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        double d = dl[r + x];
        int xr = __double2int_rz(__dadd_rn(__dsub_rn((double)x, d), 0.5));
        unsigned char s = 0;
        if (xr < 0 || xr >= W) {
            s = 1;
        } else {
            double e = drr[r + xr];
            if (!(fabs(__dsub_rn(d, e)) <= tol)) s = e > d ? 1 : 2;
        }
        st[x] = s;
        val[x] = s == 2 ? disp0[r + x] : d;
    }
    __syncthreads();
    const int chunk = (W + blockDim.x - 1) / blockDim.x;
    const int xb = min(W, (int)threadIdx.x * chunk), xe = min(W, xb + chunk);
    int lastv = -1, firstv = W;
    for (int x = xb; x < xe; ++x)
        if (st[x] != 1) { lastv = x; if (firstv == W) firstv = x; }
    const int carryL = block_excl_max(lastv, -1, sbuf);
    const int carryR = block_excl_min_suffix(firstv, W, sbuf);
    int nv = carryR;
    for (int x = xe - 1; x >= xb; --x) {
        nxt[x] = nv;
        if (st[x] != 1) nv = x;
    }
    int pv = carryL;
    for (int x = xb; x < xe; ++x) {
        double v = val[x];
        if (st[x] == 1) {
            double va = pv >= 0 ? val[pv] : 1.0e9;
            double vb = nxt[x] < W ? val[nxt[x]] : 1.0e9;
            double m = va < vb ? va : vb;
            v = m < 1.0e8 ? m : disp0[r + x];
        } else {
            pv = x;
        }
        out[r + x] = v;
        status[r + x] = st[x];
    }
}

__global__ void __launch_bounds__(256)
    k_lr_check(const double *__restrict__ dl, const double *__restrict__ drr,
               const double *__restrict__ disp0, int W, double tol,
               double *__restrict__ out, uint8_t *__restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int sbuf[32];
    const long r = (long)blockIdx.x * W;
    lr_row(dl + r, drr + r, disp0 + r, W, tol, out + r, status + r, smem_raw, sbuf);
}

// ====================================================================
// Host launchers
// ====================================================================

int launch_base(const double *disp0, long N, int32_t *base, int *flag,
                cudaStream_t st) {
    count_launch(); k_base<<<grid_for(N, 256), 256, 0, st>>>(disp0, N, base, flag);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_census(const void *img0, const void *img1, int dtype, int W, int H,
                  int rx, int ry, uint64_t *out0, uint64_t *out1, cudaStream_t st) {
    dim3 blk(CT_W, CT_H);
    dim3 grd((W + CT_W - 1) / CT_W, (H + CT_H - 1) / CT_H, img1 ? 2 : 1);
    size_t cells = (size_t)(CT_W + 2 * rx) * (CT_H + 2 * ry);
    switch (dtype) {
    case SV_U8:
        count_launch(); k_census<uint8_t><<<grd, blk, cells * 1, st>>>(
            (const uint8_t *)img0, (const uint8_t *)img1, W, H, rx, ry, out0, out1);
        break;
    case SV_F32:
        count_launch(); k_census<float><<<grd, blk, cells * 4, st>>>(
            (const float *)img0, (const float *)img1, W, H, rx, ry, out0, out1);
        break;
    case SV_F64:
        count_launch(); k_census<double><<<grd, blk, cells * 8, st>>>(
            (const double *)img0, (const double *)img1, W, H, rx, ry, out0, out1);
        break;
    default:
        set_error("unknown image dtype %d", dtype);
        return SV_ERR_PARAM;
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_band_costs(const uint64_t *cl, const uint64_t *cr, const int32_t *base0,
                      const int32_t *base1, int W, int H, int R, int invalid,
                      uint8_t *C0, uint8_t *C1, int nviews, cudaStream_t st) {
    const long N = (long)W * H;
    const int K = 2 * R + 1;
    dim3 grd(grid_for(N * K, 256, 148 * 8), nviews);
    count_launch(); k_band_costs<<<grd, 256, 0, st>>>(cl, cr, base0, base1, W, N, R, K, invalid, C0, C1);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

static int band_vals(int K) { return (K + 2 + 31) / 32; }

template <int V, typename LT, bool ADD>
static int sgm_dispatch_lt(const uint8_t *C0, const uint8_t *C1, const int32_t *b0,
                           const int32_t *b1, int W, int H, int K, int P1, int P2,
                           void *Lout, int npaths, const SgmTasks &tasks,
                           cudaStream_t st) {
    long warps = tasks.start[tasks.nseg];
    int blocks = (int)((warps * 32 + 255) / 256);
    count_launch(); k_sgm<V, LT, ADD><<<blocks, 256, 0, st>>>(C0, C1, b0, b1, W, H, K, P1, P2,
                                              (LT *)Lout, npaths, tasks);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <typename LT, bool ADD>
static int sgm_dispatch(const uint8_t *C0, const uint8_t *C1, const int32_t *b0,
                        const int32_t *b1, int W, int H, int K, int P1, int P2,
                        void *Lout, int npaths, const SgmTasks &tasks, cudaStream_t st) {
    switch (band_vals(K)) {
    case 1: return sgm_dispatch_lt<1, LT, ADD>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, tasks, st);
    case 2: return sgm_dispatch_lt<2, LT, ADD>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, tasks, st);
    case 3:
    case 4: return sgm_dispatch_lt<4, LT, ADD>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, tasks, st);
    default: return sgm_dispatch_lt<8, LT, ADD>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, tasks, st);
    }
}

int launch_sgm_add_path(const uint8_t *C, const int32_t *base, int W, int H, int K,
                        int P1, int P2, int dir, uint16_t *S, cudaStream_t st) {
    SgmTasks t = make_sgm_tasks(W, H, 1, 8, &dir, 1);
    return sgm_dispatch<uint16_t, true>(C, C, base, base, W, H, K, P1, P2, S, 1, t, st);
}

int launch_left_to_right(const double *dl, int W, int H, double *dr, int32_t *base_r,
                         cudaStream_t st, int32_t *base_l, int *flag) {
    size_t smem = (size_t)W * (8 + 4 + 1) + 16;
    if (smem > 48 * 1024)
        SV_CUDA_TRY(cudaFuncSetAttribute(k_left_to_right,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
    count_launch(); k_left_to_right<<<H, 256, smem, st>>>(dl, W, dr, base_r, base_l, flag);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_lr_check(const double *dl, const double *dr, const double *disp0, int W,
                    int H, double tol, double *out, uint8_t *status, cudaStream_t st) {
    size_t smem = (size_t)W * (8 + 4 + 1) + 16;
    if (smem > 48 * 1024)
        SV_CUDA_TRY(cudaFuncSetAttribute(k_lr_check,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
    count_launch(); k_lr_check<<<H, 256, smem, st>>>(dl, dr, disp0, W, tol, out, status);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

// ====================================================================
// Batched lr_refine, front and back: one launch per stage over every pair.
// A block finds its pair (and its row / tile / pixel chunk) in the prefix
// tables of BatchTables and runs the same per-row / per-tile code as the
// single-pair kernels above.
// ====================================================================

__global__ void __launch_bounds__(256) k_b_base(BatchTables t) {
    const int i = batch_find(t.px_blk, t.n, blockIdx.x);
    const BatchPair &P = t.pairs[i];
    const long N = (long)P.W * P.H;
    const long p0 = (long)(blockIdx.x - t.px_blk[i]) * t.px_per_block;
    const long p1 = min(N, p0 + (long)t.px_per_block);
    for (long p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        const double d = P.disp0[p];
        int b = 0;
        if (!(fabs(d) < 1073741824.0)) {
            flag_error(t.flag, SV_ERR_DISP);
        } else {
            const int v = __double2int_rz(__dadd_rn(d, 0.5));
            b = v > 0 ? v : 0;
        }
        P.base0[p] = b;
    }
}

__global__ void __launch_bounds__(256) k_b_left_to_right(BatchTables t) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int sbuf[32];
    const int i = batch_find(t.row_blk, t.n, blockIdx.x);
    const BatchPair &P = t.pairs[i];
    const long r = (long)(blockIdx.x - t.row_blk[i]) * P.W;
    l2r_row(P.disp0 + r, P.W, P.d0r + r, P.base1 + r, smem_raw, sbuf);
}

template <typename T>
__global__ void __launch_bounds__(CT_W *CT_H) k_b_census(BatchTables t) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int i = batch_find(t.tile_blk, t.n, blockIdx.x);
    const BatchPair &P = t.pairs[i];
    const int tiles_x = (P.W + CT_W - 1) / CT_W;
    const int tl = (int)(blockIdx.x - t.tile_blk[i]);
    const int ty = tl / tiles_x, tx = tl - ty * tiles_x;
    census_tile<T>(reinterpret_cast<const T *>(blockIdx.z ? P.right : P.left), P.W, P.H, t.rx,
                   t.ry, blockIdx.z ? P.cen1 : P.cen0, tx * CT_W, ty * CT_H,
                   reinterpret_cast<T *>(smem_raw));
}

__global__ void __launch_bounds__(256) k_b_lr_check(BatchTables t) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int sbuf[32];
    const int i = batch_find(t.row_blk, t.n, blockIdx.x);
    const BatchPair &P = t.pairs[i];
    const long r = (long)(blockIdx.x - t.row_blk[i]) * P.W;
    lr_row(P.dl + r, P.dr + r, P.disp0 + r, P.W, t.tol, P.out + r, P.status + r, smem_raw, sbuf);
}

int launch_batch_front(const BatchTables &t, long long px_blocks, long long rows,
                       long long tiles, cudaStream_t st) {
    count_launch();
    k_b_base<<<(unsigned)px_blocks, 256, 0, st>>>(t);
    const size_t row_smem = (size_t)t.maxW * (8 + 4 + 1) + 16;
    if (row_smem > 48 * 1024)
        SV_CUDA_TRY(cudaFuncSetAttribute(k_b_left_to_right,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)row_smem));
    count_launch();
    k_b_left_to_right<<<(unsigned)rows, 256, row_smem, st>>>(t);
    const size_t cells = (size_t)(CT_W + 2 * t.rx) * (CT_H + 2 * t.ry);
    const dim3 g((unsigned)tiles, 1, 2), blk(CT_W, CT_H);
    count_launch();
    switch (t.dtype) {
    case SV_U8: k_b_census<uint8_t><<<g, blk, cells, st>>>(t); break;
    case SV_F32: k_b_census<float><<<g, blk, cells * 4, st>>>(t); break;
    case SV_F64: k_b_census<double><<<g, blk, cells * 8, st>>>(t); break;
    default: set_error("unknown image dtype %d", t.dtype); return SV_ERR_PARAM;
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_batch_back(const BatchTables &t, long long rows, cudaStream_t st) {
    const size_t row_smem = (size_t)t.maxW * (8 + 4 + 1) + 16;
    if (row_smem > 48 * 1024)
        SV_CUDA_TRY(cudaFuncSetAttribute(k_b_lr_check, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)row_smem));
    count_launch();
    k_b_lr_check<<<(unsigned)rows, 256, row_smem, st>>>(t);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

}  // namespace sv
