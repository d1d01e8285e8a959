// sv_post.cu -- the rest of refine_disparity (stereonet.py:5865-5883):
// median_filter (2231-2259), SLIC superpixels (5394-5455) and plane_snap
// (5458-5563), all bit-identical to the reference.
//
// * median: one thread per pixel; the window is clipped at the borders, the
//   result is element n//2 of the stably sorted window (an O(n^2) rank
//   selection that also reproduces the order of equal values, signed zeros
//   included).
// * SLIC assignment: every cluster visits its window twice -- first an
//   atomicMin of the distance's bits per pixel (distances are non-negative
//   doubles, so their bits order like their values), then an atomicMin of the
//   cluster index among the clusters that reached that minimum: the first
//   strict minimum in cluster order, as the reference's loop finds it.
//   Pixels no window covers keep their label, as in the reference.
// * SLIC update: the reference sums each cluster's colours and coordinates
//   over the pixels in index order, in FP64.  When every pixel was covered in
//   the iteration, a cluster's pixels all lie in its window, so one thread
//   per cluster sums its window row by row -- the same order.  If some pixel
//   was not covered, one thread makes the reference's single pass over all
//   pixels instead (a device flag chooses; exact either way).
// * plane_snap: segments' pixel lists in index order (built from the same
//   windows, with the same exact fallback), one CTA per segment for RANSAC
//   (40 trials: planes by one thread in the reference's order, inlier counts
//   by all threads), least squares by one thread over the inliers in order,
//   and the snap.  The reference draws from one xorshift32 stream that runs
//   through the segments; xorshift32 is linear over GF(2), so each segment's
//   starting state is computed directly from the number of earlier segments
//   that drew (3 * trials draws each) by 32x32 bit-matrix powers.

#include <climits>
#include <cmath>

#include "sv_common.cuh"
#include "sv_post.cuh"

namespace sv {

// ================================================================= median
constexpr int kMedMaxR = 3;

__global__ void k_median(const double *__restrict__ in, int W, int H, int r,
                         double *__restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const int y0 = y - r > 0 ? y - r : 0, y1 = y + r < H - 1 ? y + r : H - 1;
    const int x0 = x - r > 0 ? x - r : 0, x1 = x + r < W - 1 ? x + r : W - 1;
    double v[(2 * kMedMaxR + 1) * (2 * kMedMaxR + 1)];
    int n = 0;
    for (int yy = y0; yy <= y1; ++yy)
        for (int xx = x0; xx <= x1; ++xx) v[n++] = in[(long)yy * W + xx];
    const int k = n / 2;
    double res = v[0];
    for (int i = 0; i < n; ++i) {
        int pos = 0;
        for (int j = 0; j < n; ++j) pos += (v[j] < v[i]) || (j < i && v[j] == v[i]);
        if (pos == k) {
            res = v[i];
            break;
        }
    }
    out[(long)y * W + x] = res;
}

int launch_median(const double *in, int W, int H, int radius, int passes, double *out,
                  double *tmp, cudaStream_t st) {
    if (radius < 0 || radius > kMedMaxR || passes < 0) {
        set_error("median_filter: radius %d (0..%d), passes %d", radius, kMedMaxR, passes);
        return SV_ERR_PARAM;
    }
    const long N = (long)W * H;
    if (passes == 0) {
        SV_CUDA_TRY(cudaMemcpyAsync(out, in, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        return SV_OK;
    }
    const dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
    // passes alternate between tmp and out so the last one lands in out
    const double *src = in;
    for (int p = 0; p < passes; ++p) {
        double *dst = ((passes - 1 - p) & 1) ? tmp : out;
        count_launch();
        k_median<<<grd, blk, 0, st>>>(src, W, H, radius, dst);
        src = dst;
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

// =================================================================== SLIC
struct SlicCenter {
    double r, g, b, x, y;
};

__device__ __forceinline__ int4 slic_window(const SlicCenter &c, int step, int W, int H) {
    int x0 = __double2int_rz(c.x) - step, x1 = __double2int_rz(c.x) + step;
    int y0 = __double2int_rz(c.y) - step, y1 = __double2int_rz(c.y) + step;
    if (x0 < 0) x0 = 0;
    if (y0 < 0) y0 = 0;
    if (x1 >= W) x1 = W - 1;
    if (y1 >= H) y1 = H - 1;
    return make_int4(x0, x1, y0, y1);
}

__device__ __forceinline__ double slic_dd(const double *__restrict__ rgb, long i, int xx, int yy,
                                          const SlicCenter &c, double m2) {
    const double a = __dsub_rn(__dmul_rn(rgb[3 * i], 255.0), c.r);
    const double b = __dsub_rn(__dmul_rn(rgb[3 * i + 1], 255.0), c.g);
    const double cc = __dsub_rn(__dmul_rn(rgb[3 * i + 2], 255.0), c.b);
    const double dx = __dsub_rn((double)xx, c.x), dy = __dsub_rn((double)yy, c.y);
    const double col = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(cc, cc));
    return __dadd_rn(col, __dmul_rn(m2, __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy))));
}

__global__ void k_slic_init(const double *__restrict__ rgb, int W, int step, int ncx, int nc,
                            SlicCenter *__restrict__ cs) {
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= nc) return;
    const int cx = step / 2 + (ci % ncx) * step, cy = step / 2 + (ci / ncx) * step;
    const long i = (long)cy * W + cx;
    cs[ci] = {__dmul_rn(rgb[3 * i], 255.0), __dmul_rn(rgb[3 * i + 1], 255.0),
              __dmul_rn(rgb[3 * i + 2], 255.0), (double)cx, (double)cy};
}

__global__ void k_slic_reset(long N, unsigned long long *__restrict__ dist,
                             int *__restrict__ labtmp, int *__restrict__ flag) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i == 0) *flag = 0;
    if (i >= N) return;
    dist[i] = (unsigned long long)__double_as_longlong(1.0e30);
    labtmp[i] = INT_MAX;
}

// pass 0: atomicMin of the distance bits; pass 1: cluster index at the minimum
__global__ void __launch_bounds__(256)
    k_slic_assign(const double *__restrict__ rgb, int W, int H, int step, double m2,
                  const SlicCenter *__restrict__ cs, int pass, unsigned long long *__restrict__ dist,
                  int *__restrict__ labtmp) {
    const int ci = blockIdx.x;
    const SlicCenter c = cs[ci];
    const int4 w = slic_window(c, step, W, H);
    const int ww = w.y - w.x + 1, n = ww * (w.w - w.z + 1);
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int yy = w.z + t / ww, xx = w.x + t % ww;
        const long i = (long)yy * W + xx;
        const unsigned long long dd =
            (unsigned long long)__double_as_longlong(slic_dd(rgb, i, xx, yy, c, m2));
        if (pass == 0) atomicMin(dist + i, dd);
        else if (dd == dist[i]) atomicMin(labtmp + i, ci);
    }
}

__global__ void k_slic_commit(long N, const int *__restrict__ labtmp, int *__restrict__ lab,
                              int *__restrict__ flag) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int l = labtmp[i];
    if (l != INT_MAX) lab[i] = l;
    else atomicExch(flag, 1);                          // not covered: keeps its label
}

// One warp per cluster (window order == index order): the lanes stage 32
// pixels of a window row at a time in shared memory and lane 0 adds the
// cluster's ones in order -- or one thread for everything when some pixel
// was not covered.  win[] keeps the windows of the assignment for the
// segment lists.
constexpr int kUpdWarps = 4;

__global__ void __launch_bounds__(32 * kUpdWarps)
    k_slic_update(const double *__restrict__ rgb, int W, int H, int step, int nc,
                  SlicCenter *__restrict__ cs, const int *__restrict__ lab,
                  const int *__restrict__ flag, int4 *__restrict__ win,
                  double *__restrict__ acc, int cap) {
    __shared__ double sv[kUpdWarps][32][3];
    extern __shared__ __align__(16) unsigned char upd_smem[];   // [warps][cap] staged pixels
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const int ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (*flag) {
        if (blockIdx.x != 0 || threadIdx.x != 0) return;
        for (int k = 0; k < nc; ++k) win[k] = slic_window(cs[k], step, W, H);
        for (int k = 0; k < 6 * nc; ++k) acc[k] = 0.0;
        const long N = (long)W * H;
        for (long i = 0; i < N; ++i) {
            const int l = lab[i];
            if (l < 0) continue;
            double *a = acc + 6 * l;
            a[0] = __dadd_rn(a[0], rgb[3 * i]);
            a[1] = __dadd_rn(a[1], rgb[3 * i + 1]);
            a[2] = __dadd_rn(a[2], rgb[3 * i + 2]);
            a[3] = __dadd_rn(a[3], (double)(i % W));
            a[4] = __dadd_rn(a[4], (double)(i / W));
            a[5] += 1.0;
        }
        for (int k = 0; k < nc; ++k) {
            const double *a = acc + 6 * k;
            if (a[5] != 0.0) {
                const double n = a[5];
                cs[k] = {__dmul_rn(__ddiv_rn(a[0], n), 255.0), __dmul_rn(__ddiv_rn(a[1], n), 255.0),
                         __dmul_rn(__ddiv_rn(a[2], n), 255.0), __ddiv_rn(a[3], n),
                         __ddiv_rn(a[4], n)};
            }
        }
        return;
    }
    if (ci >= nc) return;                              // whole warps leave together
    const int4 w = slic_window(cs[ci], step, W, H);
    if (lane == 0) win[ci] = w;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    long cnt = 0;
    const int ww = w.y - w.x + 1, wn = ww * (w.w - w.z + 1);
    if (wn <= cap) {
        // stage the cluster's pixels, compacted in window (= index) order
        const int nw = blockDim.x >> 5;
        double *cv = reinterpret_cast<double *>(upd_smem) + (size_t)wi * cap * 3;
        int2 *cxy = reinterpret_cast<int2 *>(reinterpret_cast<double *>(upd_smem) +
                                             (size_t)nw * cap * 3) + (size_t)wi * cap;
        int base = 0;
        for (int t0 = 0; t0 < wn; t0 += 4 * 32) {
            int xx[4], yy[4];
            bool ok[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int t = t0 + 32 * u + lane;
                ok[u] = false;
                xx[u] = yy[u] = 0;
                if (t < wn) {
                    yy[u] = w.z + t / ww;
                    xx[u] = w.x + t % ww;
                    ok[u] = lab[(long)yy[u] * W + xx[u]] == ci;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const unsigned m = __ballot_sync(kFull, ok[u]);
                if (ok[u]) {
                    const int pos = base + __popc(m & ((1u << lane) - 1u));
                    const long i = (long)yy[u] * W + xx[u];
                    cv[3 * pos] = rgb[3 * i];
                    cv[3 * pos + 1] = rgb[3 * i + 1];
                    cv[3 * pos + 2] = rgb[3 * i + 2];
                    cxy[pos] = make_int2(xx[u], yy[u]);
                }
                base += __popc(m);
            }
        }
        __syncwarp();
        if (lane == 0) {
            for (int k = 0; k < base; ++k) {
                s0 = __dadd_rn(s0, cv[3 * k]);
                s1 = __dadd_rn(s1, cv[3 * k + 1]);
                s2 = __dadd_rn(s2, cv[3 * k + 2]);
                s3 = __dadd_rn(s3, (double)cxy[k].x);
                s4 = __dadd_rn(s4, (double)cxy[k].y);
            }
            cnt = base;
        }
    } else for (int yy = w.z; yy <= w.w; ++yy) {
        for (int xb = w.x; xb <= w.y; xb += 32) {
            const int xx = xb + lane;
            const long i = (long)yy * W + xx;
            const bool ok = xx <= w.y && lab[i] == ci;
            if (ok) {
                sv[wi][lane][0] = rgb[3 * i];
                sv[wi][lane][1] = rgb[3 * i + 1];
                sv[wi][lane][2] = rgb[3 * i + 2];
            }
            unsigned m = __ballot_sync(kFull, ok);
            __syncwarp();
            if (lane == 0) {
                while (m) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1;
                    s0 = __dadd_rn(s0, sv[wi][b][0]);
                    s1 = __dadd_rn(s1, sv[wi][b][1]);
                    s2 = __dadd_rn(s2, sv[wi][b][2]);
                    s3 = __dadd_rn(s3, (double)(xb + b));
                    s4 = __dadd_rn(s4, (double)yy);
                    ++cnt;
                }
            }
            __syncwarp();
        }
    }
    if (lane == 0 && cnt) {
        const double n = (double)cnt;
        cs[ci] = {__dmul_rn(__ddiv_rn(s0, n), 255.0), __dmul_rn(__ddiv_rn(s1, n), 255.0),
                  __dmul_rn(__ddiv_rn(s2, n), 255.0), __ddiv_rn(s3, n), __ddiv_rn(s4, n)};
    }
}

// ============================================================= plane_snap
// Block-wide exclusive prefix sum of v (blockDim <= 1024); *total gets the sum.
__device__ __forceinline__ int block_excl_sum(int v, int *total, int *sbuf) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sbuf[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < nw ? sbuf[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, s, o);
            if (lane >= o) s += y;
        }
        sbuf[lane] = s;
    }
    __syncthreads();
    const int pre = wid ? sbuf[wid - 1] : 0;
    *total = sbuf[nw - 1];
    __syncthreads();
    return pre + x - v;
}

// Segment sizes (pass 0), then ordered pixel lists and valid counts
// (pass 1), from the windows of the last assignment; the exact single-thread
// path when some pixel was not covered in that assignment.
__global__ void __launch_bounds__(256)
    k_seg_lists(int W, int H, int nseg, const int *__restrict__ lab, const int4 *__restrict__ win,
                const int *__restrict__ flag, int pass, int *__restrict__ count,
                const int *__restrict__ start, int *__restrict__ list,
                const uint8_t *__restrict__ valid, int *__restrict__ nvalid) {
    __shared__ int sbuf[32];
    if (*flag) {
        if (blockIdx.x != 0 || threadIdx.x != 0) return;
        const long N = (long)W * H;
        if (pass == 0) {
            for (int g = 0; g < nseg; ++g) count[g] = 0;
            for (long i = 0; i < N; ++i)
                if (lab[i] >= 0) ++count[lab[i]];
        } else {
            for (int g = 0; g < nseg; ++g) count[g] = nvalid[g] = 0;   // count: fill cursors
            for (long i = 0; i < N; ++i) {
                const int l = lab[i];
                if (l < 0) continue;
                list[start[l] + count[l]++] = (int)i;
                nvalid[l] += valid ? (int)valid[i] : 1;
            }
        }
        return;
    }
    const int g = blockIdx.x;
    const int4 w = win[g];
    const int ww = w.y - w.x + 1, n = ww * (w.w - w.z + 1);
    int base = 0, nv = 0;
    for (int t0 = 0; t0 < n; t0 += blockDim.x) {
        const int t = t0 + threadIdx.x;
        int i = -1;
        if (t < n) {
            i = (w.z + t / ww) * W + w.x + t % ww;
            if (lab[i] != g) i = -1;
        }
        int tot;
        const int pos = block_excl_sum(i >= 0, &tot, sbuf);
        if (pass == 1) {
            if (i >= 0) list[start[g] + base + pos] = i;
            int vt;
            block_excl_sum(i >= 0 && (!valid || valid[i]), &vt, sbuf);
            nv += vt;
        }
        base += tot;
    }
    if (threadIdx.x == 0) {
        if (pass == 0) count[g] = base;
        else nvalid[g] = nv;
    }
}

// Exclusive scan of count[] into start[] (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024)
    k_seg_scan(int nseg, const int *__restrict__ count, int *__restrict__ start) {
    __shared__ int sbuf[32];
    int base = 0;
    for (int g0 = 0; g0 < nseg; g0 += blockDim.x) {
        const int g = g0 + threadIdx.x;
        const int v = g < nseg ? count[g] : 0;
        int tot;
        const int pos = block_excl_sum(v, &tot, sbuf);
        if (g < nseg) start[g] = base + pos;
        base += tot;
    }
    if (threadIdx.x == 0) start[nseg] = base;
}

__device__ __forceinline__ uint32_t xorshift32(uint32_t s) {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return s;
}

// y = A x over GF(2); A as 32 columns (column b = image of bit b)
__device__ __forceinline__ uint32_t gf2_apply(const uint32_t *A, uint32_t x) {
    uint32_t y = 0;
#pragma unroll
    for (int b = 0; b < 32; ++b)
        if ((x >> b) & 1u) y ^= A[b];
    return y;
}

constexpr int kJumpBits = 24;                // up to 2^24 segments

// Starting xorshift32 state of every segment: seed advanced by 3*trials
// draws for each earlier segment with at least 12 valid pixels.  One CTA:
// the jump matrices J_j = M^(3*trials*2^j) by squaring, then a scan of the
// eligibility and one matrix product per set bit of each segment's count.
__global__ void __launch_bounds__(1024)
    k_seg_rng(int nseg, const int *__restrict__ nvalid, int trials, uint32_t seed,
              uint32_t *__restrict__ state) {
    __shared__ uint32_t J[kJumpBits][32];
    __shared__ uint32_t T[2][32];
    __shared__ int sbuf[32];
    const int t = threadIdx.x;
    // M^(3*trials): square-and-multiply on columns (warp 0)
    if (t < 32) {
        T[0][t] = xorshift32(1u << t);                 // M
        T[1][t] = 1u << t;                             // identity (accumulator)
    }
    __syncthreads();
    int e = 3 * trials;
    while (e > 0) {
        uint32_t acc = 0, sq = 0;
        if (t < 32) {
            acc = (e & 1) ? gf2_apply(T[0], T[1][t]) : T[1][t];
            sq = gf2_apply(T[0], T[0][t]);
        }
        __syncthreads();
        if (t < 32) {
            T[1][t] = acc;
            T[0][t] = sq;
        }
        __syncthreads();
        e >>= 1;
    }
    if (t < 32) J[0][t] = T[1][t];
    __syncthreads();
    for (int j = 1; j < kJumpBits; ++j) {
        if (t < 32) J[j][t] = gf2_apply(J[j - 1], J[j - 1][t]);
        __syncthreads();
    }
    int base = 0;
    for (int g0 = 0; g0 < nseg; g0 += blockDim.x) {
        const int g = g0 + t;
        const int nv = g < nseg ? nvalid[g] : 0;
        int tot;
        const int c = base + block_excl_sum(g < nseg && nv >= 12, &tot, sbuf);
        if (g < nseg) {
            uint32_t s = seed;
            for (int j = 0; j < kJumpBits; ++j)
                if ((c >> j) & 1) s = gf2_apply(J[j], s);
            state[g] = s;
        }
        base += tot;
    }
}

// _solve3, stereonet.py:5458-5469 (0 when |det| < 1e-9)
__device__ int solve3_dev(const double A[3][3], const double bv[3], double out[3]) {
    const double a = A[0][0], bb = A[0][1], c = A[0][2];
    const double d = A[1][0], e = A[1][1], f = A[1][2];
    const double g = A[2][0], h = A[2][1], k = A[2][2];
#define M_ __dmul_rn
#define S_ __dsub_rn
#define A_ __dadd_rn
    const double m1 = S_(M_(e, k), M_(f, h)), m2 = S_(M_(d, k), M_(f, g)), m3 = S_(M_(d, h), M_(e, g));
    const double det = A_(S_(M_(a, m1), M_(bb, m2)), M_(c, m3));
    if (fabs(det) < 1.0e-9) return 0;
    const double x = A_(S_(M_(bv[0], m1), M_(bb, S_(M_(bv[1], k), M_(f, bv[2])))),
                        M_(c, S_(M_(bv[1], h), M_(e, bv[2]))));
    const double y = A_(S_(M_(a, S_(M_(bv[1], k), M_(f, bv[2]))), M_(bv[0], m2)),
                        M_(c, S_(M_(d, bv[2]), M_(bv[1], g))));
    const double z = A_(S_(M_(a, S_(M_(e, bv[2]), M_(bv[1], h))),
                           M_(bb, S_(M_(d, bv[2]), M_(bv[1], g)))),
                        M_(bv[0], m3));
    out[0] = __ddiv_rn(x, det);
    out[1] = __ddiv_rn(y, det);
    out[2] = __ddiv_rn(z, det);
    return 1;
}

__device__ __forceinline__ double plane_at(const double *pl, int i, int W) {
    return __dadd_rn(__dadd_rn(__dmul_rn(pl[0], (double)(i % W)), __dmul_rn(pl[1], (double)(i / W))),
                     pl[2]);
}

constexpr int kMaxTrials = 64;
constexpr int kSnapCap = 2048;          // segment points staged in shared memory

// One CTA per segment: RANSAC, least squares over the inliers, snap.  The
// segment's valid points (x, y, d) are staged in shared memory so the
// sequential parts (the draws and planes of thread 0, the ordered
// least-squares sums) read shared memory; segments larger than kSnapCap
// read global memory instead (same values, same order).
__global__ void __launch_bounds__(256)
    k_seg_snap(const double *__restrict__ disp, int W, const uint8_t *__restrict__ valid,
               const int *__restrict__ start, const int *__restrict__ list,
               const int *__restrict__ nvalid, const uint32_t *__restrict__ state, int trials,
               double thr, double min_inl, int *__restrict__ pts, int *__restrict__ inl,
               double *__restrict__ out) {
    __shared__ double planes[kMaxTrials][3];
    __shared__ int ok[kMaxTrials], cnt[kMaxTrials];
    __shared__ int sbuf[32];
    __shared__ int s_best;
    __shared__ double fit[3];
    __shared__ int2 sxy[kSnapCap];
    __shared__ double sdv[kSnapCap];
    __shared__ int sinl[kSnapCap];
    __shared__ int sbuf_draw[3 * kMaxTrials];
    const int g = blockIdx.x, t = threadIdx.x;
    const int s0 = start[g], gn = start[g + 1] - s0;
    if (nvalid[g] < 12) return;
    // valid pixels in index order
    int base = 0;
    for (int k0 = 0; k0 < gn; k0 += blockDim.x) {
        const int k = k0 + t;
        const int i = k < gn ? list[s0 + k] : -1;
        const int take = i >= 0 && (!valid || valid[i]);
        int tot;
        const int pos = block_excl_sum(take, &tot, sbuf);
        if (take) pts[s0 + base + pos] = i;
        base += tot;
    }
    const int n = base;
    const bool staged = n <= kSnapCap;
    __syncthreads();
    if (staged) {
        for (int j = t; j < n; j += blockDim.x) {
            const int i = pts[s0 + j];
            sxy[j] = make_int2(i % W, i / W);
            sdv[j] = disp[i];
        }
    }
    __syncthreads();
    auto P = [&](int j, double &x, double &y, double &d) {
        if (staged) {
            const int2 q = sxy[j];
            x = (double)q.x;
            y = (double)q.y;
            d = sdv[j];
        } else {
            const int i = pts[s0 + j];
            x = (double)(i % W);
            y = (double)(i / W);
            d = disp[i];
        }
    };
    auto resid_ok = [&](const double *pl, int j) {
        double x, y, d;
        P(j, x, y, d);
        const double v = __dadd_rn(__dadd_rn(__dmul_rn(pl[0], x), __dmul_rn(pl[1], y)), pl[2]);
        return fabs(__dsub_rn(v, d)) <= thr;
    };
    // the draws are one sequential stream (thread 0); the planes are not
    if (t == 0) {
        uint32_t s = state[g];
        for (int k = 0; k < 3 * trials; ++k) {
            s = xorshift32(s);
            sbuf_draw[k] = (int)(s % (uint32_t)n);
        }
    }
    __syncthreads();
    if (t < trials) {
        double A[3][3], bv[3];
        for (int u = 0; u < 3; ++u) {
            P(sbuf_draw[3 * t + u], A[u][0], A[u][1], bv[u]);
            A[u][2] = 1.0;
        }
        ok[t] = solve3_dev(A, bv, planes[t]);
        cnt[t] = 0;
    }
    __syncthreads();
    for (long q = t; q < (long)trials * n; q += blockDim.x) {
        const int tr = (int)(q / n), j = (int)(q - (long)tr * n);
        if (ok[tr] && resid_ok(planes[tr], j)) atomicAdd(&cnt[tr], 1);
    }
    __syncthreads();
    if (t == 0) {
        int best = -1, bestc = -1;
        for (int tr = 0; tr < trials; ++tr)
            if (ok[tr] && cnt[tr] > bestc) {
                bestc = cnt[tr];
                best = tr;
            }
        s_best = (best < 0 || (double)bestc < __dmul_rn(min_inl, (double)n)) ? -1 : best;
    }
    __syncthreads();
    const int best = s_best;
    if (best < 0) return;
    base = 0;
    for (int k0 = 0; k0 < n; k0 += blockDim.x) {
        const int k = k0 + t;
        const int take = k < n && resid_ok(planes[best], k);
        int tot;
        const int pos = block_excl_sum(take, &tot, sbuf);
        if (take) {
            if (staged) sinl[base + pos] = k;
            else inl[s0 + base + pos] = k;
        }
        base += tot;
    }
    __syncthreads();
    if (t == 0) {
        // _lsq_plane, stereonet.py:5472-5502: sums in inlier order
        const int ni = base;
        const double nn = (double)ni;
        double sx = 0.0, sy = 0.0, sd = 0.0, x, y, d;
        for (int k = 0; k < ni; ++k) {
            P(staged ? sinl[k] : inl[s0 + k], x, y, d);
            sx = __dadd_rn(sx, x);
        }
        for (int k = 0; k < ni; ++k) {
            P(staged ? sinl[k] : inl[s0 + k], x, y, d);
            sy = __dadd_rn(sy, y);
        }
        for (int k = 0; k < ni; ++k) {
            P(staged ? sinl[k] : inl[s0 + k], x, y, d);
            sd = __dadd_rn(sd, d);
        }
        const double mx = __ddiv_rn(sx, nn), my = __ddiv_rn(sy, nn), md = __ddiv_rn(sd, nn);
        double sxx = 0.0, sxy_ = 0.0, syy = 0.0, sxd = 0.0, syd = 0.0;
        for (int k = 0; k < ni; ++k) {
            P(staged ? sinl[k] : inl[s0 + k], x, y, d);
            const double u = __dsub_rn(x, mx), v = __dsub_rn(y, my), w = __dsub_rn(d, md);
            sxx = __dadd_rn(sxx, __dmul_rn(u, u));
            sxy_ = __dadd_rn(sxy_, __dmul_rn(u, v));
            syy = __dadd_rn(syy, __dmul_rn(v, v));
            sxd = __dadd_rn(sxd, __dmul_rn(u, w));
            syd = __dadd_rn(syd, __dmul_rn(v, w));
        }
        const double det = __dsub_rn(__dmul_rn(sxx, syy), __dmul_rn(sxy_, sxy_));
        if (fabs(det) < 1.0e-9) {
            fit[0] = 0.0;
            fit[1] = 0.0;
            fit[2] = md;
        } else {
            const double a = __ddiv_rn(__dsub_rn(__dmul_rn(sxd, syy), __dmul_rn(syd, sxy_)), det);
            const double b = __ddiv_rn(__dsub_rn(__dmul_rn(syd, sxx), __dmul_rn(sxd, sxy_)), det);
            fit[0] = a;
            fit[1] = b;
            fit[2] = __dsub_rn(__dsub_rn(md, __dmul_rn(a, mx)), __dmul_rn(b, my));
        }
    }
    __syncthreads();
    for (int k = t; k < gn; k += blockDim.x) {
        const int i = list[s0 + k];
        const double v = plane_at(fit, i, W);
        if (fabs(__dsub_rn(v, disp[i])) <= thr || (valid && !valid[i])) out[i] = v > 0.0 ? v : 0.0;
    }
#undef M_
#undef S_
#undef A_
}

__global__ void k_status_valid(long N, const uint8_t *__restrict__ status,
                               uint8_t *__restrict__ valid) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < N) valid[i] = status[i] == 0;
}

// ------------------------------------------------------------ host side
int slic_grid(int W, int H, int step, int *ncx, int *ncy) {
    int a = 0, b = 0;
    for (int x = step / 2; x < W; x += step) ++a;
    for (int y = step / 2; y < H; y += step) ++b;
    *ncx = a;
    *ncy = b;
    return a * b;
}

double slic_m2(double compactness, int step) {
    // the reference's (compactness / step) ** 2 is CPython's float power,
    // i.e. the C library's pow(); a volatile exponent keeps the compiler
    // from replacing the call by a multiplication
    volatile double two = 2.0;
    return std::pow(compactness / step, (double)two);
}

size_t carve_post(void *ws, int W, int H, int step, PostWs *o) {
    Carver cv(ws);
    PostWs p{};
    const long N = (long)W * H;
    int ncx, ncy;
    const int nc = slic_grid(W, H, step, &ncx, &ncy);
    const int nca = nc > 0 ? nc : 1;
    p.flags = cv.take<DevFlags>(1);
    p.cs = cv.take<unsigned char>(sizeof(SlicCenter) * nca);
    p.win = cv.take<int4>(nca);
    p.acc = cv.take<double>(6 * (size_t)nca);
    p.dist = cv.take<unsigned long long>(N);
    p.labtmp = cv.take<int>(N);
    p.lab = cv.take<int>(N);
    p.flag = cv.take<int>(4);
    p.count = cv.take<int>(nca);
    p.start = cv.take<int>(nca + 1);
    p.list = cv.take<int>(N);
    p.pts = cv.take<int>(N);
    p.inl = cv.take<int>(N);
    p.nvalid = cv.take<int>(nca);
    p.state = cv.take<uint32_t>(nca);
    p.valid = cv.take<uint8_t>(N);
    p.tmp = cv.take<double>(N);
    if (o) *o = p;
    return cv.off;
}

int launch_slic(const double *rgb, int W, int H, int step, double compactness, int iters,
                const PostWs &w, cudaStream_t st) {
    if (W < 1 || H < 1 || step < 1 || iters < 0) {
        set_error("slic: bad shape or step");
        return SV_ERR_PARAM;
    }
    int ncx, ncy;
    const int nc = slic_grid(W, H, step, &ncx, &ncy);
    const long N = (long)W * H;
    const double m2 = slic_m2(compactness, step);
    SlicCenter *cs = reinterpret_cast<SlicCenter *>(w.cs);
    SV_CUDA_TRY(cudaMemsetAsync(w.lab, 0xFF, sizeof(int) * N, st));       // -1
    SV_CUDA_TRY(cudaMemsetAsync(w.flag, 0, sizeof(int) * 4, st));
    if (nc == 0) return SV_OK;
    count_launch();
    k_slic_init<<<(nc + 127) / 128, 128, 0, st>>>(rgb, W, step, ncx, nc, cs);
    const int nb = grid_for(N, 256, 1 << 30);
    // SLIC update staging: (2 step + 1)^2 pixels of 32 bytes per warp
    const long wmax = (long)(2 * step + 1) * (2 * step + 1);
    // within the 48 KB default, next to the kernel's 3 KB of static shared memory
    const int wpb0 = (int)((44l * 1024) / (wmax * 32));
    const int wpb = wpb0 < 1 ? kUpdWarps : (wpb0 > kUpdWarps ? kUpdWarps : wpb0);
    const int cap = wpb0 < 1 ? 0 : (int)wmax;
    for (int it = 0; it < iters; ++it) {
        count_launch();
        k_slic_reset<<<nb, 256, 0, st>>>(N, w.dist, w.labtmp, w.flag);
        count_launch();
        k_slic_assign<<<nc, 256, 0, st>>>(rgb, W, H, step, m2, cs, 0, w.dist, w.labtmp);
        count_launch();
        k_slic_assign<<<nc, 256, 0, st>>>(rgb, W, H, step, m2, cs, 1, w.dist, w.labtmp);
        count_launch();
        k_slic_commit<<<nb, 256, 0, st>>>(N, w.labtmp, w.lab, w.flag);
        count_launch();
        k_slic_update<<<(nc + wpb - 1) / wpb, 32 * wpb, (size_t)wpb * cap * 32, st>>>(
            rgb, W, H, step, nc, cs, w.lab, w.flag, w.win, w.acc, cap);
    }
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_plane_snap(const double *disp, const double *rgb, int W, int H, const uint8_t *valid,
                      int step, double thr, double min_inl, int trials, uint32_t seed,
                      double *out, const PostWs &w, cudaStream_t st) {
    if (trials < 0 || trials > kMaxTrials) {
        set_error("plane_snap: trials %d outside 0..%d", trials, kMaxTrials);
        return SV_ERR_PARAM;
    }
    const long N = (long)W * H;
    SV_CUDA_TRY(cudaMemcpyAsync(out, disp, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    int ncx, ncy;
    const int nc = slic_grid(W, H, step, &ncx, &ncy);
    SV_TRY_POST(launch_slic(rgb, W, H, step, 10.0, 5, w, st));
    if (nc == 0 || trials == 0) return SV_OK;
    count_launch();
    k_seg_lists<<<nc, 256, 0, st>>>(W, H, nc, w.lab, w.win, w.flag, 0, w.count, w.start, w.list,
                                    valid, w.nvalid);
    count_launch();
    k_seg_scan<<<1, 1024, 0, st>>>(nc, w.count, w.start);
    count_launch();
    k_seg_lists<<<nc, 256, 0, st>>>(W, H, nc, w.lab, w.win, w.flag, 1, w.count, w.start, w.list,
                                    valid, w.nvalid);
    count_launch();
    k_seg_rng<<<1, 1024, 0, st>>>(nc, w.nvalid, trials, seed, w.state);
    count_launch();
    k_seg_snap<<<nc, 256, 0, st>>>(disp, W, valid, w.start, w.list, w.nvalid, w.state, trials,
                                   thr, min_inl, w.pts, w.inl, out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_status_valid(const uint8_t *status, long N, uint8_t *valid, cudaStream_t st) {
    count_launch();
    k_status_valid<<<grid_for(N, 256, 1 << 30), 256, 0, st>>>(N, status, valid);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

}  // namespace sv

namespace sv {

// ====================================== network-level LR consistency
// mirror_h (stereonet.py:4974-4983) of one [H][W] plane of esize-byte values
__global__ void k_mirror(const unsigned char *__restrict__ in, int esize, int W, int H,
                         unsigned char *__restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H) return;
    const long src = ((long)y * W + (W - 1 - x)) * esize, dst = ((long)y * W + x) * esize;
    for (int b = 0; b < esize; ++b) out[dst + b] = in[src + b];
}

// lr_consistency, stereonet.py:4986-5009 (FP64, the reference's order)
__global__ void k_lr_consistency(const double *__restrict__ dl, const double *__restrict__ dr,
                                 int W, int H, double tol, uint8_t *__restrict__ valid,
                                 unsigned long long *__restrict__ kept) {
    const long N = (long)W * H;
    const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
    int ok = 0;
    if (p < N) {
        const int x = (int)(p % W);
        const long row = p - x;
        const double d = dl[p];
        const double xr = __dsub_rn((double)x, d);
        ok = 1;
        if (xr < 0.0 || xr > (double)(W - 1)) {
            ok = 0;
        } else {
            const int x0 = __double2int_rz(xr);
            const int x1 = x0 + 1 < W ? x0 + 1 : x0;
            const double f = __dsub_rn(xr, (double)x0);
            const double e = __dadd_rn(__dmul_rn(dr[row + x0], __dsub_rn(1.0, f)),
                                       __dmul_rn(dr[row + x1], f));
            double diff = __dsub_rn(d, e);
            if (diff < 0.0) diff = -diff;
            if (diff > tol) ok = 0;
        }
        valid[p] = (uint8_t)ok;
    }
    unsigned c = __popc(__ballot_sync(kFull, ok));
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(kept, (unsigned long long)c);
}

// fill_invalid, stereonet.py:5012-5045: one CTA per row.  Pass 1 records the
// nearest valid column to the left of each pixel (chunked block scans),
// pass 2 walks from the right with the nearest valid column to the right
// and fills.
__global__ void __launch_bounds__(1024)
    k_fill_invalid(const double *__restrict__ disp, const uint8_t *__restrict__ valid, int W,
                   int H, int *__restrict__ left_idx, double *__restrict__ out) {
    __shared__ int sbuf[32];
    __shared__ int carry;
    const int y = blockIdx.x, t = threadIdx.x, bd = blockDim.x;
    const long row = (long)y * W;
    if (t == 0) carry = -1;
    __syncthreads();
    for (int c0 = 0; c0 < W; c0 += bd) {
        const int x = c0 + t;
        const int v = x < W && valid[row + x] ? x : -1;
        const int ex = block_excl_max(v, -1, sbuf);
        const int c = carry;
        if (x < W) left_idx[row + x] = max(c, ex);
        __syncthreads();
        if (t == bd - 1) carry = max(c, max(ex, v));
        __syncthreads();
    }
    if (t == 0) carry = W;
    __syncthreads();
    const int nch = (W + bd - 1) / bd;
    for (int ci = nch - 1; ci >= 0; --ci) {
        const int x = ci * bd + t;
        const int v = x < W && valid[row + x] ? x : W;
        const int ex = block_excl_min_suffix(v, W, sbuf);
        const int c = carry;
        if (x < W) {
            double r = disp[row + x];
            if (!valid[row + x]) {
                const int lf = left_idx[row + x], rt = min(c, ex);
                const bool hl = lf >= 0, hr = rt < W;
                if (hl && hr) {
                    const double lv = disp[row + lf], rv = disp[row + rt];
                    r = lv < rv ? lv : rv;
                } else if (hl) {
                    r = disp[row + lf];
                } else if (hr) {
                    r = disp[row + rt];
                }
            }
            out[row + x] = r;
        }
        __syncthreads();
        if (t == 0) carry = min(c, min(ex, v));
        __syncthreads();
    }
}

int launch_mirror(const void *in, int esize, int W, int H, void *out, cudaStream_t st) {
    count_launch();
    k_mirror<<<dim3((W + 255) / 256, H), 256, 0, st>>>((const unsigned char *)in, esize, W, H,
                                                       (unsigned char *)out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_lr_consistency(const double *dl, const double *dr, int W, int H, double tol,
                          uint8_t *valid, unsigned long long *kept, cudaStream_t st) {
    SV_CUDA_TRY(cudaMemsetAsync(kept, 0, sizeof(unsigned long long), st));
    const long N = (long)W * H;
    count_launch();
    k_lr_consistency<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(dl, dr, W, H, tol, valid, kept);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_fill_invalid(const double *disp, const uint8_t *valid, int W, int H, int *scratch,
                        double *out, cudaStream_t st) {
    count_launch();
    const int bd = W >= 1024 ? 1024 : (W + 31) / 32 * 32;
    k_fill_invalid<<<H, bd, 0, st>>>(disp, valid, W, H, scratch, out);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

}  // namespace sv
