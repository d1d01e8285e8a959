// sv_sgm.cu -- the band costs, 8-path SGM and winner-take-all of the fused
// refinement (refine_fullres / lr_refine), on a slot layout built for packed
// 16-bit SIMD.
//
// Slot layout.  Each pixel owns Kp bytes (Kp = K+2 rounded up to a table
// size, a multiple of 8); slot i holds band index k = i-1, so slot 0 is
// k = -1, slots 1..K the band and the rest padding.  The padding makes every
// pixel's row 8-byte aligned and gives the SGM recurrence room for the
// candidates just outside the band.
//
// SGM (stereonet.py:5192-5241).  A group of LP lanes (4..32) sweeps one
// scanline of one direction of one view; each lane holds S = Kp/LP slots as
// NR = S/2 registers of two uint16 values (u16x2).  Per pixel:
//   t(k)    = min(Lq(k), Lq(k-1) + P1, Lq(k+1) + P1)   -- byte_perm + vimin3
//   best(k) = min(t(k + shift), mq + P2)                 -- vminu2
//   L(k)    = C(k) + best(k) - mq                         -- 32-bit adds
// with INF (0x7FFF) outside 0..K-1, which is exactly the reference's set of
// candidates (mq + P2 always; the other three only inside the band).  No
// lane ever carries across the 16-bit boundary: L <= nbits + 4 + P2 <= 4164
// and INF + P1 < 0x10000.  mq, the path minimum of the predecessor, is a
// min over the group (log2 LP xor-shuffles).  A nonzero shift (band
// re-centring between neighbours, stereonet.py:5218) goes through a per-group
// shared-memory copy of t; shift 0 (most pixels) costs nothing.
//
// WTA (stereonet.py:5271-5303).  One thread per pixel sums the 8 path arrays
// 8 slots at a time (64-bit loads, byte -> u16x2 expansion), keeps the first
// minimum (strict <, ascending k) and re-reads the two neighbours of the
// winner for the FP64 parabola.

#include <cstdlib>
#include <cstring>

#include "sv_common.cuh"
#include "sv_refine.cuh"

namespace sv {

constexpr unsigned kInf2 = 0x7FFF7FFFu;

__device__ __forceinline__ void dir_of(int d, int &dx, int &dy) {
    // order of refine_fullres's dirs list (stereonet.py:5266-5268)
    dx = (d == 0 || d == 4 || d == 6) ? 1 : (d == 2 || d == 3) ? 0 : -1;
    dy = (d == 0 || d == 1) ? 0 : (d == 2 || d == 4 || d == 5) ? 1 : -1;
}

// ----------------------------------------------------------- band costs
// The Kp slots of pixel p (slot 0 and padding are 0).  KPC / KC > 0 fix Kp
// and K at compile time (the loops unroll, the band tests fold).
template <int KPC = 0, int KC = 0>
__device__ __forceinline__ void cost_pixel_slot(const uint64_t *__restrict__ ref,
                                                const uint64_t *__restrict__ oth,
                                                const int32_t *__restrict__ base, int W, long p,
                                                int R, int K, int Kp, int invalid, int view,
                                                uint8_t *__restrict__ C, int rk) {
    const int kp = KPC > 0 ? KPC : Kp;
    const int kk = KC > 0 ? KC : K;
    const int x = p <= 0x7fffffffL ? (int)p % W : (int)(p % W);
    const uint64_t a = ref[p];
    const int b = base[p] - R;
    uint64_t *dst = reinterpret_cast<uint64_t *>(C + p * kp);
#pragma unroll
    for (int c = 0; c < kp; c += 8) {
        unsigned half[2] = {0u, 0u};
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int k = c + u - 1;
            unsigned v = 0;
            if (k >= 0 && k < kk) {
                const int d = b + k;
                int cost = invalid;
                if (abs(k - R) > rk) {
                } else if (view == 0) {
                    if (d >= 0 && x - d >= 0) cost = __popcll(a ^ oth[p - d]);
                } else {
                    if (d >= 0 && x + d <= W - 1) cost = __popcll(a ^ oth[p + d]);
                }
                v = (unsigned)cost;
            }
            half[u >> 2] |= v << (8 * (u & 3));
        }
        dst[c >> 3] = ((uint64_t)half[1] << 32) | half[0];
    }
}

// One thread per pixel writes its Kp slots.
template <int KPC, int KC>
__global__ void __launch_bounds__(256)
    k_band_costs_slot(const uint64_t *__restrict__ cl, const uint64_t *__restrict__ cr,
                      const int32_t *__restrict__ base0, const int32_t *__restrict__ base1, int W,
                      long N, int R, int K, int Kp, int invalid, uint8_t *__restrict__ C0,
                      uint8_t *__restrict__ C1, const uint8_t *__restrict__ rad0) {
    const int view = blockIdx.y;
    const uint64_t *ref = view ? cr : cl;
    const uint64_t *oth = view ? cl : cr;
    const int32_t *base = view ? base1 : base0;
    uint8_t *C = view ? C1 : C0;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < N;
         p += (long)gridDim.x * blockDim.x)
        cost_pixel_slot<KPC, KC>(ref, oth, base, W, p, R, K, Kp, invalid, view, C,
                                 view == 0 && rad0 ? (int)rad0[p] : R);
}

// ------------------------------------------------------------------ SGM
constexpr int SGM_PF = 8;   // prefetch distance in pixels

template <int NR, int LP, typename LT>
__global__ void __launch_bounds__(256)
    k_sgm_packed(const uint8_t *__restrict__ C0, const uint8_t *__restrict__ C1,
                 const int32_t *__restrict__ base0, const int32_t *__restrict__ base1, int W,
                 int H, int K, int Kp, int P1, int P2, LT *__restrict__ Lout, int npaths,
                 SgmTasks tasks) {
    constexpr int S = 2 * NR;
    extern __shared__ __align__(16) unsigned char sgm_smem[];
    const int lane = threadIdx.x & 31;
    const int g = lane & (LP - 1);
    const unsigned gmask = LP == 32 ? 0xffffffffu : (((1u << LP) - 1u) << (lane & ~(LP - 1)));
    const long gid = (blockIdx.x * (long)blockDim.x + threadIdx.x) / LP;
    if (gid >= tasks.start[tasks.nseg]) return;            // whole groups leave together
    unsigned short *buf = reinterpret_cast<unsigned short *>(sgm_smem) + (threadIdx.x / LP) * Kp;

    int sg = 0;
    while (gid >= tasks.start[sg + 1]) ++sg;
    const int j0 = (int)(gid - tasks.start[sg]);
    const int view = tasks.view[sg], dir = tasks.dir[sg];
    int dx, dy;
    dir_of(dir, dx, dy);
    int x0, y0, n;
    if (dy == 0) {
        y0 = j0; x0 = dx > 0 ? 0 : W - 1; n = W;
    } else if (dx == 0) {
        x0 = j0; y0 = dy > 0 ? 0 : H - 1; n = H;
    } else {
        if (j0 < W) {
            x0 = j0; y0 = dy > 0 ? 0 : H - 1;
        } else {
            const int i = j0 - W + 1;
            x0 = dx > 0 ? 0 : W - 1;
            y0 = dy > 0 ? i : H - 1 - i;
        }
        n = min(dx > 0 ? W - x0 : x0 + 1, dy > 0 ? H - y0 : y0 + 1);
    }
    const uint8_t *__restrict__ C = view ? C1 : C0;
    const int32_t *__restrict__ base = view ? base1 : base0;
    const long N = (long)W * H;
    LT *__restrict__ Lo = Lout + (long)(view * npaths + dir) * N * Kp;
    const long step = (long)dy * W + dx;
    const long p0 = (long)y0 * W + x0;
    const int s0 = g * S;                                  // first slot of this lane

    unsigned vm[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const int sa = s0 + 2 * r, sb = sa + 1;
        vm[r] = ((sa >= 1 && sa <= K) ? 0x0000FFFFu : 0u) | ((sb >= 1 && sb <= K) ? 0xFFFF0000u : 0u);
    }
    const unsigned P1P1 = (unsigned)P1 * 0x10001u;

    // Prefetch ring: the costs and band centre of step t + SGM_PF are loaded
    // as soon as step t has read its slot, so every load has SGM_PF steps of
    // recurrence latency to arrive from L2.
    unsigned cring[SGM_PF][NR];
    int bring[SGM_PF];
    auto load = [&](int t, int slot) {
        const long pp = p0 + t * step;
        bring[slot] = __ldg(base + pp);
        const unsigned short *cp = reinterpret_cast<const unsigned short *>(C + pp * Kp + s0);
#pragma unroll
        for (int r = 0; r < NR; ++r) cring[slot][r] = (unsigned)__ldg(cp + r);
    };
#pragma unroll
    for (int u = 0; u < SGM_PF; ++u)
        if (u < n) load(u, u);

    unsigned t_[NR];
    int mq = 0, bprev = 0;
    for (int t0 = 0; t0 < n; t0 += SGM_PF) {
#pragma unroll
        for (int u = 0; u < SGM_PF; ++u) {
            const int t = t0 + u;
            if (t >= n) break;                                  // group-uniform
            unsigned c[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) c[r] = __byte_perm(cring[u][r], 0, 0x4140);
            const int bcur = bring[u];
            if (t + SGM_PF < n) load(t + SGM_PF, u);
            const long pp = p0 + t * step;
            unsigned L[NR];
            if (t == 0) {
#pragma unroll
                for (int r = 0; r < NR; ++r) L[r] = (c[r] & vm[r]) | (kInf2 & ~vm[r]);
            } else {
                const int s = bcur - bprev;                     // group-uniform
                unsigned ts[NR];
                if (s == 0) {
#pragma unroll
                    for (int r = 0; r < NR; ++r) ts[r] = t_[r];
                } else if (s == 1 || s == -1) {
                    // one-slot re-centring with two lanes' edge registers
                    unsigned tup = __shfl_up_sync(gmask, t_[NR - 1], 1, LP);
                    unsigned tdn = __shfl_down_sync(gmask, t_[0], 1, LP);
                    if (g == 0) tup = kInf2;
                    if (g == LP - 1) tdn = kInf2;
                    if (s == 1) {
#pragma unroll
                        for (int r = 0; r < NR; ++r)
                            ts[r] = __byte_perm(t_[r], r < NR - 1 ? t_[r + 1] : tdn, 0x5432);
                    } else {
#pragma unroll
                        for (int r = 0; r < NR; ++r)
                            ts[r] = __byte_perm(r > 0 ? t_[r - 1] : tup, t_[r], 0x5432);
                    }
                } else {
                    // larger jumps (depth edges): through this group's shared copy
                    const int sc = max(-Kp - 2, min(Kp + 2, s));
                    unsigned *b32 = reinterpret_cast<unsigned *>(buf);
#pragma unroll
                    for (int r = 0; r < NR; ++r) b32[(s0 >> 1) + r] = t_[r];
                    __syncwarp(gmask);
#pragma unroll
                    for (int r = 0; r < NR; ++r) {
                        const int ia = s0 + 2 * r + sc, ib = ia + 1;
                        const unsigned lo = (ia >= 0 && ia < Kp) ? buf[ia] : 0x7FFFu;
                        const unsigned hi = (ib >= 0 && ib < Kp) ? buf[ib] : 0x7FFFu;
                        ts[r] = lo | (hi << 16);
                    }
                    __syncwarp(gmask);
                }
                const unsigned cap = (unsigned)(mq + P2) * 0x10001u;
                const unsigned mm = (unsigned)mq * 0x10001u;
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    const unsigned v = c[r] + __vminu2(ts[r], cap) - mm;
                    L[r] = (v & vm[r]) | (kInf2 & ~vm[r]);
                }
            }
            bprev = bcur;
            // path minimum over the group
            unsigned m2 = L[0];
#pragma unroll
            for (int r = 1; r < NR; ++r) m2 = __vminu2(m2, L[r]);
            int m = (int)min(m2 & 0xFFFFu, m2 >> 16);
#pragma unroll
            for (int o = 1; o < LP; o <<= 1) m = min(m, __shfl_xor_sync(gmask, m, o, LP));
            mq = m;
            // store this pixel's path costs (padding slots as 0, so the WTA sums never carry)
            if (sizeof(LT) == 1) {
                unsigned short *dst = reinterpret_cast<unsigned short *>(Lo + pp * Kp + s0);
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    dst[r] = (unsigned short)__byte_perm(L[r] & vm[r], 0, 0x0020);
            } else {
                unsigned *dst = reinterpret_cast<unsigned *>(Lo + pp * Kp + s0);
#pragma unroll
                for (int r = 0; r < NR; ++r) dst[r] = L[r] & vm[r];
            }
            // t for the next pixel
            unsigned up = __shfl_up_sync(gmask, L[NR - 1], 1, LP);
            unsigned dn = __shfl_down_sync(gmask, L[0], 1, LP);
            if (g == 0) up = kInf2;
            if (g == LP - 1) dn = kInf2;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const unsigned lm = __byte_perm(r > 0 ? L[r - 1] : up, L[r], 0x5432);
                const unsigned lp = __byte_perm(L[r], r < NR - 1 ? L[r + 1] : dn, 0x5432);
                t_[r] = __vimin3_u16x2(L[r], lm + P1P1, lp + P1P1);
            }
        }
    }
}

// ------------------------------------------------- SGM, thread per scanline
// For bands up to K = 30 (Kp <= 32) one thread owns a whole scanline: its
// Kp slots are NR = Kp/2 u16x2 registers, the +-1 neighbour of a slot is a
// byte_perm of adjacent registers, the path minimum a register reduction,
// and a one-slot re-centring another byte_perm -- no shuffles, no shared
// memory, 3-4x fewer instructions per pixel-path than the lane-group kernel
// and a dozen independent chains per step.  Larger re-centring jumps
// (depth edges) go through a per-thread local copy.  Same recurrence and
// same INF conventions as k_sgm_packed.
constexpr int SGMT_PF = 4;   // prefetch distance in pixels

template <int NR>
__device__ __forceinline__ void shift_regs(const unsigned (&t)[NR], unsigned (&o)[NR], int s) {
    if (s == 1) {
#pragma unroll
        for (int r = 0; r < NR; ++r) o[r] = __byte_perm(t[r], r < NR - 1 ? t[r + 1] : kInf2, 0x5432);
    } else if (s == -1) {
#pragma unroll
        for (int r = 0; r < NR; ++r) o[r] = __byte_perm(r > 0 ? t[r - 1] : kInf2, t[r], 0x5432);
    } else {
        // Any other jump, in registers: an odd jump first moves one slot
        // towards its sign (byte_perm of adjacent registers, so no slot the
        // rest still needs is dropped), the even rest is a barrel shift by
        // whole registers (2 slots each) in stages of 1, 2, 4, 8, 16.
        unsigned a[NR];
        if ((s & 1) && s > 0) {
#pragma unroll
            for (int r = 0; r < NR; ++r) a[r] = __byte_perm(t[r], r < NR - 1 ? t[r + 1] : kInf2, 0x5432);
            s -= 1;
        } else if (s & 1) {
#pragma unroll
            for (int r = 0; r < NR; ++r) a[r] = __byte_perm(r > 0 ? t[r - 1] : kInf2, t[r], 0x5432);
            s += 1;
        } else {
#pragma unroll
            for (int r = 0; r < NR; ++r) a[r] = t[r];
        }
        const int q = s / 2;                      // s is even here
        if (q > 0) {
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                if (q & (1 << k)) {
#pragma unroll
                    for (int r = 0; r < NR; ++r) a[r] = r + (1 << k) < NR ? a[r + (1 << k)] : kInf2;
                }
            }
        } else if (q < 0) {
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                if ((-q) & (1 << k)) {
#pragma unroll
                    for (int r = NR - 1; r >= 0; --r) a[r] = r - (1 << k) >= 0 ? a[r - (1 << k)] : kInf2;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < NR; ++r) o[r] = a[r];
    }
}

// Start pixel and length of scanline j0 of direction (dx, dy) in a W x H image.
__device__ __forceinline__ void scanline_of(int W, int H, int dx, int dy, int j0, int &x0,
                                            int &y0, int &n) {
    if (dy == 0) {
        y0 = j0; x0 = dx > 0 ? 0 : W - 1; n = W;
    } else if (dx == 0) {
        x0 = j0; y0 = dy > 0 ? 0 : H - 1; n = H;
    } else {
        if (j0 < W) {
            x0 = j0; y0 = dy > 0 ? 0 : H - 1;
        } else {
            const int i = j0 - W + 1;
            x0 = dx > 0 ? 0 : W - 1;
            y0 = dy > 0 ? i : H - 1 - i;
        }
        n = min(dx > 0 ? W - x0 : x0 + 1, dy > 0 ? H - y0 : y0 + 1);
    }
}

// One scanline swept by one thread.  Cimg / base / Lo are the costs, band
// centres and path-cost array of one view (and one direction for Lo).
// KC > 0 fixes K at compile time: the band masks of the slot registers
// become constants and their selects fold away.
template <int NR, typename LT, int KC = 0>
__device__ __forceinline__ void sgm_line_thread(const uint8_t *__restrict__ Cimg,
                                                const int32_t *__restrict__ base_img,
                                                LT *__restrict__ Lo_img, int W, int K, int P1,
                                                int P2, int dx, int dy, int x0, int y0, int n) {
    constexpr int Kp = 2 * NR;
    static_assert(Kp % 8 == 0, "slot rows are 8-byte aligned");
    constexpr int NW = Kp / 8;                 // 64-bit words per pixel row of costs
    const long step = (long)dy * W + dx;
    const long p0 = (long)y0 * W + x0;
    const uint2 *__restrict__ Cw = reinterpret_cast<const uint2 *>(Cimg + p0 * Kp);
    const long cstep = step * NW;
    const int32_t *__restrict__ base = base_img + p0;
    LT *__restrict__ Lo = Lo_img + p0 * Kp;
    const long lstep = step * Kp;

    const int Kb = KC > 0 ? KC : K;
    unsigned vm[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const int sa = 2 * r, sb = sa + 1;
        vm[r] = ((sa >= 1 && sa <= Kb) ? 0x0000FFFFu : 0u) | ((sb >= 1 && sb <= Kb) ? 0xFFFF0000u : 0u);
    }
    const unsigned P1P1 = (unsigned)P1 * 0x10001u;

    uint2 cring[SGMT_PF][NW];
    int bring[SGMT_PF];
#pragma unroll
    for (int u = 0; u < SGMT_PF; ++u) {
        if (u < n) {
            bring[u] = __ldg(base + u * step);
#pragma unroll
            for (int wd = 0; wd < NW; ++wd) cring[u][wd] = __ldg(Cw + u * cstep + wd);
        }
    }
    unsigned t_[NR];
    int mq = 0, bprev = 0;
    for (int tt = 0; tt < n; tt += SGMT_PF) {
#pragma unroll
        for (int u = 0; u < SGMT_PF; ++u) {
            const int t = tt + u;
            if (t >= n) break;
            unsigned c[NR];
#pragma unroll
            for (int wd = 0; wd < NW; ++wd) {
                c[4 * wd + 0] = __byte_perm(cring[u][wd].x, 0, 0x4140);
                c[4 * wd + 1] = __byte_perm(cring[u][wd].x, 0, 0x4342);
                c[4 * wd + 2] = __byte_perm(cring[u][wd].y, 0, 0x4140);
                c[4 * wd + 3] = __byte_perm(cring[u][wd].y, 0, 0x4342);
            }
            const int bcur = bring[u];
            if (t + SGMT_PF < n) {
                bring[u] = __ldg(base + (t + SGMT_PF) * step);
#pragma unroll
                for (int wd = 0; wd < NW; ++wd) cring[u][wd] = __ldg(Cw + (t + SGMT_PF) * cstep + wd);
            }
            unsigned L[NR];
            if (t == 0) {
#pragma unroll
                for (int r = 0; r < NR; ++r) L[r] = (c[r] & vm[r]) | (kInf2 & ~vm[r]);
            } else {
                const int s = bcur - bprev;
                unsigned ts[NR];
                if (s == 0) {
#pragma unroll
                    for (int r = 0; r < NR; ++r) ts[r] = t_[r];
                } else {
                    shift_regs<NR>(t_, ts, max(-Kp - 2, min(Kp + 2, s)));
                }
                const unsigned cap = (unsigned)(mq + P2) * 0x10001u;
                const unsigned mm = (unsigned)mq * 0x10001u;
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    const unsigned v = c[r] + __vminu2(ts[r], cap) - mm;
                    L[r] = (v & vm[r]) | (kInf2 & ~vm[r]);
                }
            }
            bprev = bcur;
            unsigned mt[NR];                       // path minimum, as a depth-log2(NR) tree
#pragma unroll
            for (int r = 0; r < NR; ++r) mt[r] = L[r];
#pragma unroll
            for (int w = 1; w < NR; w *= 2) {
#pragma unroll
                for (int r = 0; r + w < NR; r += 2 * w) mt[r] = __vminu2(mt[r], mt[r + w]);
            }
            const unsigned m2 = mt[0];
            mq = (int)min(m2 & 0xFFFFu, m2 >> 16);
            // store the pixel's path costs, padding slots as 0
            LT *dst = Lo + t * lstep;
            if (sizeof(LT) == 1) {
#pragma unroll
                for (int wd = 0; wd < NW; ++wd) {
                    uint2 v;
                    v.x = __byte_perm(L[4 * wd] & vm[4 * wd], L[4 * wd + 1] & vm[4 * wd + 1], 0x6420);
                    v.y = __byte_perm(L[4 * wd + 2] & vm[4 * wd + 2], L[4 * wd + 3] & vm[4 * wd + 3],
                                      0x6420);
                    reinterpret_cast<uint2 *>(dst)[wd] = v;
                }
            } else {
#pragma unroll
                for (int wd = 0; wd < NW; ++wd) {
                    uint4 v;
                    v.x = L[4 * wd] & vm[4 * wd];
                    v.y = L[4 * wd + 1] & vm[4 * wd + 1];
                    v.z = L[4 * wd + 2] & vm[4 * wd + 2];
                    v.w = L[4 * wd + 3] & vm[4 * wd + 3];
                    reinterpret_cast<uint4 *>(dst)[wd] = v;
                }
            }
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const unsigned lm = __byte_perm(r > 0 ? L[r - 1] : kInf2, L[r], 0x5432);
                const unsigned lp = __byte_perm(L[r], r < NR - 1 ? L[r + 1] : kInf2, 0x5432);
                t_[r] = __vimin3_u16x2(L[r], lm + P1P1, lp + P1P1);
            }
        }
    }
}

template <int NR, typename LT, int KC>
__global__ void __launch_bounds__(128)
    k_sgm_thread(const uint8_t *__restrict__ C0, const uint8_t *__restrict__ C1,
                 const int32_t *__restrict__ base0, const int32_t *__restrict__ base1, int W,
                 int H, int K, int P1, int P2, LT *__restrict__ Lout, int npaths,
                 SgmTasks tasks) {
    constexpr int Kp = 2 * NR;
    const long gid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (gid >= tasks.start[tasks.nseg]) return;
    int sg = 0;
    while (gid >= tasks.start[sg + 1]) ++sg;
    const int j0 = (int)(gid - tasks.start[sg]);
    const int view = tasks.view[sg], dir = tasks.dir[sg];
    int dx, dy, x0, y0, n;
    dir_of(dir, dx, dy);
    scanline_of(W, H, dx, dy, j0, x0, y0, n);
    const long N = (long)W * H;
    sgm_line_thread<NR, LT, KC>(view ? C1 : C0, view ? base1 : base0,
                                Lout + (long)(view * npaths + dir) * N * Kp, W, K, P1, P2, dx,
                                dy, x0, y0, n);
}

// ------------------------------------------- SGM, lane group per scanline
// GL lanes share one scanline; lane gl owns the SL consecutive slots
// [SL*gl, SL*gl + SL) of every pixel as SL/2 u16x2 registers (Kp = SL*GL).
// The predecessor's path costs reach the next pixel through a per-group
// shared-memory row of u16 slots: INF padding on both sides of the Kp slots,
// two buffers alternating by pixel parity, so a step is one store, one
// __syncwarp and SL/2 + 2 word loads at the re-centred offset.  Any
// re-centring jump (stereonet.py:5218) is then the same few instructions --
// the window simply starts s slots further along, and a jump past the band
// reads only padding -- so groups of one warp never diverge on it.  From the
// aligned window B (B[r] = slots b+2r, b+2r+1 of the predecessor with
// b = SL*gl + s - 1) the re-centred candidate minimum of slot pair r is
//   min(centre, minus + P1, plus + P1) = vimin3(prmt(B[r], B[r+1]), B[r] + P1, B[r+1] + P1).
// The path minimum is an in-lane vminu2 tree and GL - 1 independent shuffles.
//
// A pixel's costs and band centre arrive through cp.async into a per-lane
// shared ring of 2 * SGMG_PF slots (laid out [slot][lane]), issued SGMG_PF
// pixels ahead and read one pixel ahead.  Register prefetch rings of loads
// in flight stalled every step: loads share a warp's few scoreboards, so a
// use waited for later loads as well; async copies are tracked by commit
// groups instead.  Same recurrence, INF conventions and output layout as
// k_sgm_thread, except that uint8 path costs keep the padding slots' INF
// byte (0xFF): the WTA reads slots 1..K only, and 8 x 255 cannot carry.
template <int SL, int GL>
struct SgmGroupGeom {
    static constexpr int Kp = SL * GL;
    static constexpr int NR = SL / 2;                            // u16x2 registers per lane
    static constexpr int PADL = ((Kp + 4 + 7) / 8) * 8;          // INF slots before slot 0
    // last word a window can touch (s <= Kp + 2); rows are 8-byte aligned
    // and 2 mod 4 words long, so the window loads of a warp's groups spread
    // over twice the banks of 16-byte rows (at most 2-way conflicts at
    // shift 0 instead of 4-way for 10 groups of 3 lanes)
    static constexpr int LASTW = ((PADL + SL * (GL - 1) + Kp + 1) >> 1) + NR + 1;
    static constexpr int ROWW = (LASTW + 1) % 4 == 2   ? LASTW + 1
                                : (LASTW + 1) % 4 == 1 ? LASTW + 2
                                : (LASTW + 1) % 4 == 0 ? LASTW + 3
                                                       : LASTW + 4;   // words per row
    static constexpr int GPW = 32 / GL;                          // groups per warp
};
constexpr int SGMG_WARPS = 4;    // warps per CTA of k_sgm_group
constexpr int SGMG_PF = 8;       // copy distance in pixels (even: buffer parity is static)

template <int SL>
struct SgmCostWord;
template <>
struct SgmCostWord<8> { using T = uint2; };
template <>
struct SgmCostWord<4> { using T = unsigned; };

template <int BYTES>
__device__ __forceinline__ void cp_async_bytes(void *smem_dst, const void *gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(smem_dst)),
                 "l"(gsrc), "n"(BYTES)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int SL, int GL, typename LT, int KC>
__device__ __forceinline__ void sgm_line_group(const uint8_t *__restrict__ Cimg,
                                               const int32_t *__restrict__ base_img,
                                               LT *__restrict__ Lo_img, int W, int K, int P1,
                                               int P2, int dx, int dy, int x0, int y0, int n,
                                               int gl, unsigned gmask, int glane0, int lane,
                                               unsigned *__restrict__ row0,
                                               unsigned *__restrict__ row1,
                                               typename SgmCostWord<SL>::T *__restrict__ cst,
                                               int *__restrict__ bst) {
    using G = SgmGroupGeom<SL, GL>;
    using CW = typename SgmCostWord<SL>::T;
    constexpr int NR = G::NR, Kp = G::Kp, PF = SGMG_PF;
    const long step = (long)dy * W + dx;
    const long p0 = (long)y0 * W + x0;
    const long cstep = step * Kp;
    const uint8_t *cnx = Cimg + p0 * Kp + SL * gl;     // next pixel to copy
    const int32_t *bnx = base_img + p0;
    LT *__restrict__ lpx = Lo_img + p0 * Kp + SL * gl;

    const int Kb = KC > 0 ? KC : K;
    unsigned vm[NR], ninf[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const int sa = SL * gl + 2 * r, sb = sa + 1;
        vm[r] = ((sa >= 1 && sa <= Kb) ? 0x0000FFFFu : 0u) | ((sb >= 1 && sb <= Kb) ? 0xFFFF0000u : 0u);
        ninf[r] = kInf2 & ~vm[r];
    }
    const unsigned P1P1 = (unsigned)P1 * 0x10001u;
    int nb[GL > 1 ? GL - 1 : 1];                   // the other lanes of the group
#pragma unroll
    for (int j = 1; j < GL; ++j) nb[j - 1] = glane0 + (gl + j) % GL;

    for (int w = gl; w < G::ROWW; w += GL) {
        row0[w] = kInf2;
        row1[w] = kInf2;
    }
    // pixels 0 .. PF-1 into ring slots 0 .. PF-1, one commit group each
#pragma unroll
    for (int u = 0; u < PF; ++u) {
        if (u < n) {
            cp_async_bytes<SL>(cst + u * 32 + lane, cnx);
            cp_async_bytes<4>(bst + u * 32 + lane, bnx);
        }
        cp_async_commit();
        cnx += cstep;
        bnx += step;
    }
    cp_async_wait<PF - 1>();
    __syncwarp(gmask);
    CW cw = cst[lane];                             // pixel 0
    int bnext = bst[lane];
    int mq = 0, bprev = 0;
    for (int tt = 0; tt < n; tt += PF) {
        const int h = (tt / PF & 1) * PF;          // ring half of pixels tt .. tt+PF-1
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int t = tt + u;
            if (t >= n) break;                     // group-uniform
            unsigned c[NR];
            if constexpr (SL == 8) {
                c[0] = __byte_perm(cw.x, 0, 0x4140);
                c[1] = __byte_perm(cw.x, 0, 0x4342);
                c[2] = __byte_perm(cw.y, 0, 0x4140);
                c[3] = __byte_perm(cw.y, 0, 0x4342);
            } else {
                c[0] = __byte_perm(cw, 0, 0x4140);
                c[1] = __byte_perm(cw, 0, 0x4342);
            }
            const int bcur = bnext;
            // the next pixel's copy has landed (PF - 2 younger groups may not)
            cp_async_wait<PF - 2>();
            {
                const int sn = u + 1 < PF ? h + u + 1 : PF - h;   // ring slot of pixel t+1
                cw = cst[sn * 32 + lane];
                bnext = bst[sn * 32 + lane];
            }
            if (t + PF < n) {                      // pixel t+PF into the other half
                const int sp = PF - h + u;
                cp_async_bytes<SL>(cst + sp * 32 + lane, cnx);
                cp_async_bytes<4>(bst + sp * 32 + lane, bnx);
            }
            cp_async_commit();
            cnx += cstep;
            bnx += step;
            unsigned L[NR];
            if (t == 0) {
#pragma unroll
                for (int r = 0; r < NR; ++r) L[r] = (c[r] & vm[r]) | ninf[r];
            } else {
                // the predecessor's row, written at step t - 1 (tt is even)
                const unsigned *__restrict__ rw = (u & 1) ? row0 : row1;
                const int s = max(-Kp - 2, min(Kp + 2, bcur - bprev));
                const int b = G::PADL + SL * gl + s - 1;
                const unsigned *a = rw + (b >> 1);
                unsigned A[NR + 2];
#pragma unroll
                for (int i = 0; i < NR + 2; ++i) A[i] = a[i];
                const unsigned sel = (b & 1) ? 0x5432u : 0x3210u;
                unsigned B[NR + 1];
#pragma unroll
                for (int i = 0; i < NR + 1; ++i) B[i] = __byte_perm(A[i], A[i + 1], sel);
                const unsigned cap = (unsigned)(mq + P2) * 0x10001u;
                const unsigned mm = (unsigned)mq * 0x10001u;
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    const unsigned tr = __vimin3_u16x2(__byte_perm(B[r], B[r + 1], 0x5432),
                                                       B[r] + P1P1, B[r + 1] + P1P1);
                    const unsigned v = c[r] + __vminu2(tr, cap) - mm;
                    // with K fixed, a register whose two slots lie inside 1..K
                    // for every lane of the group needs no band mask
                    if (KC > 0 && r >= 1 && SL * (GL - 1) + 2 * r + 1 <= KC) L[r] = v;
                    else L[r] = (v & vm[r]) | ninf[r];
                }
            }
            bprev = bcur;
            {   // this pixel's path costs for the successor
                unsigned *__restrict__ ww = ((u & 1) ? row1 : row0) + (G::PADL >> 1) + NR * gl;
                if constexpr (NR == 4) {
                    *reinterpret_cast<uint2 *>(ww) = make_uint2(L[0], L[1]);
                    *reinterpret_cast<uint2 *>(ww + 2) = make_uint2(L[2], L[3]);
                } else {
                    *reinterpret_cast<uint2 *>(ww) = make_uint2(L[0], L[1]);
                }
            }
            // path minimum over the group
            unsigned m2 = L[0];
#pragma unroll
            for (int r = 1; r < NR; ++r) m2 = __vminu2(m2, L[r]);
            const int m0 = (int)min(m2 & 0xFFFFu, m2 >> 16);
            int m = m0;
#pragma unroll
            for (int j = 0; j < GL - 1; ++j) m = min(m, __shfl_sync(gmask, m0, nb[j]));
            mq = m;
            // store the pixel's path costs (uint8: padding keeps INF's low byte;
            // uint16: padding 0, so the WTA's 16-bit sums never carry)
            LT *dst = lpx;
            lpx += cstep;
            if constexpr (sizeof(LT) == 1) {
                if constexpr (NR == 4)
                    *reinterpret_cast<uint2 *>(dst) =
                        make_uint2(__byte_perm(L[0], L[1], 0x6420), __byte_perm(L[2], L[3], 0x6420));
                else
                    *reinterpret_cast<unsigned *>(dst) = __byte_perm(L[0], L[1], 0x6420);
            } else {
                if constexpr (NR == 4)
                    *reinterpret_cast<uint4 *>(dst) =
                        make_uint4(L[0] & vm[0], L[1] & vm[1], L[2] & vm[2], L[3] & vm[3]);
                else
                    *reinterpret_cast<uint2 *>(dst) = make_uint2(L[0] & vm[0], L[1] & vm[1]);
            }
            __syncwarp(gmask);
        }
    }
    cp_async_wait<0>();
}

template <int SL, int GL, typename LT, int KC>
__global__ void __launch_bounds__(SGMG_WARPS * 32)
    k_sgm_group(const uint8_t *__restrict__ C0, const uint8_t *__restrict__ C1,
                const int32_t *__restrict__ base0, const int32_t *__restrict__ base1, int W,
                int H, int K, int P1, int P2, LT *__restrict__ Lout, int npaths,
                SgmTasks tasks) {
    using G = SgmGroupGeom<SL, GL>;
    using CW = typename SgmCostWord<SL>::T;
    constexpr int Kp = G::Kp, GPW = G::GPW;
    __shared__ __align__(16) unsigned rows[SGMG_WARPS][2][GPW][G::ROWW];
    __shared__ __align__(16) CW cstage[SGMG_WARPS][2 * SGMG_PF][32];
    __shared__ __align__(16) int bstage[SGMG_WARPS][2 * SGMG_PF][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / GL, gl = lane - g * GL;
    if (g >= GPW) return;                                  // lanes past the last whole group
    const long gid = ((long)blockIdx.x * SGMG_WARPS + warp) * GPW + g;
    if (gid >= tasks.start[tasks.nseg]) return;            // whole groups leave together
    const unsigned gmask = ((1u << GL) - 1u) << (g * GL);
    int sg = 0;
    while (gid >= tasks.start[sg + 1]) ++sg;
    const int j0 = (int)(gid - tasks.start[sg]);
    const int view = tasks.view[sg], dir = tasks.dir[sg];
    int dx, dy, x0, y0, n;
    dir_of(dir, dx, dy);
    scanline_of(W, H, dx, dy, j0, x0, y0, n);
    const long N = (long)W * H;
    sgm_line_group<SL, GL, LT, KC>(view ? C1 : C0, view ? base1 : base0,
                                   Lout + (long)(view * npaths + dir) * N * Kp, W, K, P1, P2,
                                   dx, dy, x0, y0, n, gl, gmask, g * GL, lane, rows[warp][0][g],
                                   rows[warp][1][g], &cstage[warp][0][0], &bstage[warp][0][0]);
}

// ------------------------------------------------------------------ WTA
template <typename LT>
__device__ __forceinline__ int path_sum_slot(const LT *__restrict__ L, long stride, int npaths,
                                             int slot) {
    int acc = 0;
    for (int d = 0; d < npaths; ++d) acc += (int)L[d * stride + slot];
    return acc;
}

template <typename LT, int KPC = 0, int NPC = 0>
__device__ __forceinline__ void wta_pixel(const LT *__restrict__ Lp, long stride, int npaths,
                                          int K, int Kp, int R, int32_t base_p,
                                          const double *__restrict__ d0p, double uniq,
                                          bool want_conf, double *__restrict__ outp,
                                          double *__restrict__ confp);

// nviews <= 2; KPC / NPC > 0 fix Kp and the path count at compile time, so
// a pixel's loads all issue before its first sum.
template <typename LT, int KPC, int NPC>
__global__ void __launch_bounds__(256)
    k_wta_slot(const LT *__restrict__ Lall, int npaths, int nviews, long N, int K, int Kp, int R,
               const int32_t *__restrict__ base0, const int32_t *__restrict__ base1,
               const double *__restrict__ d00, const double *__restrict__ d01, double uniq,
               int want_conf, double *__restrict__ out0, double *__restrict__ out1,
               double *__restrict__ conf0) {
    const long stride = N * Kp;                            // between path arrays
    for (long w = blockIdx.x * (long)blockDim.x + threadIdx.x; w < nviews * N;
         w += (long)gridDim.x * blockDim.x) {
        const int view = w >= N ? 1 : 0;
        const long p = w - view * N;
        wta_pixel<LT, KPC, NPC>(Lall + (long)view * npaths * stride + p * Kp, stride, npaths, K, Kp, R,
                      (view ? base1 : base0)[p], (view ? d01 : d00) + p, uniq,
                      want_conf && view == 0, (view ? out1 : out0) + p,
                      conf0 ? conf0 + p : nullptr);
    }
}

// S = sum of the path costs at one pixel (Lp: its row in path array 0),
// first minimum, FP64 parabola (stereonet.py:5271-5303).
template <typename LT, int KPC, int NPC>
__device__ __forceinline__ void wta_pixel(const LT *__restrict__ Lp, long stride, int npaths,
                                          int K, int Kp, int R, int32_t base_p,
                                          const double *__restrict__ d0p, double uniq,
                                          bool want_conf, double *__restrict__ outp,
                                          double *__restrict__ confp) {
    constexpr int PER64 = 8 / sizeof(LT);                  // slots per 64-bit load
    const int kp = KPC > 0 ? KPC : Kp, np = NPC > 0 ? NPC : npaths;
    {
        int bv = 0x7FFFFFFF, bs = -1;                      // best value, its slot
#pragma unroll
        for (int c = 0; c < kp; c += 8) {
            unsigned acc[4] = {0u, 0u, 0u, 0u};            // 8 slots as u16x2
#pragma unroll
            for (int d = 0; d < np; ++d) {
                if (PER64 == 8) {
                    const uint2 v = __ldg(reinterpret_cast<const uint2 *>(Lp + d * stride + c));
                    acc[0] += __byte_perm(v.x, 0, 0x4140);
                    acc[1] += __byte_perm(v.x, 0, 0x4342);
                    acc[2] += __byte_perm(v.y, 0, 0x4140);
                    acc[3] += __byte_perm(v.y, 0, 0x4342);
                } else {
                    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(Lp + d * stride + c));
                    acc[0] += v.x;
                    acc[1] += v.y;
                    acc[2] += v.z;
                    acc[3] += v.w;
                }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int slot = c + u;
                const int v = (int)((acc[u >> 1] >> (16 * (u & 1))) & 0xFFFFu);
                if (slot >= 1 && slot <= K && v < bv) {
                    bv = v;
                    bs = slot;
                }
            }
        }
        const int bk = bs - 1;
        if (bk == 0 || bk == K - 1) {
            *outp = *d0p;
            if (want_conf) *confp = 0.0;
            return;
        }
        const int va = path_sum_slot(Lp, stride, np, bs - 1);
        const int vb = path_sum_slot(Lp, stride, np, bs + 1);
        bool use_d0 = false;
        if (uniq > 0.0 || want_conf) {
            // second best away from the winner's neighbours (stereonet.py:5286-5290)
            int sv = 0x7FFFFFFF;
            for (int k = 0; k < K; ++k)
                if (k < bk - 1 || k > bk + 1) sv = min(sv, path_sum_slot(Lp, stride, np, k + 1));
            double conf = 1.0;
            if (sv != 0x7FFFFFFF) {
                const double dsv = (double)sv, dbv = (double)bv;
                conf = __ddiv_rn(__dsub_rn(dsv, dbv), __dadd_rn(dbv, 1.0e-6));
            }
            if (want_conf) *confp = conf;
            use_d0 = conf < uniq;
        }
        if (use_d0) {
            *outp = *d0p;
            return;
        }
        const double a = (double)va, b = (double)vb, dbv = (double)bv;
        const double den = __dadd_rn(__dsub_rn(a, __dmul_rn(2.0, dbv)), b);
        double off = 0.0;
        if (den > 1.0e-9) off = __ddiv_rn(__dmul_rn(0.5, __dsub_rn(a, b)), den);
        *outp = __dadd_rn((double)(base_p - R + bk), off);
    }
}

// ====================================================================
// Host
// ====================================================================

// (Kp, lanes per scanline, registers per lane) for K + 2 slots
struct SgmGeom {
    int Kp, LP, NR;
};
static const SgmGeom kGeom[] = {{8, 4, 1},    {16, 4, 2},   {24, 4, 3},  {32, 4, 4},
                                {48, 8, 3},   {64, 8, 4},   {96, 16, 3}, {128, 16, 4},
                                {192, 32, 3}, {256, 32, 4}};

static SgmGeom geom_for(int K) {
    for (const SgmGeom &g : kGeom)
        if (g.Kp >= K + 2) return g;
    return kGeom[sizeof(kGeom) / sizeof(kGeom[0]) - 1];
}

int slot_width(int K) { return geom_for(K).Kp; }

int launch_band_costs_slot(const uint64_t *cl, const uint64_t *cr, const int32_t *base0,
                           const int32_t *base1, int W, int H, int R, int invalid, uint8_t *C0,
                           uint8_t *C1, int nviews, cudaStream_t st, const uint8_t *rad0) {
    const long N = (long)W * H;
    const int K = 2 * R + 1;
    dim3 grd(grid_for(N, 256, 148 * 8), nviews);
    count_launch();
    if (K == 21)    // R = 10, the refine_disparity default: 24 slots
        k_band_costs_slot<24, 21><<<grd, 256, 0, st>>>(cl, cr, base0, base1, W, N, R, K, 24,
                                                       invalid, C0, C1, rad0);
    else
        k_band_costs_slot<0, 0><<<grd, 256, 0, st>>>(cl, cr, base0, base1, W, N, R, K,
                                                     slot_width(K), invalid, C0, C1, rad0);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <int NR, int LP, typename LT>
static int sgm_packed_go(const uint8_t *C0, const uint8_t *C1, const int32_t *b0,
                         const int32_t *b1, int W, int H, int K, int Kp, int P1, int P2,
                         void *Lout, int npaths, const SgmTasks &t, cudaStream_t st) {
    const long groups = t.start[t.nseg];
    const long threads = groups * LP;
    const int blocks = (int)((threads + 255) / 256);
    const size_t smem = (size_t)(256 / LP) * Kp * sizeof(unsigned short);
    count_launch();
    k_sgm_packed<NR, LP, LT><<<blocks, 256, smem, st>>>(C0, C1, b0, b1, W, H, K, Kp, P1, P2,
                                                         (LT *)Lout, npaths, t);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <int NR, typename LT, int KC = 0>
static int sgm_thread_go(const uint8_t *C0, const uint8_t *C1, const int32_t *b0,
                         const int32_t *b1, int W, int H, int K, int P1, int P2, void *Lout,
                         int npaths, const SgmTasks &t, cudaStream_t st) {
    const long threads = t.start[t.nseg];
    const int blocks = (int)((threads + 127) / 128);
    count_launch();
    k_sgm_thread<NR, LT, KC><<<blocks, 128, 0, st>>>(C0, C1, b0, b1, W, H, K, P1, P2,
                                                      (LT *)Lout, npaths, t);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

template <int SL, int GL, typename LT, int KC = 0>
static int sgm_group_go(const uint8_t *C0, const uint8_t *C1, const int32_t *b0,
                        const int32_t *b1, int W, int H, int K, int P1, int P2, void *Lout,
                        int npaths, const SgmTasks &t, cudaStream_t st) {
    constexpr int GPW = SgmGroupGeom<SL, GL>::GPW;
    const long groups = t.start[t.nseg];
    const long warps = (groups + GPW - 1) / GPW;
    const int blocks = (int)((warps + SGMG_WARPS - 1) / SGMG_WARPS);
    count_launch();
    k_sgm_group<SL, GL, LT, KC><<<blocks, SGMG_WARPS * 32, 0, st>>>(C0, C1, b0, b1, W, H, K, P1,
                                                                     P2, (LT *)Lout, npaths, t);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

// Single-pair SGM kernel for bands up to K = 30: 0 = lane groups of 8 slots
// per lane (default), 1 = lane groups of 4 slots per lane, 2 = one thread per
// scanline.  SV_SGM_KERNEL = group8 | group4 | thread overrides it (all three
// give the same refined output; the choice only moves time).
static int sgm_variant() {
    static const int v = [] {
        const char *e = getenv("SV_SGM_KERNEL");
        if (e && !strcmp(e, "group4")) return 1;
        if (e && !strcmp(e, "thread")) return 2;
        return 0;
    }();
    return v;
}

template <typename LT>
static int sgm_packed_dispatch(const uint8_t *C0, const uint8_t *C1, const int32_t *b0,
                               const int32_t *b1, int W, int H, int K, int P1, int P2,
                               void *Lout, int npaths, const SgmTasks &t, cudaStream_t st) {
    const SgmGeom g = geom_for(K);
    const int var = sgm_variant();
    if (var == 0 && g.Kp <= 32) {
        switch (g.Kp) {
        case 8: return sgm_group_go<8, 1, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        case 16: return sgm_group_go<8, 2, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        case 24:
            if (K == 21)
                return sgm_group_go<8, 3, LT, 21>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
            return sgm_group_go<8, 3, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        default: return sgm_group_go<8, 4, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        }
    }
    if (var == 1 && g.Kp <= 32) {
        switch (g.Kp) {
        case 8: return sgm_group_go<4, 2, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        case 16: return sgm_group_go<4, 4, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        case 24:
            if (K == 21)
                return sgm_group_go<4, 6, LT, 21>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
            return sgm_group_go<4, 6, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        default: return sgm_group_go<4, 8, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        }
    }
    // bands up to K = 30: one thread per scanline
    switch (g.Kp) {
    case 8: return sgm_thread_go<4, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
    case 16: return sgm_thread_go<8, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
    case 24:
        if (K == 21)    // R = 10, the refine_disparity default
            return sgm_thread_go<12, LT, 21>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
        return sgm_thread_go<12, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
    case 32: return sgm_thread_go<16, LT>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
    default: break;
    }
#define SV_GEOM(KP, LPV, NRV)                                                                \
    if (g.Kp == KP)                                                                          \
        return sgm_packed_go<NRV, LPV, LT>(C0, C1, b0, b1, W, H, K, KP, P1, P2, Lout, npaths, \
                                           t, st);
    SV_GEOM(8, 4, 1)
    SV_GEOM(16, 4, 2)
    SV_GEOM(24, 4, 3)
    SV_GEOM(32, 4, 4)
    SV_GEOM(48, 8, 3)
    SV_GEOM(64, 8, 4)
    SV_GEOM(96, 16, 3)
    SV_GEOM(128, 16, 4)
    SV_GEOM(192, 32, 3)
    SV_GEOM(256, 32, 4)
#undef SV_GEOM
    set_error("no SGM geometry for K=%d", K);
    return SV_ERR_SHAPE;
}

int launch_sgm_packed(const uint8_t *C0, const uint8_t *C1, const int32_t *b0,
                      const int32_t *b1, int W, int H, int K, int P1, int P2, void *Lout,
                      bool l16, int nviews, int npaths, cudaStream_t st) {
    SgmTasks t = make_sgm_tasks(W, H, nviews, npaths, nullptr, 0);
    if (l16)
        return sgm_packed_dispatch<uint16_t>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
    return sgm_packed_dispatch<uint8_t>(C0, C1, b0, b1, W, H, K, P1, P2, Lout, npaths, t, st);
}

int launch_wta_slot(const void *L, bool l16, int npaths, int nviews, int W, int H, int R,
                    const int32_t *b0, const int32_t *b1, const double *d00, const double *d01,
                    double uniq, double *out0, double *out1, double *conf0, cudaStream_t st) {
    const long N = (long)W * H;
    const int K = 2 * R + 1;
    const int Kp = slot_width(K);
    const int blocks = grid_for(nviews * N, 256, 148 * 16);
    count_launch();
    if (nviews < 1 || nviews > 2) {
        set_error("wta: nviews=%d", nviews);
        return SV_ERR_PARAM;
    }
    if (l16)
        k_wta_slot<uint16_t, 0, 0><<<blocks, 256, 0, st>>>(
            (const uint16_t *)L, npaths, nviews, N, K, Kp, R, b0, b1, d00, d01, uniq,
            conf0 != nullptr, out0, out1, conf0);
    else if (Kp == 24 && npaths == 8)    // R = 10 over the 8 paths
        k_wta_slot<uint8_t, 24, 8><<<blocks, 256, 0, st>>>(
            (const uint8_t *)L, npaths, nviews, N, K, Kp, R, b0, b1, d00, d01, uniq,
            conf0 != nullptr, out0, out1, conf0);
    else
        k_wta_slot<uint8_t, 0, 0><<<blocks, 256, 0, st>>>(
            (const uint8_t *)L, npaths, nviews, N, K, Kp, R, b0, b1, d00, d01, uniq,
            conf0 != nullptr, out0, out1, conf0);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

// ====================================================================
// Batched lr_refine, middle stages.  Costs and WTA run one block per
// px_per_block pixels of a pair (blockIdx.y = view).  The SGM is a
// persistent kernel over a device-side queue: every warp takes sgm_fetch
// (32 by default) scanline tasks at a time from one atomic counter, tasks
// ordered longest scanline first (segments of (pair, view, direction) sorted by length on the host),
// so all pairs' scanlines share one launch and finish together.
// ====================================================================

// KPC / KC / NPC > 0: the band geometry fixed at compile time, as in the
// single-pair kernels (the whole batch shares K).
template <int KPC, int KC>
__global__ void __launch_bounds__(256) k_b_costs(BatchTables t) {
    const int i = batch_find(t.px_blk, t.n, blockIdx.x);
    const BatchPair &P = t.pairs[i];
    const int view = blockIdx.y;
    const long N = (long)P.W * P.H;
    const long p0 = (long)(blockIdx.x - t.px_blk[i]) * t.px_per_block;
    const long p1 = min(N, p0 + (long)t.px_per_block);
    const uint64_t *ref = view ? P.cen1 : P.cen0;
    const uint64_t *oth = view ? P.cen0 : P.cen1;
    for (long p = p0 + threadIdx.x; p < p1; p += blockDim.x)
        cost_pixel_slot<KPC, KC>(ref, oth, view ? P.base1 : P.base0, P.W, p, t.R, t.K, t.Kp,
                                 t.invalid, view, view ? P.C1 : P.C0, t.R);
}

template <int NR, typename LT, int KC>
__global__ void __launch_bounds__(256) k_b_sgm(BatchTables t, long long total) {
    constexpr int Kp = 2 * NR;
    const int lane = threadIdx.x & 31;
    const int fetch = t.sgm_fetch;                         // a multiple of 32
    for (;;) {
        long long first = 0;
        if (lane == 0) first = atomicAdd(t.queue, fetch);
        first = __shfl_sync(kFull, first, 0);
        if (first >= total) return;                        // warp-uniform
        for (int j = lane; j < fetch; j += 32) {
            const long long task = first + j;
            if (task >= total) break;
            const int s = batch_find(t.seg_start, t.nseg, task);
            const BatchPair &P = t.pairs[t.seg_pair[s]];
            const int view = t.seg_vd[s] >> 3, dir = t.seg_vd[s] & 7;
            int dx, dy, x0, y0, n;
            dir_of(dir, dx, dy);
            scanline_of(P.W, P.H, dx, dy, (int)(task - t.seg_start[s]), x0, y0, n);
            const long N = (long)P.W * P.H;
            sgm_line_thread<NR, LT, KC>(view ? P.C1 : P.C0, view ? P.base1 : P.base0,
                                    reinterpret_cast<LT *>(P.L) + (long)(view * t.npaths + dir) * N * Kp,
                                    P.W, t.K, t.P1, t.P2, dx, dy, x0, y0, n);
        }
    }
}

template <typename LT, int KPC, int NPC>
__global__ void __launch_bounds__(256) k_b_wta(BatchTables t) {
    const int i = batch_find(t.px_blk, t.n, blockIdx.x);
    const BatchPair &P = t.pairs[i];
    const int view = blockIdx.y;
    const long N = (long)P.W * P.H;
    const long stride = N * t.Kp;
    const long p0 = (long)(blockIdx.x - t.px_blk[i]) * t.px_per_block;
    const long p1 = min(N, p0 + (long)t.px_per_block);
    const LT *Lv = reinterpret_cast<const LT *>(P.L) + (long)view * t.npaths * stride;
    for (long p = p0 + threadIdx.x; p < p1; p += blockDim.x)
        wta_pixel<LT, KPC, NPC>(Lv + p * t.Kp, stride, t.npaths, t.K, t.Kp, t.R,
                      (view ? P.base1 : P.base0)[p], (view ? P.d0r : P.disp0) + p, t.uniq, false,
                      (view ? P.dr : P.dl) + p, nullptr);
}

int launch_batch_front(const BatchTables &t, long long px_blocks, long long rows,
                       long long tiles, cudaStream_t st);
int launch_batch_back(const BatchTables &t, long long rows, cudaStream_t st);

template <int NR, typename LT, int KC = 0>
static int batch_sgm_go(const BatchTables &t, long long tasks, int threads, int ctas_per_sm,
                        cudaStream_t st) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long want = (tasks + threads - 1) / threads;
    const long long cap = (long long)sms * ctas_per_sm;    // persistent: a few CTAs per SM
    const unsigned blocks = (unsigned)(want < cap ? (want < 1 ? 1 : want) : cap);
    count_launch();
    k_b_sgm<NR, LT, KC><<<blocks, threads, 0, st>>>(t, tasks);
    SV_LAUNCH_CHECK();
    return SV_OK;
}

int launch_batch_refine(const BatchTables &t, long long px_blocks, long long rows,
                        long long tiles, long long tasks, bool l16, int sgm_threads,
                        int sgm_ctas_per_sm, cudaStream_t st) {
    int rc = launch_batch_front(t, px_blocks, rows, tiles, st);
    if (rc) return rc;
    const bool k21 = t.K == 21 && t.Kp == 24;       // R = 10, the refine_disparity default
    count_launch();
    if (k21)
        k_b_costs<24, 21><<<dim3((unsigned)px_blocks, 2), 256, 0, st>>>(t);
    else
        k_b_costs<0, 0><<<dim3((unsigned)px_blocks, 2), 256, 0, st>>>(t);
    SV_LAUNCH_CHECK();
    if (k21 && !l16)
        rc = batch_sgm_go<12, uint8_t, 21>(t, tasks, sgm_threads, sgm_ctas_per_sm, st);
    else switch (t.Kp) {
#define SV_BGO(KP)                                                                      \
    case KP:                                                                            \
        rc = l16 ? batch_sgm_go<KP / 2, uint16_t>(t, tasks, sgm_threads, sgm_ctas_per_sm, st) \
                 : batch_sgm_go<KP / 2, uint8_t>(t, tasks, sgm_threads, sgm_ctas_per_sm, st);  \
        break;
        SV_BGO(8)
        SV_BGO(16)
        SV_BGO(24)
        SV_BGO(32)
#undef SV_BGO
    default:
        set_error("batched refinement supports bands up to K = 30 (got K = %d)", t.K);
        return SV_ERR_SHAPE;
    }
    if (rc) return rc;
    count_launch();
    if (l16)
        k_b_wta<uint16_t, 0, 0><<<dim3((unsigned)px_blocks, 2), 256, 0, st>>>(t);
    else if (k21 && t.npaths == 8)
        k_b_wta<uint8_t, 24, 8><<<dim3((unsigned)px_blocks, 2), 256, 0, st>>>(t);
    else
        k_b_wta<uint8_t, 0, 0><<<dim3((unsigned)px_blocks, 2), 256, 0, st>>>(t);
    SV_LAUNCH_CHECK();
    return launch_batch_back(t, rows, st);
}

}  // namespace sv
