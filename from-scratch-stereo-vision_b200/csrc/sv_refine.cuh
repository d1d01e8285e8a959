// sv_refine.cuh -- host launchers of the refinement kernels (sv_refine.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace sv {

// Scanline work table of the SGM kernels: segment i covers the scanlines of
// (view[i], dir[i]); start[] are cumulative scanline counts.
struct SgmTasks {
    int nseg;
    int start[17];
    int view[16];
    int dir[16];
};

// Longest scanlines first (horizontal, vertical, diagonal) so that the
// longest-running warps start in the first wave.  dirs_only restricts the
// table to the listed directions (one view).
inline SgmTasks make_sgm_tasks(int W, int H, int nviews, int npaths, const int *dirs_only,
                               int ndirs_only) {
    SgmTasks t{};
    int order[8] = {0, 1, 2, 3, 4, 5, 6, 7};
    if (H > W) { order[0] = 2; order[1] = 3; order[2] = 0; order[3] = 1; }
    t.start[0] = 0;
    for (int oi = 0; oi < 8; ++oi) {
        const int d = order[oi];
        if (dirs_only) {
            bool keep = false;
            for (int i = 0; i < ndirs_only; ++i) keep |= dirs_only[i] == d;
            if (!keep) continue;
        } else if (d >= npaths) {
            continue;
        }
        const int cnt = d < 2 ? H : d < 4 ? W : W + H - 1;
        for (int v = 0; v < nviews; ++v) {
            t.view[t.nseg] = v;
            t.dir[t.nseg] = d;
            t.start[t.nseg + 1] = t.start[t.nseg] + cnt;
            t.nseg++;
        }
    }
    return t;
}

// Bytes per pixel of the slot layout used by the fused refinement (K + 2
// slots rounded up to a multiple of 8).
int slot_width(int K);

// Validated refinement parameters (sv_api.cu).
struct RefineCfg {
    int R, K, P1, P2, rx, ry, nbits, npaths, invalid;
    double uniq;
    bool l16;
};
int check_refine(int W, int H, const sv_refine_params *p, bool rows, RefineCfg *c);
int check_ws(void *ws, size_t have, size_t need);

// ------------------------------------------------------------- batches
// One pair of a batched lr_refine: its inputs/outputs and its slice of the
// workspace (device table entry).
struct BatchPair {
    const void *left, *right;
    const double *disp0;
    double *out;
    uint8_t *status;
    int W, H;
    int32_t *base0, *base1;
    double *d0r, *dl, *dr;
    uint64_t *cen0, *cen1;
    uint8_t *C0, *C1;
    void *L;
};

constexpr int kBatchPxPerBlock = 2048;   // default pixels per block of the per-pixel kernels

// Everything a batched kernel needs, passed by value.  Prefix tables map a
// block (or an SGM task) to its pair by binary search.
struct BatchTables {
    const BatchPair *pairs;
    int n;
    const long long *px_blk;     // [n+1] blocks of px_per_block pixels
    const long long *row_blk;    // [n+1] image rows
    const long long *tile_blk;   // [n+1] census tiles
    const long long *seg_start;  // [nseg+1] scanlines per (pair, view, dir) segment
    const int *seg_pair;         // [nseg]
    const int *seg_vd;           // [nseg] view * 8 + dir
    int nseg;
    int *queue;                  // SGM task counter, zeroed per call
    int *flag;                   // data errors (first wins)
    int R, K, Kp, P1, P2, npaths, invalid, rx, ry, dtype, maxW;
    int px_per_block;            // pixels per CTA of the per-pixel stages
    int sgm_fetch;               // scanline tasks a warp claims per queue fetch
    double tol, uniq;
};

// Largest i in [0, n) with prefix[i] <= v (prefix is non-decreasing).
__device__ __forceinline__ int batch_find(const long long *prefix, int n, long long v) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// A batch's layout in its workspace: per-pair slices and the host copies of
// the device tables (sv_batch_api.cu).
struct BatchPlan {
    std::vector<BatchPair> pairs;
    std::vector<long long> px_blk, row_blk, tile_blk, seg_start;
    std::vector<int> seg_pair, seg_vd;
    long long px_blocks = 0, rows = 0, tiles = 0, tasks = 0;
    int maxW = 1;
    size_t off_tables = 0, off_pairs = 0, off_px = 0, off_row = 0, off_tile = 0, off_seg = 0,
           off_segp = 0, off_segvd = 0, total = 0;
};
// Sizes and offsets; with ws != nullptr also fills the per-pair pointers.
int plan_batch(const sv_pair_desc *in, int n, const RefineCfg &c, int px_per_block, char *ws,
               BatchPlan *pl);
int upload_batch(const BatchPlan &pl, int n, char *ws, cudaStream_t st);
BatchTables batch_tables(const BatchPlan &pl, int n, char *ws, const RefineCfg &c, int dtype,
                         double tol, const sv_batch_config &cfg);

int launch_batch_refine(const BatchTables &t, long long px_blocks, long long rows,
                        long long tiles, long long tasks, bool l16, int sgm_threads,
                        int sgm_ctas_per_sm, cudaStream_t st);

int launch_base(const double *disp0, long N, int32_t *base, int *flag, cudaStream_t st);
int launch_census(const void *img0, const void *img1, int dtype, int W, int H, int rx,
                  int ry, uint64_t *out0, uint64_t *out1, cudaStream_t st);
int launch_band_costs(const uint64_t *cl, const uint64_t *cr, const int32_t *base0,
                      const int32_t *base1, int W, int H, int R, int invalid, uint8_t *C0,
                      uint8_t *C1, int nviews, cudaStream_t st);
int launch_sgm_add_path(const uint8_t *C, const int32_t *base, int W, int H, int K, int P1,
                        int P2, int dir, uint16_t *S, cudaStream_t st);
// rad0 (may be NULL): per-pixel half-width of the left view's band; slots
// with |k - R| > rad0[p] get the invalid cost.
int launch_band_costs_slot(const uint64_t *cl, const uint64_t *cr, const int32_t *base0,
                           const int32_t *base1, int W, int H, int R, int invalid, uint8_t *C0,
                           uint8_t *C1, int nviews, cudaStream_t st,
                           const uint8_t *rad0 = nullptr);
int launch_sgm_packed(const uint8_t *C0, const uint8_t *C1, const int32_t *b0,
                      const int32_t *b1, int W, int H, int K, int P1, int P2, void *Lout,
                      bool l16, int nviews, int npaths, cudaStream_t st);
int launch_wta_slot(const void *L, bool l16, int npaths, int nviews, int W, int H, int R,
                    const int32_t *b0, const int32_t *b1, const double *d00, const double *d01,
                    double uniq, double *out0, double *out1, double *conf0, cudaStream_t st);
// base_l (optional): also k_base's band centres of dl, errors into flag.
int launch_left_to_right(const double *dl, int W, int H, double *dr, int32_t *base_r,
                         cudaStream_t st, int32_t *base_l = nullptr, int *flag = nullptr);
int launch_lr_check(const double *dl, const double *dr, const double *disp0, int W, int H,
                    double tol, double *out, uint8_t *status, cudaStream_t st);

}  // namespace sv
