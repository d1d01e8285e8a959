// sv_batch_api.cu -- lr_refine over a batch of rectified pairs of uneven
// sizes in one launch per stage (extern "C" sv_batch_lr_refine).
//
// Every pair gets the same arithmetic as sv_lr_refine (so its outputs are
// bit-identical to refining it alone); what changes is the scheduling: the
// workspace holds one slice per pair, small device tables map blocks and
// SGM tasks to pairs, and the SGM stage is a persistent kernel draining a
// device-side queue of (pair, view, direction, scanline) tasks, longest
// scanlines first.

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "sv_common.cuh"
#include "sv_refine.cuh"

namespace sv {

namespace {
constexpr int kTileW = 32, kTileH = 8;   // census tile (k_census)
}  // namespace

// Sizes and offsets; with ws != nullptr also fills the per-pair pointers.
int plan_batch(const sv_pair_desc *in, int n, const RefineCfg &c, int px_per_block, char *ws,
               BatchPlan *pl) {
    BatchPlan &P = *pl;
    const int Kp = slot_width(c.K);
    const size_t lt = c.l16 ? 2 : 1;
    Carver cv(ws);
    cv.take<DevFlags>(1);
    cv.take<int>(64);                                      // queue counter (+ padding)
    P.off_pairs = cv.off;
    cv.take<BatchPair>(n);
    P.off_px = cv.off;
    cv.take<long long>(n + 1);
    P.off_row = cv.off;
    cv.take<long long>(n + 1);
    P.off_tile = cv.off;
    cv.take<long long>(n + 1);
    const int nseg = n * 2 * c.npaths;
    P.off_seg = cv.off;
    cv.take<long long>(nseg + 1);
    P.off_segp = cv.off;
    cv.take<int>(nseg);
    P.off_segvd = cv.off;
    cv.take<int>(nseg);
    P.pairs.resize(n);
    P.px_blk.assign(n + 1, 0);
    P.row_blk.assign(n + 1, 0);
    P.tile_blk.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        const sv_pair_desc &d = in[i];
        if (d.W < 1 || d.H < 1 || d.W > kMaxRowW) {
            set_error("pair %d: %dx%d outside 1..%d wide", i, d.W, d.H, kMaxRowW);
            return SV_ERR_SHAPE;
        }
        if (ws && (!d.left || !d.right || !d.disp0 || !d.out || !d.status)) {
            set_error("pair %d: NULL pointer", i);
            return SV_ERR_NULL;
        }
        const size_t N = (size_t)d.W * d.H;
        BatchPair &b = P.pairs[i];
        b.left = d.left;
        b.right = d.right;
        b.disp0 = d.disp0;
        b.out = d.out;
        b.status = d.status;
        b.W = d.W;
        b.H = d.H;
        b.base0 = cv.take<int32_t>(N);
        b.base1 = cv.take<int32_t>(N);
        b.d0r = cv.take<double>(N);
        b.dl = cv.take<double>(N);
        b.dr = cv.take<double>(N);
        b.cen0 = cv.take<uint64_t>(N);
        b.cen1 = cv.take<uint64_t>(N);
        b.C0 = cv.take<uint8_t>(N * Kp);
        b.C1 = cv.take<uint8_t>(N * Kp);
        b.L = cv.take<uint8_t>(2 * (size_t)c.npaths * N * Kp * lt);
        P.px_blk[i + 1] = P.px_blk[i] + (long long)((N + px_per_block - 1) / px_per_block);
        P.row_blk[i + 1] = P.row_blk[i] + d.H;
        P.tile_blk[i + 1] = P.tile_blk[i] + (long long)((d.W + kTileW - 1) / kTileW) *
                                                ((d.H + kTileH - 1) / kTileH);
        P.maxW = std::max(P.maxW, d.W);
    }
    P.total = cv.off;
    P.px_blocks = P.px_blk[n];
    P.rows = P.row_blk[n];
    P.tiles = P.tile_blk[n];
    // SGM segments, longest scanlines first
    struct Seg { int pair, vd, count, len; };
    std::vector<Seg> segs;
    segs.reserve(nseg);
    for (int i = 0; i < n; ++i) {
        const int W = in[i].W, H = in[i].H;
        for (int v = 0; v < 2; ++v)
            for (int d = 0; d < c.npaths; ++d) {
                const int cnt = d < 2 ? H : d < 4 ? W : W + H - 1;
                const int len = d < 2 ? W : d < 4 ? H : std::min(W, H);
                segs.push_back({i, v * 8 + d, cnt, len});
            }
    }
    std::stable_sort(segs.begin(), segs.end(),
                     [](const Seg &a, const Seg &b) { return a.len > b.len; });
    P.seg_start.assign(nseg + 1, 0);
    P.seg_pair.resize(nseg);
    P.seg_vd.resize(nseg);
    for (int s = 0; s < nseg; ++s) {
        P.seg_start[s + 1] = P.seg_start[s] + segs[s].count;
        P.seg_pair[s] = segs[s].pair;
        P.seg_vd[s] = segs[s].vd;
    }
    P.tasks = P.seg_start[nseg];
    return SV_OK;
}

int upload_batch(const BatchPlan &pl, int n, char *ws, cudaStream_t st) {
    SV_CUDA_TRY(cudaMemcpyAsync(ws + pl.off_pairs, pl.pairs.data(), sizeof(BatchPair) * n,
                                cudaMemcpyHostToDevice, st));
    SV_CUDA_TRY(cudaMemcpyAsync(ws + pl.off_px, pl.px_blk.data(), sizeof(long long) * (n + 1),
                                cudaMemcpyHostToDevice, st));
    SV_CUDA_TRY(cudaMemcpyAsync(ws + pl.off_row, pl.row_blk.data(), sizeof(long long) * (n + 1),
                                cudaMemcpyHostToDevice, st));
    SV_CUDA_TRY(cudaMemcpyAsync(ws + pl.off_tile, pl.tile_blk.data(),
                                sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, st));
    const int nseg = (int)pl.seg_pair.size();
    SV_CUDA_TRY(cudaMemcpyAsync(ws + pl.off_seg, pl.seg_start.data(),
                                sizeof(long long) * (nseg + 1), cudaMemcpyHostToDevice, st));
    SV_CUDA_TRY(cudaMemcpyAsync(ws + pl.off_segp, pl.seg_pair.data(), sizeof(int) * nseg,
                                cudaMemcpyHostToDevice, st));
    SV_CUDA_TRY(cudaMemcpyAsync(ws + pl.off_segvd, pl.seg_vd.data(), sizeof(int) * nseg,
                                cudaMemcpyHostToDevice, st));
    return SV_OK;
}

BatchTables batch_tables(const BatchPlan &pl, int n, char *ws, const RefineCfg &c, int dtype,
                         double tol, const sv_batch_config &cfg) {
    BatchTables t{};
    t.pairs = reinterpret_cast<const BatchPair *>(ws + pl.off_pairs);
    t.n = n;
    t.px_blk = reinterpret_cast<const long long *>(ws + pl.off_px);
    t.row_blk = reinterpret_cast<const long long *>(ws + pl.off_row);
    t.tile_blk = reinterpret_cast<const long long *>(ws + pl.off_tile);
    t.seg_start = reinterpret_cast<const long long *>(ws + pl.off_seg);
    t.seg_pair = reinterpret_cast<const int *>(ws + pl.off_segp);
    t.seg_vd = reinterpret_cast<const int *>(ws + pl.off_segvd);
    t.nseg = (int)pl.seg_pair.size();
    t.flag = reinterpret_cast<int *>(ws);
    t.queue = reinterpret_cast<int *>(ws + sizeof(DevFlags));
    t.R = c.R;
    t.K = c.K;
    t.Kp = slot_width(c.K);
    t.P1 = c.P1;
    t.P2 = c.P2;
    t.npaths = c.npaths;
    t.invalid = c.invalid;
    t.rx = c.rx;
    t.ry = c.ry;
    t.dtype = dtype;
    t.maxW = pl.maxW;
    t.tol = tol;
    t.uniq = c.uniq;
    t.px_per_block = cfg.px_per_block;
    t.sgm_fetch = cfg.sgm_fetch;
    return t;
}

}  // namespace sv

using namespace sv;

extern "C" {

size_t sv_batch_lr_refine_workspace_size(const sv_pair_desc *pairs, int n,
                                         const sv_refine_params *p) {
    if (!pairs || n < 1) return 0;
    RefineCfg c;
    if (check_refine(1, 1, p, true, &c) != SV_OK) return 0;
    if (slot_width(c.K) > 32) {
        set_error("batched refinement supports bands up to K = 30 (got K = %d)", c.K);
        return 0;
    }
    BatchPlan pl;
    if (plan_batch(pairs, n, c, kBatchPxPerBlock, nullptr, &pl) != SV_OK) return 0;
    return pl.total;
}

void sv_batch_config_default(sv_batch_config *cfg) {
    if (!cfg) return;
    cfg->px_per_block = kBatchPxPerBlock;
    cfg->sgm_threads = 128;
    cfg->sgm_ctas_per_sm = 8;
    cfg->sgm_fetch = 32;
}

int sv_batch_lr_refine(const sv_pair_desc *pairs, int n, int dtype, double tol,
                       const sv_refine_params *p, void *workspace, size_t workspace_bytes,
                       void *stream) {
    sv_batch_config cfg;
    sv_batch_config_default(&cfg);
    return sv_batch_lr_refine_ex(pairs, n, dtype, tol, p, &cfg, workspace, workspace_bytes,
                                 stream);
}

int sv_batch_lr_refine_ex(const sv_pair_desc *pairs, int n, int dtype, double tol,
                          const sv_refine_params *p, const sv_batch_config *cfg,
                          void *workspace, size_t workspace_bytes, void *stream) {
    if (!pairs || n < 1) { set_error("no pairs"); return SV_ERR_NULL; }
    if (!cfg) { set_error("NULL config"); return SV_ERR_NULL; }
    {
        const int px = cfg->px_per_block, th = cfg->sgm_threads, f = cfg->sgm_fetch;
        if (px < 256 || px > 8192 || (px & (px - 1)) || (th != 32 && th != 64 && th != 128 &&
                                                          th != 256) ||
            cfg->sgm_ctas_per_sm < 1 || cfg->sgm_ctas_per_sm > 32 ||
            (f != 32 && f != 64 && f != 128)) {
            set_error("batch config: px_per_block a power of 2 in 256..8192, sgm_threads "
                      "32/64/128/256, sgm_ctas_per_sm 1..32, sgm_fetch 32/64/128");
            return SV_ERR_PARAM;
        }
    }
    RefineCfg c;
    int rc = check_refine(1, 1, p, true, &c);
    if (rc) return rc;
    if (slot_width(c.K) > 32) {
        set_error("batched refinement supports bands up to K = 30 (got K = %d)", c.K);
        return SV_ERR_SHAPE;
    }
    if (!std::isfinite(tol)) { set_error("tol must be finite"); return SV_ERR_PARAM; }
    if (dtype != SV_U8 && dtype != SV_F32 && dtype != SV_F64) {
        set_error("unknown image dtype %d", dtype);
        return SV_ERR_PARAM;
    }
    BatchPlan pl;
    if ((rc = plan_batch(pairs, n, c, cfg->px_per_block, nullptr, &pl))) return rc;
    if ((rc = check_ws(workspace, workspace_bytes, pl.total))) return rc;
    if ((rc = plan_batch(pairs, n, c, cfg->px_per_block, static_cast<char *>(workspace), &pl)))
        return rc;
    char *ws = static_cast<char *>(workspace);
    cudaStream_t st = (cudaStream_t)stream;
    // tables to the device (pageable copies are staged before the call returns)
    if ((rc = upload_batch(pl, n, ws, st))) return rc;
    SV_CUDA_TRY(cudaMemsetAsync(ws, 0, sizeof(DevFlags) + 256, st));   // flag + queue
    const BatchTables t = batch_tables(pl, n, ws, c, dtype, tol, *cfg);
    return launch_batch_refine(t, pl.px_blocks, pl.rows, pl.tiles, pl.tasks, c.l16,
                               cfg->sgm_threads, cfg->sgm_ctas_per_sm, st);
}

}  // extern "C"
