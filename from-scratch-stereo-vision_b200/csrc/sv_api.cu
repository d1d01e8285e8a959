// sv_api.cu -- the extern "C" entry points of include/sv_b200.h (refinement).
//
// Argument checks happen before anything is enqueued; data-dependent errors
// (a NaN disparity) are flagged by the kernels in the workspace header.

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "sv_common.cuh"
#include "sv_refine.cuh"

namespace sv {

static thread_local char g_err[512];
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launches(unsigned long long n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
unsigned long long launch_count_now() { return g_launches.load(std::memory_order_relaxed); }

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

// Validated refinement parameters.
int check_refine(int W, int H, const sv_refine_params *p, bool rows, RefineCfg *c) {
    if (!p) { set_error("params is NULL"); return SV_ERR_NULL; }
    if (W < 1 || H < 1) { set_error("W=%d H=%d must be positive", W, H); return SV_ERR_SHAPE; }
    if (rows && W > kMaxRowW) {
        set_error("W=%d exceeds the row-kernel limit %d", W, kMaxRowW);
        return SV_ERR_SHAPE;
    }
    if (p->R < 0 || 2 * p->R + 1 > kMaxK) {
        set_error("R=%d outside 0..%d", p->R, (kMaxK - 1) / 2);
        return SV_ERR_SHAPE;
    }
    if (p->rx < 0 || p->ry < 0 || (2 * p->rx + 1) * (2 * p->ry + 1) - 1 > 64) {
        set_error("census window rx=%d ry=%d needs more than 64 bits", p->rx, p->ry);
        return SV_ERR_SHAPE;
    }
    if (p->ad_weight != 0.0 || p->prior_w != 0.0 || !std::isfinite(p->ad_trunc) ||
        !std::isfinite(p->prior_t)) {
        set_error("only ad_weight == 0 and prior_w == 0 are supported by the exact path");
        return SV_ERR_PARAM;
    }
    auto int_pen = [](double v) {
        return std::isfinite(v) && v >= 0.0 && v <= kMaxPenalty && v == std::floor(v);
    };
    if (!int_pen(p->P1) || !int_pen(p->P2)) {
        set_error("P1=%g P2=%g must be integers in 0..%d", p->P1, p->P2, kMaxPenalty);
        return SV_ERR_PARAM;
    }
    if (!std::isfinite(p->uniq)) { set_error("uniq must be finite"); return SV_ERR_PARAM; }
    c->R = p->R;
    c->K = 2 * p->R + 1;
    c->P1 = (int)p->P1;
    c->P2 = (int)p->P2;
    c->rx = p->rx;
    c->ry = p->ry;
    c->nbits = (2 * p->rx + 1) * (2 * p->ry + 1) - 1;
    c->npaths = p->paths == 8 ? 8 : 4;      // stereonet.py:5267: anything else is 4
    c->invalid = c->nbits + 4;               // stereonet.py:5261-5262 with zero weights
    c->uniq = p->uniq;
    c->l16 = c->invalid + c->P2 > 255;
    return SV_OK;
}

struct RefineWs {
    DevFlags *flags;
    int32_t *base0, *base1;
    double *d0r, *dl, *dr;
    uint64_t *cen0, *cen1;
    uint8_t *C0, *C1;
    void *L;
};

static size_t carve_refine(void *ws, int W, int H, const RefineCfg &c, int nviews,
                           RefineWs *o) {
    const size_t N = (size_t)W * H, NK = N * slot_width(c.K);
    Carver cv(ws);
    RefineWs r{};
    r.flags = cv.take<DevFlags>(1);
    r.base0 = cv.take<int32_t>(N);
    r.cen0 = cv.take<uint64_t>(N);
    r.cen1 = cv.take<uint64_t>(N);
    r.C0 = cv.take<uint8_t>(NK);
    if (nviews == 2) {
        r.base1 = cv.take<int32_t>(N);
        r.d0r = cv.take<double>(N);
        r.dl = cv.take<double>(N);
        r.dr = cv.take<double>(N);
        r.C1 = cv.take<uint8_t>(NK);
    }
    size_t lbytes = (size_t)nviews * c.npaths * NK * (c.l16 ? 2 : 1);
    r.L = cv.take<uint8_t>(lbytes);
    if (o) *o = r;
    return cv.off;
}

int check_ws(void *ws, size_t have, size_t need) {
    if (!ws) { set_error("workspace is NULL"); return SV_ERR_WORKSPACE; }
    if ((uintptr_t)ws & 255) { set_error("workspace must be 256-byte aligned"); return SV_ERR_WORKSPACE; }
    if (have < need) {
        set_error("workspace has %zu bytes, %zu needed", have, need);
        return SV_ERR_WORKSPACE;
    }
    return SV_OK;
}

#define SV_TRY(expr)                  \
    do {                              \
        int rc_ = (expr);             \
        if (rc_ != SV_OK) return rc_; \
    } while (0)

}  // namespace sv

using namespace sv;

extern "C" {

const char *sv_status_string(int s) {
    switch (s) {
    case SV_OK: return "ok";
    case SV_ERR_SHAPE: return "shape out of the supported range";
    case SV_ERR_PARAM: return "unsupported parameter";
    case SV_ERR_DISP: return "disparity is NaN, infinite or out of range";
    case SV_ERR_WORKSPACE: return "workspace missing, misaligned or too small";
    case SV_ERR_CUDA: return "CUDA error";
    case SV_ERR_NULL: return "NULL pointer";
    case SV_ERR_NET: return "weights do not match the architecture";
    case SV_ERR_TIMEOUT: return "a bounded device wait or host poll gave up";
    default: return "unknown status";
    }
}

const char *sv_last_error(void) { return g_err; }

int sv_version(void) { return 1; }

unsigned long long sv_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

void sv_refine_params_default(sv_refine_params *p) {
    if (!p) return;
    p->R = 3;
    p->P1 = 1.0;
    p->P2 = 12.0;
    p->rx = 2;
    p->ry = 2;
    p->paths = 8;
    p->uniq = 0.0;
    p->ad_weight = 0.0;
    p->ad_trunc = 20.0;
    p->prior_w = 0.0;
    p->prior_t = 4.0;
}

int sv_workspace_status(const void *workspace, void *stream) {
    if (!workspace) return SV_ERR_NULL;
    int flag = 0;
    SV_CUDA_TRY(cudaMemcpyAsync(&flag, workspace, sizeof(int), cudaMemcpyDeviceToHost,
                                (cudaStream_t)stream));
    SV_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    if (flag) set_error("kernel reported: %s", sv_status_string(flag));
    return flag;
}

int sv_census(const void *img, int dtype, int W, int H, int rx, int ry, uint64_t *out,
              void *stream) {
    if (!img || !out) { set_error("NULL image or output"); return SV_ERR_NULL; }
    if (W < 1 || H < 1) { set_error("bad shape %dx%d", W, H); return SV_ERR_SHAPE; }
    if (rx < 0 || ry < 0 || (2 * rx + 1) * (2 * ry + 1) - 1 > 64) {
        set_error("census window rx=%d ry=%d needs more than 64 bits", rx, ry);
        return SV_ERR_SHAPE;
    }
    return launch_census(img, nullptr, dtype, W, H, rx, ry, out, nullptr,
                         (cudaStream_t)stream);
}

int sv_band_costs(const uint64_t *cl, const uint64_t *cr, const int32_t *base, int W,
                  int H, int R, int invalid, uint8_t *C, void *stream) {
    if (!cl || !cr || !base || !C) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1 || R < 0 || 2 * R + 1 > kMaxK) {
        set_error("bad shape W=%d H=%d R=%d", W, H, R);
        return SV_ERR_SHAPE;
    }
    if (invalid < 0 || invalid > 255) {
        set_error("invalid cost %d outside 0..255", invalid);
        return SV_ERR_PARAM;
    }
    return launch_band_costs(cl, cr, base, nullptr, W, H, R, invalid, C, nullptr, 1,
                             (cudaStream_t)stream);
}

int sv_aggregate_path(const uint8_t *C, const int32_t *base, int W, int H, int K, int P1,
                      int P2, int dx, int dy, uint16_t *S, void *stream) {
    if (!C || !base || !S) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1 || K < 1 || K > kMaxK || !(K & 1)) {
        set_error("bad shape W=%d H=%d K=%d", W, H, K);
        return SV_ERR_SHAPE;
    }
    if (P1 < 0 || P2 < 0 || P1 > kMaxPenalty || P2 > kMaxPenalty) {
        set_error("P1=%d P2=%d outside 0..%d", P1, P2, kMaxPenalty);
        return SV_ERR_PARAM;
    }
    int dir = -1;
    static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1},
                                   {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
    for (int i = 0; i < 8; ++i)
        if (dirs[i][0] == dx && dirs[i][1] == dy) dir = i;
    if (dir < 0) { set_error("direction (%d,%d) is not an SGM path", dx, dy); return SV_ERR_PARAM; }
    return launch_sgm_add_path(C, base, W, H, K, P1, P2, dir, S, (cudaStream_t)stream);
}

int sv_left_to_right(const double *dl, int W, int H, double *dr, void *stream) {
    if (!dl || !dr) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1 || W > kMaxRowW) { set_error("bad shape %dx%d", W, H); return SV_ERR_SHAPE; }
    return launch_left_to_right(dl, W, H, dr, nullptr, (cudaStream_t)stream);
}

size_t sv_refine_workspace_size(int W, int H, const sv_refine_params *p) {
    RefineCfg c;
    if (check_refine(W, H, p, false, &c) != SV_OK) return 0;
    return carve_refine(nullptr, W, H, c, 1, nullptr);
}

size_t sv_lr_refine_workspace_size(int W, int H, const sv_refine_params *p) {
    RefineCfg c;
    if (check_refine(W, H, p, true, &c) != SV_OK) return 0;
    return carve_refine(nullptr, W, H, c, 2, nullptr);
}

int sv_refine_fullres(const void *left, const void *right, int dtype, const double *disp0,
                      int W, int H, const sv_refine_params *p, double *out, double *conf,
                      void *workspace, size_t workspace_bytes, void *stream) {
    if (!left || !right || !disp0 || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    RefineCfg c;
    SV_TRY(check_refine(W, H, p, false, &c));
    SV_TRY(check_ws(workspace, workspace_bytes, carve_refine(nullptr, W, H, c, 1, nullptr)));
    RefineWs w;
    carve_refine(workspace, W, H, c, 1, &w);
    cudaStream_t st = (cudaStream_t)stream;
    const long N = (long)W * H;
    SV_CUDA_TRY(cudaMemsetAsync(w.flags, 0, sizeof(DevFlags), st));
    SV_TRY(launch_base(disp0, N, w.base0, &w.flags->status, st));
    SV_TRY(launch_census(left, right, dtype, W, H, c.rx, c.ry, w.cen0, w.cen1, st));
    SV_TRY(launch_band_costs_slot(w.cen0, w.cen1, w.base0, nullptr, W, H, c.R, c.invalid, w.C0,
                             nullptr, 1, st));
    SV_TRY(launch_sgm_packed(w.C0, nullptr, w.base0, nullptr, W, H, c.K, c.P1, c.P2, w.L, c.l16, 1,
                      c.npaths, st));
    SV_TRY(launch_wta_slot(w.L, c.l16, c.npaths, 1, W, H, c.R, w.base0, nullptr, disp0, nullptr,
                      c.uniq, out, nullptr, conf, st));
    return SV_OK;
}

// part: LR_ALL, LR_CENSUS (the census of both views only: it needs the
// images alone, so a caller may run it while the disparity is still being
// computed) or LR_AFTER_CENSUS (the rest, over the census already in the
// workspace).
enum { LR_ALL = 0, LR_CENSUS = 1, LR_AFTER_CENSUS = 2 };

static int lr_refine_impl(const void *left, const void *right, int dtype, const double *disp0,
                          int W, int H, double tol, const sv_refine_params *p, double *out,
                          uint8_t *status, void *workspace, size_t workspace_bytes,
                          void *stream, void *const *events, int n_events,
                          const uint8_t *rad = nullptr, int part = LR_ALL) {
    if (!left || !right || (part != LR_CENSUS && (!disp0 || !out || !status))) {
        set_error("NULL argument");
        return SV_ERR_NULL;
    }
    RefineCfg c;
    SV_TRY(check_refine(W, H, p, true, &c));
    if (!std::isfinite(tol)) { set_error("tol must be finite"); return SV_ERR_PARAM; }
    if (events && n_events < SV_LR_STAGES + 1) {
        set_error("stage timing needs %d events", SV_LR_STAGES + 1);
        return SV_ERR_PARAM;
    }
    SV_TRY(check_ws(workspace, workspace_bytes, carve_refine(nullptr, W, H, c, 2, nullptr)));
    RefineWs w;
    carve_refine(workspace, W, H, c, 2, &w);
    cudaStream_t st = (cudaStream_t)stream;
    int ev = 0;
    auto mark = [&]() -> int {
        if (events) SV_CUDA_TRY(cudaEventRecord((cudaEvent_t)events[ev++], st));
        return SV_OK;
    };
    if (part == LR_CENSUS)
        return launch_census(left, right, dtype, W, H, c.rx, c.ry, w.cen0, w.cen1, st);
    SV_TRY(mark());
    SV_CUDA_TRY(cudaMemsetAsync(w.flags, 0, sizeof(DevFlags), st));
    SV_TRY(launch_left_to_right(disp0, W, H, w.d0r, w.base1, st, w.base0, &w.flags->status));
    SV_TRY(mark());
    if (part != LR_AFTER_CENSUS)
        SV_TRY(launch_census(left, right, dtype, W, H, c.rx, c.ry, w.cen0, w.cen1, st));
    SV_TRY(mark());
    SV_TRY(launch_band_costs_slot(w.cen0, w.cen1, w.base0, w.base1, W, H, c.R, c.invalid, w.C0,
                             w.C1, 2, st, rad));
    SV_TRY(mark());
    SV_TRY(launch_sgm_packed(w.C0, w.C1, w.base0, w.base1, W, H, c.K, c.P1, c.P2, w.L, c.l16, 2,
                      c.npaths, st));
    SV_TRY(mark());
    SV_TRY(launch_wta_slot(w.L, c.l16, c.npaths, 2, W, H, c.R, w.base0, w.base1, disp0, w.d0r,
                      c.uniq, w.dl, w.dr, nullptr, st));
    SV_TRY(mark());
    SV_TRY(launch_lr_check(w.dl, w.dr, disp0, W, H, tol, out, status, st));
    SV_TRY(mark());
    return SV_OK;
}

}  // extern "C"

namespace sv {
int lr_refine_census(const void *left, const void *right, int dtype, int W, int H,
                     const sv_refine_params *p, void *workspace, size_t workspace_bytes,
                     cudaStream_t st) {
    return lr_refine_impl(left, right, dtype, nullptr, W, H, 0.0, p, nullptr, nullptr, workspace,
                          workspace_bytes, st, nullptr, 0, nullptr, LR_CENSUS);
}
int lr_refine_after_census(const void *left, const void *right, int dtype, const double *disp0,
                           int W, int H, double tol, const sv_refine_params *p, double *out,
                           uint8_t *status, void *workspace, size_t workspace_bytes,
                           cudaStream_t st) {
    return lr_refine_impl(left, right, dtype, disp0, W, H, tol, p, out, status, workspace,
                          workspace_bytes, st, nullptr, 0, nullptr, LR_AFTER_CENSUS);
}
}  // namespace sv

extern "C" {

int sv_lr_refine(const void *left, const void *right, int dtype, const double *disp0, int W,
                 int H, double tol, const sv_refine_params *p, double *out, uint8_t *status,
                 void *workspace, size_t workspace_bytes, void *stream) {
    return lr_refine_impl(left, right, dtype, disp0, W, H, tol, p, out, status, workspace,
                          workspace_bytes, stream, nullptr, 0);
}

int sv_lr_refine_band(const void *left, const void *right, int dtype, const double *centre,
                      const uint8_t *rad, int W, int H, double tol, const sv_refine_params *p,
                      double *out, uint8_t *status, void *workspace, size_t workspace_bytes,
                      void *stream) {
    if (!rad) { set_error("NULL half-width map"); return SV_ERR_NULL; }
    return lr_refine_impl(left, right, dtype, centre, W, H, tol, p, out, status, workspace,
                          workspace_bytes, stream, nullptr, 0, rad);
}

int sv_lr_refine_timed(const void *left, const void *right, int dtype, const double *disp0,
                       int W, int H, double tol, const sv_refine_params *p, double *out,
                       uint8_t *status, void *workspace, size_t workspace_bytes, void *stream,
                       void *const *events, int n_events) {
    if (!events) { set_error("events is NULL"); return SV_ERR_NULL; }
    return lr_refine_impl(left, right, dtype, disp0, W, H, tol, p, out, status, workspace,
                          workspace_bytes, stream, events, n_events);
}

}  // extern "C"
