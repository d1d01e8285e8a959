// sv_noalloc.cu -- refine_fullres for callers that cannot allocate.
//
// Some callers of this library have no way to hand it device memory for
// scratch: an engine that reserves all of its GPU memory at start-up and
// forbids allocations afterwards, a plugin host that gives its plugins no
// allocator, or code on a path where a cudaMalloc would stall or fail.
// sv_refine_fullres_noalloc serves them: it runs the same kernels as
// sv_refine_fullres, but its scratch (band centres, census words, band costs
// and the path-cost arrays) lives in one file-scope __device__ array of
// SV_NOALLOC_SCRATCH_BYTES.  The caller still passes the images, the
// disparity, the output and a device int for the data-error status; nothing
// is allocated.
//
// Capacity.  The scratch holds, each rounded up to 256 bytes, a 256-byte
// header, 4N bytes of band centres, 2 x 8N of census words, N*Kp of band
// costs and npaths*N*Kp*(1 or 2) of path costs (N = W*H, Kp = K+2 rounded up
// to 8, 16, 24, 32, 48, ...; 2 bytes per path cost when 4+bits+P2 > 255).
// For refine_disparity's parameters (K = 21 -> Kp = 24, 8 paths, 1 byte) that
// is 236 bytes per pixel, so up to about 71,000 pixels (300x236 fits, 320x240
// does not); with paths = 4 it is 140 bytes per pixel.  Larger inputs are
// rejected with SV_ERR_SHAPE before anything runs.
//
// Rules that come with a shared static array:
//  * every GPU that loads this library holds the array until the process
//    exits;
//  * the array's device address is resolved with cudaGetSymbolAddress on the
//    first call on a device (with that device current) and cached per CUDA
//    context, so a new context on the device (after cudaDeviceReset, or a
//    driver-API context) resolves it again; make the first call on a device
//    before any stream capture;
//  * all calls share the one array and it keeps the last call's contents:
//    every byte a call reads is written by the same call first;
//  * calls whose work overlaps on the GPU (two streams, or two host threads
//    without ordering) race on the array and corrupt each other's results;
//    serialise them.

#include <cmath>
#include <mutex>

#include "sv_common.cuh"
#include "sv_refine.cuh"

namespace sv {

// The scratch.  Host code must not take this name's address: on the host it
// is a stand-in symbol, not device memory.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SV_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
struct ScratchSlot {
    unsigned long long ctx_id;   // the CUDA context the address belongs to
    void *ptr;
};
ScratchSlot g_scratch[kMaxDevices] = {};

// Unique id of the current CUDA context (never reused within a process), or
// 0 when the driver offers no such query or no context is current yet.
typedef int (*CtxGetCurrentFn)(void **);
typedef int (*CtxGetIdFn)(void *, unsigned long long *);
unsigned long long current_ctx_id() {
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_cur = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
    });
    if (!get_cur || !get_id) return 0;
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch in the current device's current context.
int scratch_address(void **out) {
    int dev = 0;
    SV_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device %d beyond the %d supported", dev, kMaxDevices);
        return SV_ERR_PARAM;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    ScratchSlot &slot = g_scratch[dev];
    const unsigned long long id = current_ctx_id();
    if (!slot.ptr || id == 0 || id != slot.ctx_id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress of the static scratch failed: %s",
                      cudaGetErrorString(e));
            return SV_ERR_CUDA;
        }
        slot.ptr = p;
        slot.ctx_id = id ? id : current_ctx_id();   // the lookup made a context current
    }
    *out = slot.ptr;
    return SV_OK;
}

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace sv

using namespace sv;

extern "C" int sv_refine_fullres_noalloc(const void *left, const void *right, int dtype,
                                         const double *disp0, int W, int H,
                                         const sv_refine_params *p, double *out,
                                         int *data_status, void *stream) {
    if (!left || !right || !disp0 || !out || !p || !data_status) {
        set_error("NULL argument (data_status is required: it is the only report of a "
                  "NaN, infinite or out-of-range disparity)");
        return SV_ERR_NULL;
    }
    if (W < 1 || H < 1) { set_error("W=%d H=%d must be positive", W, H); return SV_ERR_SHAPE; }
    if (p->R < 0 || 2 * p->R + 1 > kMaxK) {
        set_error("R=%d outside 0..%d", p->R, (kMaxK - 1) / 2);
        return SV_ERR_SHAPE;
    }
    if (p->rx < 0 || p->ry < 0 || (2 * p->rx + 1) * (2 * p->ry + 1) - 1 > 64) {
        set_error("census window rx=%d ry=%d needs more than 64 bits", p->rx, p->ry);
        return SV_ERR_SHAPE;
    }
    if (p->ad_weight != 0.0 || p->prior_w != 0.0 || !std::isfinite(p->ad_trunc) ||
        !std::isfinite(p->prior_t) || !std::isfinite(p->uniq)) {
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
    const int K = 2 * p->R + 1;
    const int nbits = (2 * p->rx + 1) * (2 * p->ry + 1) - 1;
    const int invalid = nbits + 4;
    const int P1 = (int)p->P1, P2 = (int)p->P2;
    const int npaths = p->paths == 8 ? 8 : 4;
    const bool l16 = invalid + P2 > 255;
    const size_t N = (size_t)W * H, NK = N * slot_width(K);
    // layout: header | base | census left | census right | costs | path costs
    const size_t o_base = 256;
    const size_t o_cl = o_base + up256(N * 4);
    const size_t o_cr = o_cl + up256(N * 8);
    const size_t o_c = o_cr + up256(N * 8);
    const size_t o_l = o_c + up256(NK);
    const size_t need = o_l + up256(NK * npaths * (l16 ? 2 : 1));
    if (need > SV_NOALLOC_SCRATCH_BYTES) {
        set_error("%dx%d with K=%d needs %zu scratch bytes; the static scratch holds %u "
                  "(use sv_refine_fullres with a workspace)", W, H, K, need,
                  (unsigned)SV_NOALLOC_SCRATCH_BYTES);
        return SV_ERR_SHAPE;
    }
    char *s = nullptr;
    int rc = scratch_address(reinterpret_cast<void **>(&s));
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int *flag = data_status;
    int32_t *base = reinterpret_cast<int32_t *>(s + o_base);
    uint64_t *cl = reinterpret_cast<uint64_t *>(s + o_cl);
    uint64_t *cr = reinterpret_cast<uint64_t *>(s + o_cr);
    uint8_t *C = reinterpret_cast<uint8_t *>(s + o_c);
    void *L = s + o_l;
    SV_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), st));
    if ((rc = launch_base(disp0, (long)N, base, flag, st))) return rc;
    if ((rc = launch_census(left, right, dtype, W, H, p->rx, p->ry, cl, cr, st))) return rc;
    if ((rc = launch_band_costs_slot(cl, cr, base, nullptr, W, H, p->R, invalid, C, nullptr, 1,
                                    st)))
        return rc;
    if ((rc = launch_sgm_packed(C, nullptr, base, nullptr, W, H, K, P1, P2, L, l16, 1, npaths,
                               st)))
        return rc;
    return launch_wta_slot(L, l16, npaths, 1, W, H, p->R, base, nullptr, disp0, nullptr, p->uniq,
                      out, nullptr, nullptr, st);
}
