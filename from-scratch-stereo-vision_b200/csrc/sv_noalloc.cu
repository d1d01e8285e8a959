// sv_noalloc.cu -- refine_fullres for callers that cannot allocate.
//
// Some callers of this library have no way to hand it device memory for
// scratch: an engine that reserves all of its GPU memory at start-up and
// forbids allocations afterwards, a plugin host that gives its plugins no
// allocator, or code on a path where a cudaMalloc would stall or fail.
// sv_refine_fullres_noalloc serves them: it runs the same kernels as
// sv_refine_fullres, but its scratch (band centres, census words, band costs,
// the eight path-cost arrays and the data-error flag) lives in one
// file-scope __device__ array of SV_NOALLOC_SCRATCH_BYTES.  The caller still
// passes the images, the disparity and the output; nothing is allocated.
//
// Rules that come with a shared static array:
//  * every GPU that loads this library holds the array until the process
//    exits;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current); make
//    that first call before any stream capture;
//  * all calls share the one array and it keeps the last call's contents:
//    the data-error flag is cleared at the start of every call and every
//    other byte a call reads is written by the same call first;
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
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch on the current device (resolved once).
int scratch_address(void **out) {
    int dev = 0;
    SV_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device %d beyond the %d supported", dev, kMaxDevices);
        return SV_ERR_PARAM;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress of the static scratch failed: %s",
                      cudaGetErrorString(e));
            return SV_ERR_CUDA;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
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
    if (!left || !right || !disp0 || !out || !p) {
        set_error("NULL argument");
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
    // layout: flag | base | census left | census right | costs | path costs
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
    int *flag = data_status ? data_status : reinterpret_cast<int *>(s);
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
