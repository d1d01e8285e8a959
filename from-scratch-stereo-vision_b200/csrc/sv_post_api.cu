// sv_post_api.cu -- extern "C" entry points of the rest of refine_disparity
// (stereonet.py:5865-5883): median_filter, slic, plane_snap and
// refine_disparity itself.

#include <cstdint>

#include "sv_common.cuh"
#include "sv_post.cuh"

using namespace sv;

namespace {

int check_ws_post(void *ws, size_t bytes, size_t need) {
    if (!ws || ((uintptr_t)ws & 255) || bytes < need) {
        set_error("workspace needs %zu bytes, 256-aligned (have %zu)", need, bytes);
        return SV_ERR_WORKSPACE;
    }
    return SV_OK;
}

int check_shape(int W, int H) {
    if (W < 1 || H < 1 || (long)W * H >= (1l << 31)) {
        set_error("bad shape %dx%d", W, H);
        return SV_ERR_SHAPE;
    }
    return SV_OK;
}

}  // namespace

extern "C" {

size_t sv_median_workspace_size(int W, int H) {
    if (W < 1 || H < 1) return 0;
    Carver cv(nullptr);
    cv.take<DevFlags>(1);
    cv.take<double>((size_t)W * H);
    return cv.off;
}

int sv_median_filter(const double *disp, int W, int H, int radius, int passes, double *out,
                     void *workspace, size_t workspace_bytes, void *stream) {
    if (!disp || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (disp == out) { set_error("median_filter: out must not alias disp"); return SV_ERR_PARAM; }
    SV_TRY_POST(check_shape(W, H));
    SV_TRY_POST(check_ws_post(workspace, workspace_bytes, sv_median_workspace_size(W, H)));
    Carver cv(workspace);
    cv.take<DevFlags>(1);
    double *tmp = cv.take<double>((size_t)W * H);
    return launch_median(disp, W, H, radius, passes, out, tmp, (cudaStream_t)stream);
}

size_t sv_postproc_workspace_size(int W, int H, int step) {
    if (W < 1 || H < 1 || step < 1) return 0;
    return carve_post(nullptr, W, H, step, nullptr);
}

int sv_slic_count(int W, int H, int step) {
    if (W < 1 || H < 1 || step < 1) return 0;
    int a, b;
    return slic_grid(W, H, step, &a, &b);
}

int sv_slic(const double *rgb, int W, int H, int step, double compactness, int iters,
            int32_t *labels, void *workspace, size_t workspace_bytes, void *stream) {
    if (!rgb || !labels) { set_error("NULL argument"); return SV_ERR_NULL; }
    SV_TRY_POST(check_shape(W, H));
    if (step < 1) { set_error("step %d", step); return SV_ERR_PARAM; }
    SV_TRY_POST(check_ws_post(workspace, workspace_bytes, sv_postproc_workspace_size(W, H, step)));
    PostWs w;
    carve_post(workspace, W, H, step, &w);
    cudaStream_t st = (cudaStream_t)stream;
    SV_TRY_POST(launch_slic(rgb, W, H, step, compactness, iters, w, st));
    SV_CUDA_TRY(cudaMemcpyAsync(labels, w.lab, sizeof(int32_t) * W * H, cudaMemcpyDeviceToDevice,
                                st));
    return SV_OK;
}

int sv_plane_snap(const double *disp, const double *rgb, int W, int H, const uint8_t *valid,
                  int step, double thr, double min_inl, int trials, uint32_t seed, double *out,
                  void *workspace, size_t workspace_bytes, void *stream) {
    if (!disp || !rgb || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (disp == out) { set_error("plane_snap: out must not alias disp"); return SV_ERR_PARAM; }
    SV_TRY_POST(check_shape(W, H));
    if (step < 1) { set_error("step %d", step); return SV_ERR_PARAM; }
    SV_TRY_POST(check_ws_post(workspace, workspace_bytes, sv_postproc_workspace_size(W, H, step)));
    PostWs w;
    carve_post(workspace, W, H, step, &w);
    return launch_plane_snap(disp, rgb, W, H, valid, step, thr, min_inl, trials, seed, out, w,
                             (cudaStream_t)stream);
}

size_t sv_refine_disparity_workspace_size(int W, int H, const sv_refine_params *p,
                                          int plane_step) {
    const size_t a = sv_lr_refine_workspace_size(W, H, p);
    const size_t b = sv_postproc_workspace_size(W, H, plane_step < 1 ? 1 : plane_step);
    if (!a || !b) return 0;
    return align256(a) + b;
}

int sv_refine_disparity(const void *left, const void *right, int dtype, const double *rgb,
                        const double *disp0, int W, int H, double tol,
                        const sv_refine_params *p, int planes, int plane_step, double plane_thr,
                        double plane_min_inl, double *out, uint8_t *status, void *workspace,
                        size_t workspace_bytes, void *stream) {
    if (!out || !status) { set_error("NULL argument"); return SV_ERR_NULL; }
    SV_TRY_POST(check_shape(W, H));
    if (plane_step < 1) { set_error("plane_step %d", plane_step); return SV_ERR_PARAM; }
    const size_t a = sv_lr_refine_workspace_size(W, H, p);
    if (!a) return sv_lr_refine(left, right, dtype, disp0, W, H, tol, p, out, status, nullptr, 0,
                                stream);   // reports the parameter error
    const size_t need = sv_refine_disparity_workspace_size(W, H, p, plane_step);
    SV_TRY_POST(check_ws_post(workspace, workspace_bytes, need));
    cudaStream_t st = (cudaStream_t)stream;
    char *base = static_cast<char *>(workspace);
    SV_TRY_POST(sv_lr_refine(left, right, dtype, disp0, W, H, tol, p, out, status, base,
                             align256(a), stream));
    PostWs w;
    carve_post(base + align256(a), W, H, plane_step, &w);
    const long N = (long)W * H;
    if (planes && rgb) {
        SV_TRY_POST(launch_status_valid(status, N, w.valid, st));
        SV_TRY_POST(launch_plane_snap(out, rgb, W, H, w.valid, plane_step, plane_thr,
                                      plane_min_inl, 40, 12345u, w.tmp, w, st));
    } else {
        SV_CUDA_TRY(cudaMemcpyAsync(w.tmp, out, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    }
    // median_filter(d, W, H, radius=1, passes=1) from tmp into out
    return launch_median(w.tmp, W, H, 1, 1, out, nullptr, st);
}

}  // extern "C"

extern "C" {

int sv_lr_consistency(const double *disp_l, const double *disp_r, int W, int H, double tol,
                      uint8_t *valid, unsigned long long *kept, void *stream) {
    if (!disp_l || !disp_r || !valid || !kept) { set_error("NULL argument"); return SV_ERR_NULL; }
    SV_TRY_POST(check_shape(W, H));
    return launch_lr_consistency(disp_l, disp_r, W, H, tol, valid, kept, (cudaStream_t)stream);
}

size_t sv_fill_invalid_workspace_size(int W, int H) {
    if (W < 1 || H < 1) return 0;
    Carver cv(nullptr);
    cv.take<int>((size_t)W * H);
    return cv.off;
}

int sv_fill_invalid(const double *disp, const uint8_t *valid, int W, int H, double *out,
                    void *workspace, size_t workspace_bytes, void *stream) {
    if (!disp || !valid || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (disp == out) { set_error("fill_invalid: out must not alias disp"); return SV_ERR_PARAM; }
    SV_TRY_POST(check_shape(W, H));
    SV_TRY_POST(check_ws_post(workspace, workspace_bytes, sv_fill_invalid_workspace_size(W, H)));
    return launch_fill_invalid(disp, valid, W, H, static_cast<int *>(workspace), out,
                               (cudaStream_t)stream);
}

}  // extern "C"
