// sv_network.cuh -- network kernels' host launchers (sv_network.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace sv {

// Device pointers of one uploaded checkpoint (FP32 copies of the FP64
// parameters), in StereoNet.all_params() order.
struct NetView {
    int C, Cm, D, Rc, ndil;
    int dil[8];
    const float *fw[4], *fb[4];          // FeatureNet c1..c4
    const float *cw[3], *cb[3];          // CostFilter c1..c3
    const float *rw[2][9], *rb[2][9];    // Refinement levels: ndil convs + final
    // BF16 precision: tensor-core operand B of FeatureNet c1..c4 and
    // CostFilter c1, c2 (sv_tc.cuh layout)
    const uint16_t *tw[6];
};

// Scratch of one forward at (H, W).
struct FwdBufs {
    float *fa[2], *fb[2];    // feature maps, left/right
    float *v0, *v1;          // filtered cost volumes [Cm][D][h][w]
    float *rin, *ra, *rb;    // refinement input [2][H][W] and ping-pong [Rc][H][W]
    int *flag;               // device error flag (the workspace's DevFlags)
};

int launch_resize_pair(const void *l, const void *r, int dtype, int W, int H, int W2, int H2,
                       float *lo, float *ro, cudaStream_t st);
int launch_to_f32_pair(const void *l, const void *r, int dtype, long n, float *lo, float *ro,
                       cudaStream_t st);
int launch_resize_f64(const double *x, int W, int H, int W2, int H2, double *out,
                      cudaStream_t st);
int launch_upscale_disp(const float *dw, int Ww, int Hw, int W, int H, double inv, double *out,
                        cudaStream_t st);
int launch_promote(const float *x, long n, double *out, cudaStream_t st);
int launch_avgpool2(const float *img, int H, int W, float *out, cudaStream_t st);
int launch_avgpool2_f64(const double *img, int C, int H, int W, double *out, cudaStream_t st);
int launch_forward(const NetView &n, const float *left, const float *right, int H, int W,
                   const float *gh, const float *gf, float *d0, float *d1, float *d2,
                   const FwdBufs &b, int precision, cudaStream_t st);

struct SelState;
int launch_select(const double *x, long n, long long rank, SelState *state, unsigned *hist,
                  cudaStream_t st);
size_t select_state_bytes();
size_t select_value_offset();
size_t select_hist_words();

}  // namespace sv
