// sv_network.cuh -- network kernels' host launchers (sv_network.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "sv_b200.h"

namespace sv {

struct Taps {
    int i00, i01, i10, i11;
    double w00, w01, w10, w11;
};

// BilinearUpsample.forward tap computation, stereonet.py:921-949.
__device__ __forceinline__ Taps bilinear_taps(int oy, int ox, int H, int W, int H2,
                                              int W2) {
    double sy = __ddiv_rn((double)H, (double)H2);
    double sx = __ddiv_rn((double)W, (double)W2);
    double fy = __dsub_rn(__dmul_rn(__dadd_rn((double)oy, 0.5), sy), 0.5);
    if (fy < 0.0) fy = 0.0;
    int y0 = (int)fy;
    if (y0 > H - 1) y0 = H - 1;
    int y1 = y0 + 1 < H ? y0 + 1 : y0;
    double wy = __dsub_rn(fy, (double)y0);
    double fx = __dsub_rn(__dmul_rn(__dadd_rn((double)ox, 0.5), sx), 0.5);
    if (fx < 0.0) fx = 0.0;
    int x0 = (int)fx;
    if (x0 > W - 1) x0 = W - 1;
    int x1 = x0 + 1 < W ? x0 + 1 : x0;
    double wx = __dsub_rn(fx, (double)x0);
    Taps t;
    t.w00 = __dmul_rn(__dsub_rn(1.0, wy), __dsub_rn(1.0, wx));
    t.w01 = __dmul_rn(__dsub_rn(1.0, wy), wx);
    t.w10 = __dmul_rn(wy, __dsub_rn(1.0, wx));
    t.w11 = __dmul_rn(wy, wx);
    t.i00 = y0 * W + x0;
    t.i01 = y0 * W + x1;
    t.i10 = y1 * W + x0;
    t.i11 = y1 * W + x1;
    return t;
}

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
    // optional, [h][w]: the soft-argmin distribution's spread (std, quarter
    // px) and peak probability (both or neither)
    float *qspread, *qpmax;
    // optional: the network's output convolution also runs this width
    // decision over the values it writes (its state cleared beforehand)
    const struct SelFuse *decide;
};

struct SelState;
struct WidthRule;
struct WidthFuse;

// A full-resolution select whose pass 0 runs inside a network stage: the
// stage's resize starts the selection of `rank` (state and histograms
// cleared), the kernel writing the FP64 map histograms its values, and
// launch_select_after_pass0 finishes it.
struct SelFuse {
    SelState *state;
    unsigned *hist;         // the select's histogram words (select_hist_words)
    long long rank;
    const WidthFuse *width = nullptr;   // a width decision instead of the value
    double *mirror = nullptr;           // the decision's host-visible copy
};

// gh (optional): also avgpool2 of the resized left view, [H2/2][W2/2]
int launch_resize_pair(const void *l, const void *r, int dtype, int W, int H, int W2, int H2,
                       float *lo, float *ro, cudaStream_t st, float *gh = nullptr,
                       const SelFuse *fuse = nullptr);
int launch_work_outputs(const float *d, int Ww, int Hw, int W, int H, double inv,
                        double *work64, double *full64, cudaStream_t st,
                        const SelFuse *fuse = nullptr);
int launch_to_f32_pair(const void *l, const void *r, int dtype, long n, float *lo, float *ro,
                       cudaStream_t st);
int launch_resize_f64(const double *x, int W, int H, int W2, int H2, double *out,
                      cudaStream_t st);
int launch_upscale_disp(const float *dw, int Ww, int Hw, int W, int H, double inv, double *out,
                        cudaStream_t st);
int launch_promote(const float *x, long n, double *out, cudaStream_t st);
// bilinear resample of an FP32 map to FP64 (resize_gray's arithmetic), no scaling
int launch_resize_f32(const float *x, int W, int H, int W2, int H2, double *out,
                      cudaStream_t st);
int launch_avgpool2(const float *img, int H, int W, float *out, cudaStream_t st);
int launch_avgpool2_f64(const double *img, int C, int H, int W, double *out, cudaStream_t st);
int launch_forward(const NetView &n, const float *left, const float *right, int H, int W,
                   const float *gh, const float *gf, float *d0, float *d1, float *d2,
                   const FwdBufs &b, int precision, cudaStream_t st);

// ------------------------------------------------ batched predict_auto
// (sv_netbatch.cuh describes the scheme.)  Kernels of one stage, in launch
// order; a stage's CTA prefix tables are indexed by these.
enum NetKind { NK_RESIZE, NK_C1, NK_C2, NK_V1, NK_V2, NK_SA, NK_R0, NK_R0F, NK_R1, NK_R1F,
               NK_C1W, NK_C2W, NK_COUNT };
struct NetPair;
struct NetLaunch;

// One stage (the probe, or a pass) of a batched predict_auto.
struct NetStageLaunch {
    const long long *pre[NK_COUNT];   // device CTA prefixes, [n+1] each
    long long total[NK_COUNT];        // CTAs of each launch
    const NetPair *pairs;
    int n;
    long long slab;
};

// Pair 0's network scratch (the other pairs' sit `slab` bytes apart).
struct NetSlab {
    float *lw, *rw, *gh, *d0, *d1, *d2;
    FwdBufs f;
    double *full;
    SelState *sel;
    unsigned *hist;
};

int net_stage_ctas(const NetView &n, int Hm, int Wm, long long *ctas);
const NetView &net_view(const sv_net *net);
int launch_b_resize(const NetStageLaunch &g, const void *const *lt, const void *const *rt,
                    int dtype, const NetSlab &s, bool with_sel, cudaStream_t st);
int launch_b_forward(const NetView &n, const NetStageLaunch &g, const NetSlab &s,
                     cudaStream_t st);
// A CTA of the batched map kernel covers 32 columns x 8 * kWorkRowsBatched
// rows of its pair's full-resolution map.
constexpr int kWorkRowsBatched = 8;
// rule_width > 0: each pair's width decision (predict_auto's rule with
// target and max_width = rule_width) instead of pass 0 of its value select.
int launch_b_work_outputs(const NetLaunch &L, long long total, const NetSlab &s, bool with_sel,
                          double target, int rule_width, cudaStream_t st);
// The probe's select (one CTA per pair) and passes 1..5 of the
// full-resolution select after the pass's work outputs ran pass 0.
int launch_b_sel_probe(const NetLaunch &L, const NetSlab &s, cudaStream_t st);
// The probe's width decision of every pair (one CTA each, rule with scale W / pw).
int launch_b_width_probe(const NetLaunch &L, const NetSlab &s, double target, int max_width,
                         cudaStream_t st);
int launch_b_sel_rest(const NetLaunch &L, long long total, const NetSlab &s, cudaStream_t st);
long long select_ctas(long n);

// Passes 1.. of a select whose pass 0 a network stage ran (SelFuse), n >
// select_small_cap().
int launch_select_after_pass0(const double *x, long n, SelState *state, unsigned *hist,
                              cudaStream_t st, double *mirror = nullptr);
long select_small_cap();
// The rank-th smallest of x into state's value; with mirror (a device
// pointer, e.g. to mapped pinned host memory) the last kernel also stores
// the value there.
int launch_select(const double *x, long n, long long rank, SelState *state, unsigned *hist,
                  cudaStream_t st, double *mirror = nullptr);
// the same over FP32 values (exactly their FP64 promotions), n <= 16384
// predict_auto's width decision over a whole map (clears the state and
// histogram first when it needs them).
template <typename T>
int launch_width_map(const T *x, long n, const WidthFuse &f, SelState *state, unsigned *hist,
                     cudaStream_t st, double *mirror);

int launch_select_small_f32(const float *x, long n, long long rank, SelState *state,
                            cudaStream_t st, double *mirror = nullptr);
size_t select_state_bytes();
size_t select_value_offset();
size_t select_hist_words();

}  // namespace sv
