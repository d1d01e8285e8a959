// sv_tc.cuh -- BF16 tensor-core (tcgen05) implicit-GEMM convolutions
// (sv_tc.cu): the network's BF16 precision for the feature tower and the
// cost filter's first two 3-D convolutions.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace sv {

// One convolution launch.  Tensors are [channels][D][H][W] FP32 (D = 1 for
// 2-D); the GEMM operands are rounded to BF16, accumulation is FP32.
//  mode 0: y[i] = act(conv(x[i]) + bias) for the nimg images i;
//  mode 1: y[0] = act(conv3d(V) + bias) where V is the cost volume of the
//          feature maps x[0] (left) and x[1] (right) with D disparities:
//          V[c][d][y][x] = |x0[c][y][x] - x1[c][y][x-d]|, or 2 where x < d
//          (CostVolume, stereonet.py:803-825).
//  nb > 1 batches items: item i of side s reads x[s] + i * xs and writes
//  y[s] + i * ys (aux + i * ys).
struct TcConv {
    int mode, nd, nimg;
    int IC, OC, K, Kpad;       // K = IC * taps (taps = 9 or 27), Kpad = K rounded up to 16
    int D, H, W;               // input extent (mode 1: disparities and feature size)
    int OD, OH, OW;            // output extent
    int stride, pad, dil;
    int act;                   // 0 none, 1 leaky 0.2, 2 times leaky'(aux): aux > 0 ? 1 : 0.2
    const float *x[2];
    float *y[2];
    const uint16_t *wB;        // tc_pack_weights layout, Kpad x 16 BF16
    const float *bias;         // OC FP32 (may be NULL: no bias)
    int *err;                  // device error flag (first error wins)
    int nb;                    // batch items per side (0 counts as 1)
    long xs, ys;               // element strides between batch items
    const float *aux;          // act 2: [OC][positions] per item, strided like y
};

// Weight gradient of a 3x3 stride-1 "same" convolution (pad = dil) on the
// tensor cores: gw[o][c][t] += sum over pixels of g[o][p] * x[c][p + tap t],
// gb[o] += sum of g[o][p], over nb items ([IC][H][W] and [OC][H][W] each).
struct TcWgrad {
    int IC, OC, dil, H, W, nb;
    long xs, gs;
    const float *x, *g;
    float *gw, *gb;
    int *err;
};
int launch_wgrad_tc(const TcWgrad &a, cudaStream_t st);

// Device-side packing of FP32 weights [OC][IC][3][3] into operand B:
// forward (n = o, k = c*9 + t) and, for the input gradient, transposed and
// flipped (n = c, k = o*9 + (8 - t)).
int launch_pack_weights(const float *w, int OC, int IC, int transpose, uint16_t *out,
                        cudaStream_t st);

inline int tc_kpad(int K) { return (K + 15) / 16 * 16; }
// BF16 elements of one packed weight block.
inline size_t tc_weight_elems(int K) { return (size_t)tc_kpad(K) * 16; }
// Host: FP64 weights [OC][K] (OC <= 16) -> packed BF16 operand B.
void tc_pack_weights(const double *w, int OC, int K, uint16_t *out);
int launch_conv_tc(const TcConv &a, cudaStream_t st);
// One CTA that holds tensor memory and waits at most `limit` polls on an
// mbarrier nothing arrives at; *flag gets SV_ERR_TIMEOUT, *done 1 (gave up)
// or 2 (the barrier completed).
int launch_selftest_wait(unsigned limit, int *flag, int *done, cudaStream_t st);

}  // namespace sv
