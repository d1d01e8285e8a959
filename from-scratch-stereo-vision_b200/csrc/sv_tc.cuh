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
struct TcConv {
    int mode, nd, nimg;
    int IC, OC, K, Kpad;       // K = IC * taps (taps = 9 or 27), Kpad = K rounded up to 16
    int D, H, W;               // input extent (mode 1: disparities and feature size)
    int OD, OH, OW;            // output extent
    int stride, pad, dil;
    int act;                   // 0 none, 1 leaky 0.2
    const float *x[2];
    float *y[2];
    const uint16_t *wB;        // tc_pack_weights layout, Kpad x 16 BF16
    const float *bias;         // OC FP32
    int *err;                  // device error flag (first error wins)
};

inline int tc_kpad(int K) { return (K + 15) / 16 * 16; }
// BF16 elements of one packed weight block.
inline size_t tc_weight_elems(int K) { return (size_t)tc_kpad(K) * 16; }
// Host: FP64 weights [OC][K] (OC <= 16) -> packed BF16 operand B.
void tc_pack_weights(const double *w, int OC, int K, uint16_t *out);
int launch_conv_tc(const TcConv &a, cudaStream_t st);

}  // namespace sv
