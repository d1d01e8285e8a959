// sv_refine.cuh -- host launchers of the refinement kernels (sv_refine.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sv {

int launch_base(const double *disp0, long N, int32_t *base, int *flag, cudaStream_t st);
int launch_census(const void *img0, const void *img1, int dtype, int W, int H, int rx,
                  int ry, uint64_t *out0, uint64_t *out1, cudaStream_t st);
int launch_band_costs(const uint64_t *cl, const uint64_t *cr, const int32_t *base0,
                      const int32_t *base1, int W, int H, int R, int invalid, uint8_t *C0,
                      uint8_t *C1, int nviews, cudaStream_t st);
int launch_sgm(const uint8_t *C0, const uint8_t *C1, const int32_t *b0, const int32_t *b1,
               int W, int H, int K, int P1, int P2, void *Lout, bool l16, int nviews,
               int npaths, cudaStream_t st);
int launch_sgm_add_path(const uint8_t *C, const int32_t *base, int W, int H, int K, int P1,
                        int P2, int dir, uint16_t *S, cudaStream_t st);
int launch_wta(const void *L, bool l16, int npaths, int nviews, int W, int H, int R,
               const int32_t *b0, const int32_t *b1, const double *d00, const double *d01,
               double uniq, double *out0, double *out1, double *conf0, cudaStream_t st);
int launch_left_to_right(const double *dl, int W, int H, double *dr, int32_t *base_r,
                         cudaStream_t st);
int launch_lr_check(const double *dl, const double *dr, const double *disp0, int W, int H,
                    double tol, double *out, uint8_t *status, cudaStream_t st);

}  // namespace sv
