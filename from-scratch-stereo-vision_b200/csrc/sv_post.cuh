// sv_post.cuh -- median_filter, SLIC and plane_snap launchers (sv_post.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace sv {

struct DevFlags;

// Workspace of the post-processing of one W x H disparity map.
struct PostWs {
    DevFlags *flags;
    unsigned char *cs;          // SLIC centres
    int4 *win;                  // each cluster's window of the last assignment
    double *acc;                // exact single-thread update path
    unsigned long long *dist;   // per-pixel minimum distance bits
    int *labtmp, *lab;          // assignment scratch, labels
    int *flag;                  // "a pixel was not covered" in the current iteration
    int *count, *start, *list;  // segment sizes, offsets, pixel lists in index order
    int *pts, *inl;             // per segment: valid pixels, inliers (same offsets)
    int *nvalid;
    uint32_t *state;            // per segment: xorshift32 state at its first draw
    uint8_t *valid;             // status == 0 (refine_disparity)
    double *tmp;                // intermediate disparity
};

#define SV_TRY_POST(expr)             \
    do {                              \
        int rc_ = (expr);             \
        if (rc_ != 0) return rc_;     \
    } while (0)

int slic_grid(int W, int H, int step, int *ncx, int *ncy);
double slic_m2(double compactness, int step);
size_t carve_post(void *ws, int W, int H, int step, PostWs *o);
int launch_median(const double *in, int W, int H, int radius, int passes, double *out,
                  double *tmp, cudaStream_t st);
int launch_slic(const double *rgb, int W, int H, int step, double compactness, int iters,
                const PostWs &w, cudaStream_t st);
int launch_plane_snap(const double *disp, const double *rgb, int W, int H, const uint8_t *valid,
                      int step, double thr, double min_inl, int trials, uint32_t seed,
                      double *out, const PostWs &w, cudaStream_t st);
int launch_status_valid(const uint8_t *status, long N, uint8_t *valid, cudaStream_t st);
int launch_mirror(const void *in, int esize, int W, int H, void *out, cudaStream_t st);
int launch_lr_consistency(const double *dl, const double *dr, int W, int H, double tol,
                          uint8_t *valid, unsigned long long *kept, cudaStream_t st);
int launch_fill_invalid(const double *disp, const uint8_t *valid, int W, int H, int *scratch,
                        double *out, cudaStream_t st);

}  // namespace sv
