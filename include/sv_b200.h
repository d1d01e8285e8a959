/*
 * sv_b200.h -- C ABI of the B200 (sm_100a) disparity hot path.
 *
 * Each entry point replaces one function of the reference's stereonet.py
 * (Ray-5106/From-Scratch-Stereo-Vision); the comment above it names the
 * reference lines.  Conventions:
 *
 *  - All image-sized buffers are row-major [H][W], device pointers owned by
 *    the caller.  "K" is the band width 2R+1; band arrays are [H][W][K].
 *  - Work is enqueued on `stream` (a cudaStream_t, 0 = legacy default).
 *    Nothing synchronises unless the comment says so.
 *  - Scratch memory comes from a caller-owned workspace whose size the
 *    matching *_workspace_size() call returns (256-byte aligned pointer).
 *    The library itself allocates device memory only for network weights
 *    (sv_net_create).
 *  - Every call returns an SV_* status.  Argument errors are detected before
 *    anything is enqueued.  Errors that depend on data (a NaN disparity) are
 *    recorded in the workspace by the kernels and returned by
 *    sv_workspace_status(), which synchronises the stream.
 *  - Reentrant: no global mutable state; sv_last_error() is thread-local.
 */
#ifndef SV_B200_H
#define SV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum sv_status {
    SV_OK = 0,
    SV_ERR_SHAPE = 1,     /* W, H, R or census window outside the supported range   */
    SV_ERR_PARAM = 2,     /* a parameter the exact integer path cannot honour        */
    SV_ERR_DISP = 3,      /* a disparity is NaN, infinite or |d| >= 2^30             */
    SV_ERR_WORKSPACE = 4, /* workspace NULL, misaligned or smaller than required     */
    SV_ERR_CUDA = 5,      /* a CUDA runtime call failed (detail in sv_last_error)    */
    SV_ERR_NULL = 6,      /* a required pointer is NULL                               */
    SV_ERR_NET = 7,       /* weights do not match the architecture                    */
    SV_ERR_TIMEOUT = 8    /* a bounded device wait or host poll gave up               */
};

enum sv_dtype { SV_U8 = 0, SV_F32 = 1, SV_F64 = 2 };

/* Network arithmetic (sv_stereonet_forward and the predict_* calls). */
enum sv_precision { SV_FP32 = 0, SV_BF16 = 1 };

const char *sv_status_string(int status);
const char *sv_last_error(void);
int sv_version(void);

/* Number of kernels this library has launched in this process, on any
 * device (a reporting counter; the difference across a region is that
 * region's launch count).  No reference counterpart. */
unsigned long long sv_launch_count(void);

/* Refinement parameters, the keyword arguments of refine_fullres
 * (stereonet.py:5244-5246).  The exact integer path requires ad_weight == 0,
 * prior_w == 0 and integer-valued 0 <= P1, P2 <= 4096 (every value the
 * reference's pipeline uses: refine_disparity passes P1=12, P2=150). */
typedef struct sv_refine_params {
    int R;            /* band half-width, K = 2R+1, 0 <= R <= 126           */
    double P1, P2;    /* SGM penalties                                      */
    int rx, ry;       /* census window half-sizes, (2rx+1)(2ry+1)-1 <= 64   */
    int paths;        /* 8 or 4                                             */
    double uniq;      /* uniqueness threshold (0 disables)                  */
    double ad_weight; /* must be 0                                          */
    double ad_trunc;
    double prior_w;   /* must be 0                                          */
    double prior_t;
} sv_refine_params;

/* refine_fullres's own defaults (R=3, P1=1, P2=12, rx=ry=2, 8 paths). */
void sv_refine_params_default(sv_refine_params *p);

/* Returns the first data-dependent error the kernels recorded in this
 * workspace since the last sv_* call that used it (synchronises stream). */
int sv_workspace_status(const void *workspace, void *stream);

/* census, stereonet.py:5115-5142.  img is [H][W] of `dtype` (gray values,
 * compared exactly as stored).  out[p] has bit (nbits-1-i) set when the i-th
 * window offset (dy-major, dx-minor, centre skipped) is darker than the
 * centre; borders clamp to the edge.  Bit-identical to the reference. */
int sv_census(const void *img, int dtype, int W, int H, int rx, int ry,
              uint64_t *out, void *stream);

/* band_costs, stereonet.py:5156-5189, for ad_weight = 0 and no prior term:
 * C[p][k] = popcount(cl[p] ^ cr[p - (base[p]-R+k)]), or `invalid` (0..255;
 * refine_fullres passes nbits+4) where that column is outside the image or
 * the candidate is negative.  base is int32 [H][W]. */
int sv_band_costs(const uint64_t *cl, const uint64_t *cr, const int32_t *base,
                  int W, int H, int R, int invalid, uint8_t *C, void *stream);

/* _aggregate_path, stereonet.py:5192-5241: S += L for direction (dx, dy)
 * with integer penalties.  C is uint8 [H][W][K], S uint16 [H][W][K]. */
int sv_aggregate_path(const uint8_t *C, const int32_t *base, int W, int H, int K,
                      int P1, int P2, int dx, int dy, uint16_t *S, void *stream);

/* left_to_right, stereonet.py:5317-5340 (FP64, bit-identical). */
int sv_left_to_right(const double *dl, int W, int H, double *dr, void *stream);

/* refine_fullres, stereonet.py:5244-5305 (one view, bit-identical output).
 * left/right are [H][W] of `dtype`; disp0 and out are FP64 [H][W];
 * conf (optional, may be NULL) receives the return_conf values. */
size_t sv_refine_workspace_size(int W, int H, const sv_refine_params *p);
int sv_refine_fullres(const void *left, const void *right, int dtype,
                      const double *disp0, int W, int H,
                      const sv_refine_params *p, double *out, double *conf,
                      void *workspace, size_t workspace_bytes, void *stream);

/* lr_refine, stereonet.py:5343-5391: both views, left-right check and the
 * occlusion / mismatch fills.  status: 0 ok, 1 occluded, 2 mismatch. */
size_t sv_lr_refine_workspace_size(int W, int H, const sv_refine_params *p);
int sv_lr_refine(const void *left, const void *right, int dtype,
                 const double *disp0, int W, int H, double tol,
                 const sv_refine_params *p, double *out, uint8_t *status,
                 void *workspace, size_t workspace_bytes, void *stream);

/* sv_lr_refine with stage timing for profiling: events[0..SV_LR_STAGES] are
 * caller-created cudaEvent_t recorded on `stream` before the first kernel
 * and after each stage (base + left_to_right, census, band costs, SGM, WTA,
 * left-right check), so cudaEventElapsedTime(events[i], events[i+1]) is the
 * device time of stage i.  Same results as sv_lr_refine. */
#define SV_LR_STAGES 6
int sv_lr_refine_timed(const void *left, const void *right, int dtype,
                       const double *disp0, int W, int H, double tol,
                       const sv_refine_params *p, double *out, uint8_t *status,
                       void *workspace, size_t workspace_bytes, void *stream,
                       void *const *events, int n_events);

/* lr_refine over many pairs of uneven sizes (the batched form of
 * stereonet.py:5343-5391 that serves callers such as eval_real.evaluate,
 * eval_real.py:133-152, over a whole test split).  Each pair's outputs are
 * bit-identical to sv_lr_refine on that pair alone; the work runs as one
 * launch per stage, the SGM stage as a persistent kernel over a device-side
 * queue of (pair, view, path, scanline) tasks, longest scanlines first.
 * Bands up to K = 30 (R <= 14).  `pairs` is a host array; its pointers are
 * device buffers.  The tables are copied from host memory during the call. */
typedef struct sv_pair_desc {
    const void *left, *right;   /* [H][W] of the call's dtype  */
    const double *disp0;        /* [H][W] network disparity    */
    double *out;                /* [H][W] refined disparity    */
    uint8_t *status;            /* [H][W] 0 ok, 1 occluded, 2 mismatch */
    int W, H;
} sv_pair_desc;
size_t sv_batch_lr_refine_workspace_size(const sv_pair_desc *pairs, int n,
                                         const sv_refine_params *p);
int sv_batch_lr_refine(const sv_pair_desc *pairs, int n, int dtype, double tol,
                       const sv_refine_params *p, void *workspace,
                       size_t workspace_bytes, void *stream);

/* Scheduling of sv_batch_lr_refine_ex (results do not depend on it): pixels
 * per CTA of the per-pixel stages (base, band costs, WTA, left-right check;
 * a power of 2 in 256..8192), threads per CTA of the persistent SGM kernel
 * (32/64/128/256), its CTAs per SM (1..32), and the scanline tasks a warp
 * claims per fetch from the queue (32/64/128).  batch.autotune picks them by
 * timing the caller's batch.  No reference counterpart. */
typedef struct sv_batch_config {
    int px_per_block;
    int sgm_threads;
    int sgm_ctas_per_sm;
    int sgm_fetch;
} sv_batch_config;
/* 2048, 128, 8, 32: what sv_batch_lr_refine uses */
void sv_batch_config_default(sv_batch_config *cfg);
int sv_batch_lr_refine_ex(const sv_pair_desc *pairs, int n, int dtype, double tol,
                          const sv_refine_params *p, const sv_batch_config *cfg,
                          void *workspace, size_t workspace_bytes, void *stream);

/* refine_fullres for callers that cannot allocate device memory (an engine
 * that reserves all GPU memory up front, a plugin host without an
 * allocator): same kernels and bit-identical output as sv_refine_fullres,
 * but the scratch is one static device array of SV_NOALLOC_SCRATCH_BYTES
 * inside this library, held on every GPU that loads it until exit.  No
 * counterpart in the reference (it is an allocation-free variant of this
 * library's own sv_refine_fullres).
 *  - Capacity: with N = W*H and Kp = K+2 rounded up to 8, 16, 24, 32, 48,
 *    64, 96, 128, 192 or 256, the scratch needs 256 + 4N + 2*8N + N*Kp +
 *    npaths*N*Kp*b bytes (b = 1, or 2 when 4 + nbits + P2 > 255), each term
 *    rounded up to 256.  At refine_disparity's parameters (K = 21, Kp = 24,
 *    8 paths, b = 1) that is 236 bytes per pixel: up to about 71,000 pixels
 *    (300x236 fits, 320x240 does not); paths = 4 needs 140 bytes per pixel.
 *    Larger sizes return SV_ERR_SHAPE and run nothing.
 *  - The array's device address is resolved (cudaGetSymbolAddress) on the
 *    first call on a device and again in each new CUDA context on it; make
 *    the first call on a device before any stream capture.
 *  - All calls share the array, which keeps the last call's contents; each
 *    call writes every scratch byte it reads.  Calls that overlap on the GPU
 *    race on it: serialise them.
 *  - data_status (required): a device int, cleared by the call, that
 *    receives SV_ERR_DISP if a disparity is NaN, infinite or out of range;
 *    a NULL data_status returns SV_ERR_NULL. */
#define SV_NOALLOC_SCRATCH_BYTES (16u << 20)
int sv_refine_fullres_noalloc(const void *left, const void *right, int dtype,
                              const double *disp0, int W, int H,
                              const sv_refine_params *p, double *out,
                              int *data_status, void *stream);

/* Failure-path self-tests (no reference counterpart: the reference only
 * raises Python exceptions, serve.py:72-84).  They exercise the bounded waits
 * every long-running path here relies on, without faulting the GPU.
 *  - sv_selftest_wait_timeout: one CTA allocates tensor memory and waits at
 *    most `limit` polls on an mbarrier that nothing arrives at -- the wait of
 *    the tcgen05 convolutions.  flag_done is two device ints: [0] receives
 *    SV_ERR_TIMEOUT (clear it first), [1] becomes 1 once the CTA gave up and
 *    freed its tensor memory (2 if the barrier had completed).
 *  - sv_selftest_slot_wait: polls a mapped host slot that no kernel writes,
 *    on an idle stream -- the host side of predict_auto's peak hand-off --
 *    and returns SV_ERR_TIMEOUT. */
int sv_selftest_wait_timeout(unsigned limit, int *flag_done, void *stream);
int sv_selftest_slot_wait(void *stream);

/* ------------------------------------------------------------ network */
typedef struct sv_net sv_net;

/* Uploads a StereoNet checkpoint.  arch = {feat_C, cost_C, D, refine_C,
 * ndil, dil[0..ndil-1]} (the header fields of save_weights,
 * stereonet.py:1774-1779); params = all blocks concatenated in
 * StereoNet.all_params() order (stereonet.py:1193-1195), FP64.
 * Allocates device memory for the weights (freed by sv_net_destroy). */
int sv_net_create(const int *arch, int n_arch, const double *params,
                  long n_params, sv_net **out);
void sv_net_destroy(sv_net *net);

/* resize_gray / BilinearUpsample.forward, stereonet.py:3843-3845, 913-956:
 * half-pixel bilinear resample computed in FP64. */
int sv_resize(const double *img, int W, int H, int W2, int H2, double *out,
              void *stream);

/* avgpool2, stereonet.py:979-995: 2x2 mean of C planes [C][H][W] into
 * [C][H/2][W/2], FP64 in the reference's order (bit-identical). */
int sv_avgpool2(const double *img, int C, int H, int W, double *out, void *stream);

/* StereoNet.forward, stereonet.py:1203-1233 (note the reference's H, W order).
 * left/right/guide_full are FP32 [H][W], guide_half FP32 [H/2][W/2];
 * d0 [h][w], d1 [H/2][W/2], d2 [H][W] FP32. */
size_t sv_forward_workspace_size(const sv_net *net, int H, int W);
int sv_stereonet_forward(const sv_net *net, const float *left, const float *right,
                         int H, int W, const float *guide_half,
                         const float *guide_full, float *d0, float *d1, float *d2,
                         int precision, void *workspace, size_t workspace_bytes,
                         void *stream);

/* predict_auto, stereonet.py:3872-3929 (with predict_at_scale 3932-3960 and
 * predict 5891-5897).  left/right are the full-resolution gray images of
 * `dtype`.  disp_full: FP64 [H][W]; disp_work: FP64, at least W*H elements.
 * The work-width choice needs the peak of each pass on the host, so this
 * call synchronises the stream once per pass.  *work_trace (optional, at
 * least passes+1 ints) receives the work widths tried, 0-terminated.
 * precision = SV_BF16 applies to the last permitted pass only (the one no
 * work-width decision follows); the probe and the passes whose 95%
 * quantile picks the next width run FP32, so the widths chosen are FP32's. */
size_t sv_predict_workspace_size(const sv_net *net, int W, int H, int max_width);
int sv_predict_auto(const sv_net *net, const void *left, const void *right,
                    int dtype, int W, int H, double target_peak, int probe_width,
                    int max_width, int passes, int precision, double *disp_full,
                    double *disp_work, int *Ww, int *Hw, int *work_trace,
                    void *workspace, size_t workspace_bytes, void *stream);

/* predict_auto followed by lr_refine on its full-resolution disparity: one
 * pair's disparity hot path in one call (the callers' predict_auto then
 * refine_disparity's lr_refine, stereonet.py:3872-3929 and 5865-5872), with
 * no host work between the last work-width read and the refinement's
 * launches.  disp_full receives predict_auto's disparity, out / status
 * lr_refine's; pworkspace is predict_auto's workspace, rworkspace
 * lr_refine's (sv_lr_refine_workspace_size). */
int sv_predict_refine(const sv_net *net, const void *left, const void *right, int dtype,
                      int W, int H, double target_peak, int probe_width, int max_width,
                      int passes, int precision, double *disp_full, double *disp_work,
                      int *Ww, int *Hw, int *work_trace, void *pworkspace,
                      size_t pworkspace_bytes, double tol, const sv_refine_params *p,
                      double *out, uint8_t *status, void *rworkspace,
                      size_t rworkspace_bytes, void *stream);

/* predict_at_scale, stereonet.py:3932-3960. */
int sv_predict_at_scale(const sv_net *net, const void *left, const void *right,
                        int dtype, int W, int H, int work_width, int precision,
                        double *disp_full, double *disp_work, int *Ww, int *Hw,
                        void *workspace, size_t workspace_bytes, void *stream);

/* How sure the network was, per pixel, in the last pass of the
 * sv_predict_auto (or sv_predict_refine) call that used this workspace:
 * the spread (standard deviation, in full-resolution pixels) and the peak
 * probability of its soft-argmin distribution (SoftArgmin.forward,
 * stereonet.py:858-885), bilinearly resampled from the quarter-resolution
 * volume to W x H (FP64).  Ww x Hw is that call's final work size;
 * probe_width and max_width must be the call's.  No reference counterpart:
 * they feed the learned band's net. */
int sv_predict_confidence(const sv_net *net, int W, int H, int Ww, int Hw, int probe_width,
                          int max_width, const void *workspace, size_t workspace_bytes,
                          double *spread, double *pmax, void *stream);

/* predict_auto followed by lr_refine for many pairs of uneven sizes
 * (predict_auto, stereonet.py:3872-3929; lr_refine, 5343-5391), with the
 * work-width decisions taken on the device: the probe, every pass and the
 * peaks between them, and the batched refinement behind them, are one fixed
 * launch sequence, recorded into a CUDA graph by the first run on a
 * capturable stream and replayed afterwards.  Each pair's network
 * disparity, work-width trace and refined output are those of predict_auto
 * and lr_refine run on that pair alone.  FP32 network.
 *  - create: plans the batch for the pairs' sizes (W[i], H[i]) and
 *    predict_auto's / lr_refine's parameters; allocates host memory only.
 *  - bind: the pairs' device buffers (left, right, out, status of each
 *    sv_pair_desc; disp0 is ignored: the network writes it) and a workspace
 *    of sv_netbatch_workspace_size bytes, 256-aligned; uploads the tables
 *    and synchronises the stream.
 *  - run: enqueues the whole batch (no host synchronisation); predict runs
 *    the network part only.
 *  - disparity: device pointer of pair i's network disparity (FP64, W x H).
 *  - trace: each pair's chosen widths (0-terminated, trace_len per pair)
 *    and final work size; synchronises the stream. */
typedef struct sv_netbatch sv_netbatch;
int sv_netbatch_create(const sv_net *net, const int *W, const int *H, int n, int dtype,
                       double target_peak, int probe_width, int max_width, int passes,
                       int precision, double tol, const sv_refine_params *p,
                       sv_netbatch **out);
size_t sv_netbatch_workspace_size(const sv_netbatch *nb);
int sv_netbatch_bind(sv_netbatch *nb, const sv_pair_desc *pairs, void *workspace,
                     size_t workspace_bytes, void *stream);
int sv_netbatch_run(sv_netbatch *nb, void *stream);
int sv_netbatch_predict(sv_netbatch *nb, void *stream);
int sv_netbatch_disparity(const sv_netbatch *nb, int i, const double **disp_full);
int sv_netbatch_trace(const sv_netbatch *nb, int *work_trace, int trace_len, int *work_size,
                      void *stream);
int sv_netbatch_data_status(const sv_netbatch *nb, void *stream);
void sv_netbatch_destroy(sv_netbatch *nb);

/* predict_consistent, stereonet.py:5048-5076 (with mirror_h 4974-4983,
 * lr_consistency 4986-5009, fill_invalid 5012-5045): the network on the pair
 * (predict_auto when work_width <= 0, else predict_at_scale) and on the
 * mirrored pair at the same work width, the left-right check with `tol`, and
 * the row fill of the rejected pixels.  *kept (host) receives the number of
 * consistent pixels (valid fraction = kept / (W H)); the call synchronises
 * the stream. */
size_t sv_predict_consistent_workspace_size(const sv_net *net, int W, int H,
                                            int dtype, int max_width);
int sv_predict_consistent(const sv_net *net, const void *left, const void *right,
                          int dtype, int W, int H, int work_width,
                          double target_peak, int probe_width, int max_width,
                          int passes, double tol, int precision, double *disp_out,
                          long long *kept, void *workspace,
                          size_t workspace_bytes, void *stream);

/* lr_consistency, stereonet.py:4986-5009 (disp_r in the right image's frame):
 * valid[p] = 1 where the two maps agree within tol; *kept (device) receives
 * the count of valid pixels */
int sv_lr_consistency(const double *disp_l, const double *disp_r, int W, int H,
                      double tol, uint8_t *valid, unsigned long long *kept,
                      void *stream);
/* fill_invalid, stereonet.py:5012-5045 */
size_t sv_fill_invalid_workspace_size(int W, int H);
int sv_fill_invalid(const double *disp, const uint8_t *valid, int W, int H,
                    double *out, void *workspace, size_t workspace_bytes, void *stream);

/* ------------------------------------------------------------------------
 * The rest of refine_disparity (stereonet.py:5865-5883), bit-identical.
 * disp / out are FP64 [H][W]; rgb is interleaved FP64 RGB in [0, 1] as
 * read_image gives it; out must not alias the input disparity.
 * ---------------------------------------------------------------------- */
/* median_filter, stereonet.py:2231-2259 (radius <= 3) */
size_t sv_median_workspace_size(int W, int H);
int sv_median_filter(const double *disp, int W, int H, int radius, int passes,
                     double *out, void *workspace, size_t workspace_bytes,
                     void *stream);
/* slic, stereonet.py:5394-5455: labels [H][W] (-1 where no cluster ever
 * covered the pixel); sv_slic_count gives the number of clusters */
size_t sv_postproc_workspace_size(int W, int H, int step);
int sv_slic_count(int W, int H, int step);
int sv_slic(const double *rgb, int W, int H, int step, double compactness,
            int iters, int32_t *labels, void *workspace, size_t workspace_bytes,
            void *stream);
/* plane_snap, stereonet.py:5505-5563 (SLIC with compactness 10, 5 iterations;
 * valid may be NULL; trials <= 64) */
int sv_plane_snap(const double *disp, const double *rgb, int W, int H,
                  const uint8_t *valid, int step, double thr, double min_inl,
                  int trials, uint32_t seed, double *out, void *workspace,
                  size_t workspace_bytes, void *stream);
/* refine_disparity, stereonet.py:5865-5883: lr_refine, plane_snap on the
 * status-0 pixels when planes != 0 and rgb != NULL, 3x3 median */
size_t sv_refine_disparity_workspace_size(int W, int H, const sv_refine_params *p,
                                          int plane_step);
int sv_refine_disparity(const void *left, const void *right, int dtype,
                        const double *rgb, const double *disp0, int W, int H,
                        double tol, const sv_refine_params *p, int planes,
                        int plane_step, double plane_thr, double plane_min_inl,
                        double *out, uint8_t *status, void *workspace,
                        size_t workspace_bytes, void *stream);

/* ------------------------------------------------------------------------
 * Learned adaptive band (no counterpart in the reference: it extends
 * lr_refine, stereonet.py:5343-5391, whose band is fixed at +-R around the
 * network disparity).  A 4-layer convolutional band net (5810 parameters,
 * BF16 tensor-core kernels with FP32 accumulation) reads SV_BAND_FEATURES
 * per-pixel features and predicts a shift of the band centre and a Laplace
 * scale; confident pixels get the shifted centre and a narrower band, the
 * rest keep the fixed band.  Trained with Adam (stereonet.py:1354-1387) on
 * full-range SGM disparities.  All tensors are device buffers, [item][c][H][W].
 * ---------------------------------------------------------------------- */
#define SV_BAND_FEATURES 6
#define SV_BAND_OUTPUTS 2
typedef struct sv_band sv_band;
long sv_band_param_count(void);
int sv_band_create(const double *params, long n_params, sv_band **out);
void sv_band_destroy(sv_band *band);
/* copies the (FP32 master) parameters to host memory as doubles; syncs */
int sv_band_get_params(const sv_band *band, double *out, long n_params);

/* Band-net input planes [8][H][W] FP32.  sv_band_features writes planes
 * 0-5 from the two views (9x7 census) and disp0 (FP64), disparities
 * searched over 0..dmax (dmax <= 255); sv_band_conf_features writes planes
 * 6-7 from the network's spread and peak probability of the same pass
 * (sv_predict_confidence). */
size_t sv_band_features_workspace_size(int W, int H);
int sv_band_features(const void *left, const void *right, int dtype,
                     const double *disp0, int W, int H, int dmax, float *feat,
                     void *workspace, size_t workspace_bytes, void *stream);
int sv_band_conf_features(const double *spread, const double *pmax, int W, int H, float *feat,
                          void *stream);
/* The rule centre the learned band refines around: disp0 + 64 * feat[1]
 * (the wide search's first argmin) where feat[2] (its 9-row census cost /
 * 558) < tau, else disp0 (FP64). */
int sv_band_rule_centre(const float *feat, const double *disp0, int W, int H, double tau,
                        double *centre, void *stream);

/* forward of nb items: feat [nb][8][H][W] -> out [nb][2][H][W] */
size_t sv_band_workspace_size(int nb, int W, int H);
int sv_band_forward(const sv_band *band, const float *feat, int nb, int W, int H,
                    float *out, void *workspace, size_t workspace_bytes,
                    void *stream);
/* loss and gradients (FP32, parameter order) of target [nb][H][W] shifts on
 * the mask [nb][H][W] (1 = labelled); grads / loss (device) may be NULL */
int sv_band_grads(sv_band *band, const float *feat, const float *target,
                  const uint8_t *mask, int nb, int W, int H, float *grads,
                  double *loss, void *workspace, size_t workspace_bytes,
                  void *stream);
/* sv_band_grads followed by one Adam step (b1 0.9, b2 0.999, eps 1e-8,
 * gradient clip 5) at learning rate lr */
int sv_band_train_step(sv_band *band, const float *feat, const float *target,
                       const uint8_t *mask, int nb, int W, int H, double lr,
                       double *loss, void *workspace, size_t workspace_bytes,
                       void *stream);
/* target = clamp(label - disp0, +-shift_max), mask = (status == 0) */
int sv_band_targets(const double *label, const uint8_t *status,
                    const double *disp0, long n, double shift_max, float *target,
                    uint8_t *mask, void *stream);
/* out [2][H][W] of one item -> band centre (FP64) and half-width per pixel:
 * b = exp(clamp(out1 + 1)); b <= b_thr: centre = disp0 + clamp(32 out0),
 * half-width = clamp(ceil(rad_k * b), rad_min, R); else centre = disp0,
 * half-width R */
int sv_band_apply(const float *out, const double *disp0, int W, int H,
                  double b_thr, double rad_k, int rad_min, int R,
                  double shift_max, double *centre, uint8_t *rad, void *stream);
/* lr_refine around `centre` with the left view's band restricted to
 * |k - R| <= rad[p] (other slots cost the invalid value); same workspace as
 * sv_lr_refine.  rad[p] = R everywhere gives sv_lr_refine's result. */
int sv_lr_refine_band(const void *left, const void *right, int dtype,
                      const double *centre, const uint8_t *rad, int W, int H,
                      double tol, const sv_refine_params *p, double *out,
                      uint8_t *status, void *workspace, size_t workspace_bytes,
                      void *stream);

/* _peak (stereonet.py:3866-3869): sorted(disp)[int(len(disp) * q)], floored
 * at 0.5, written to *out (device FP64), exact; disp is device FP64 [n],
 * n < 2^32 (six radix passes over order-preserving 64-bit keys). */
size_t sv_peak_workspace_size(void);
int sv_peak(const double *disp, long n, double q, double *out, void *workspace,
            size_t workspace_bytes, void *stream);

/* predict_auto's work-width decision over a map (stereonet.py:3866-3869
 * _peak, then predict_auto's width rule, stereonet.py:3915-3919): the width
 * int(W * target_peak / max(p, 1e-6) + 0.5) clamped to [48, min(W,
 * max_width)], p = max(sorted(map)[int(n * 0.95)], 0.5) * scale (scale = W
 * / probe width for the probe's map, 1 for a full-size one).  Exact for
 * every map, from a histogram of the widths the rule gives each value (the
 * rule is monotone in the value), without selecting the quantile itself --
 * the way predict_auto decides.  map: device FP64 [n], n < 2^32; at most
 * 2049 possible widths (min(W, max_width) <= 2096).  Synchronises the
 * stream to return *width.  Same workspace as sv_peak. */
int sv_work_width(const double *map, long n, int W, double target_peak, int max_width,
                  double scale, int *width, void *workspace, size_t workspace_bytes,
                  void *stream);

/* ------------------------------------------------------------------------
 * Input images: PNG (stereonet.py:3499-3601 read_png, with zlib_decompress
 * 3421, inflate 3335 and _unfilter 3456) and PGM/PPM (stereonet.py:265-324
 * read_pnm); read_image (3604) picks by the magic bytes.  Decoding runs on
 * the host into raw samples; sv_raw_to_float forms the FP64 images on the
 * GPU, bit-identical to the reference's (gray = 0.299 r + 0.587 g + 0.114 b;
 * a PGM keeps its sample as gray).
 * ---------------------------------------------------------------------- */
#define SV_IMAGE_PNG 1
#define SV_IMAGE_PNM 2
typedef struct sv_raw_image {
    int kind;        /* SV_IMAGE_PNG or SV_IMAGE_PNM                          */
    int width, height;
    int depth;       /* bits per sample in `raw` (PNM: 8, or 16 big-endian)   */
    int colortype;   /* PNG colour type; PNM: 0 (P2/P5) or 2 (P3/P6)          */
    int channels;    /* samples per pixel in `raw`                            */
    int stride;      /* bytes per row of `raw`                                */
    int interlace;   /* PNG IHDR interlace method (only 0 is decoded)         */
    int maxval;      /* PNM maxval                                            */
    int ascii;       /* PNM P2/P3                                             */
    int palette_len; /* PLTE bytes                                            */
    double inv;      /* 1 / (2^depth - 1) for PNG, 1 / maxval for PNM         */
    uint8_t palette[768];
} sv_raw_image;
/* header only (no decompression): fills desc; raw bytes = stride * height */
int sv_image_info(const uint8_t *data, size_t n, sv_raw_image *desc);
/* decodes the file held in host memory into raw samples (host memory,
 * stride * height bytes), rejecting what the reference rejects */
int sv_image_decode_raw(const uint8_t *data, size_t n, uint8_t *raw,
                        size_t raw_bytes, sv_raw_image *desc);
/* sv_image_decode_raw of n files on up to `threads` host threads (decoding
 * is serial within a file; the files are independent).  status[i] (may be
 * NULL) receives each file's code; the first failure is returned and its
 * message is kept for sv_last_error. */
int sv_image_decode_batch(int n, const uint8_t *const *data, const size_t *sizes,
                          uint8_t *const *raw, const size_t *raw_bytes,
                          sv_raw_image *descs, int *status, int threads);
/* device raw samples -> gray [H][W] and rgb [H][W][3] (FP64 device buffers;
 * either may be NULL) */
int sv_raw_to_float(const uint8_t *raw, const sv_raw_image *desc, double *gray,
                    double *rgb, void *stream);

/* ------------------------------------------------------------------------
 * StereoNet training: train_grads (stereonet.py:1619-1653, with
 * build_targets 1572-1611, pseudo_huber 1326-1351, disparity_ce 1274-1323,
 * StereoNet.backward 1235-1267) over a batch of B crops, and Adam.step
 * (1368-1387).  The batch gradient is the mean of the per-sample gradients,
 * as the reference's data-parallel harness forms it (train_parallel.py
 * 144-156); B = 1 is train_grads itself.  FP32 activations and gradients,
 * FP64 parameters, weight-gradient sums and Adam state; deterministic.
 * Architectures: feat_C/cost_C/refine_C 12/6/8 or 8/4/8, D <= 16,
 * dilations <= 8.  Crops: W, H multiples of 4 (the reference's targets
 * line up with its outputs only then) and W/4 > D - 2.
 * ---------------------------------------------------------------------- */
typedef struct sv_trainer sv_trainer;
/* arch as sv_net_create; params (host, FP64) in all_params() order */
int sv_trainer_create(const int *arch, int n_arch, const double *params, long n_params,
                      sv_trainer **out);
void sv_trainer_destroy(sv_trainer *t);
long sv_trainer_param_count(const sv_trainer *t);
/* host copies of the parameters / the last gradient (synchronise) */
int sv_trainer_get_params(const sv_trainer *t, double *out, long n);
int sv_trainer_get_grads(const sv_trainer *t, double *out, long n);
int sv_trainer_set_params(sv_trainer *t, const double *params, long n);
int sv_trainer_set_grads(sv_trainer *t, const double *grads, long n);
size_t sv_train_workspace_size(const sv_trainer *t, int B, int W, int H);
/* left, right, disp: FP32 [B][H][W] (gray in [0, 1], ground-truth
 * disparity); valid: [B][H][W] (nonzero = known).  Leaves the batch
 * gradient in the trainer; loss (device FP64 [B], may be NULL) gets each
 * sample's total loss, pred (device FP32 [B][H][W], may be NULL) the
 * full-resolution prediction. */
int sv_train_grads(sv_trainer *t, const float *left, const float *right, const float *disp,
                   const uint8_t *valid, int B, int W, int H, double *loss, float *pred,
                   void *workspace, size_t workspace_bytes, void *stream);
/* one Adam step (b1 0.9, b2 0.999, eps 1e-8, per-element clip) on the
 * trainer's gradient at learning rate lr */
int sv_train_adam(sv_trainer *t, double lr, double clip, void *stream);
/* zero Adam's moments and restart its bias correction */
int sv_trainer_reset_adam(sv_trainer *t);

#ifdef __cplusplus
}
#endif
#endif /* SV_B200_H */
