// sv_netbatch.cu -- predict_auto followed by lr_refine for a batch of pairs
// of uneven sizes, with every decision on the device (extern "C"
// sv_netbatch_*).
//
// predict_auto (stereonet.py:3872-3929) probes each pair at 64 px wide,
// picks a work width from the probe's 95% disparity quantile, runs the
// network there, re-measures the quantile on the result and reruns while
// the implied width moves by more than 8% (at most `passes` passes).  The
// single-pair path reads each quantile back on the host to size the next
// pass.  Here the quantiles and the width rule run on the device
// (k_nb_decide), every network kernel reads its pair's current work size
// from a NetPair record (sv_netbatch.cuh), and the launch grids cover each
// pair's largest possible work size; so the whole batch -- probe, passes,
// and the batched lr_refine behind them (sv_batch_api.cu) -- is one fixed
// launch sequence, captured once in a CUDA graph and replayed.  Each pair
// gets exactly the arithmetic of the single-pair path, so its disparity,
// work-width trace and refined output are identical to running it alone.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "sv_common.cuh"
#include "sv_netbatch.cuh"
#include "sv_network.cuh"
#include "sv_refine.cuh"
#include "sv_select.cuh"

namespace sv {

// predict_auto's width rule (stereonet.py:3909-3917), FP64 as the host does.
__host__ __device__ inline int nb_width_for(int W, double tp, int max_width, double pk) {
    const double m = pk > 1.0e-6 ? pk : 1.0e-6;
#ifdef __CUDA_ARCH__
    int w = (int)__dadd_rn(__ddiv_rn(__dmul_rn((double)W, tp), m), 0.5);
#else
    int w = (int)((double)W * tp / m + 0.5);
#endif
    if (w > W) w = W;
    if (w > max_width) w = max_width;
    if (w < 48) w = 48;
    return w;
}

// The pass's work size for a requested width (predict_at_scale,
// stereonet.py:3941-3952).
__device__ inline void nb_set_work(NetPair &p, int work) {
    p.work = work;
    if (work >= p.W) {
        p.native = 1;
        p.Ww = p.W;
        p.Hw = p.H;
        p.inv = 1.0;
        return;
    }
    const double scale = __ddiv_rn((double)work, (double)p.W);
    int hw = (int)__dadd_rn(__dmul_rn((double)p.H, scale), 0.5);
    p.native = 0;
    p.Ww = work;
    p.Hw = hw < 8 ? 8 : hw;
    p.inv = __ddiv_rn(1.0, scale);
}

// Before the probe: every pair runs, at its probe size, resampled.
__global__ void k_nb_probe_init(NetPair *pairs, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    NetPair &p = pairs[i];
    p.active = 1;
    p.native = 0;
    p.work = p.pw;
    p.Ww = p.pw;
    p.Hw = p.ph;
    p.inv = 1.0;
    p.ntrace = 0;
    p.peak = 0.0;
}

// After a stage's select: the next pass's width.  stage 0 is the probe
// (its peak scaled by W / pw); stage k > 0 the k-th pass, which stops the
// pair when the width moved by at most 8%.
// by_rule: the stage's decision already holds the width (a width
// decision, not a value select).
__global__ void k_nb_decide(NetPair *pairs, int n, const char *slab0, long long slab,
                            long long sel_off, double tp, int max_width, int stage, int by_rule) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    NetPair &p = pairs[i];
    if (!p.active) return;
    const SelState *s = reinterpret_cast<const SelState *>(slab0 + (long long)i * slab + sel_off);
    const double v = s->value;
    const double pk = v > 0.5 ? v : 0.5;                 // _peak's floor
    p.peak = by_rule ? 0.0 : pk;
    if (stage == 0) {
        const double peak = __dmul_rn(pk, __ddiv_rn((double)p.W, (double)p.pw));
        const int work = by_rule ? (int)v : nb_width_for(p.W, tp, max_width, peak);
        nb_set_work(p, work);
        if (p.ntrace < kNetTrace) p.trace[p.ntrace++] = work;
        return;
    }
    const int nw = by_rule ? (int)v : nb_width_for(p.W, tp, max_width, pk);
    if ((double)abs(nw - p.work) <= __dmul_rn(0.08, (double)p.work)) {
        p.active = 0;                                    // this pass's disparity is final
        return;
    }
    nb_set_work(p, nw);
    if (p.ntrace < kNetTrace) p.trace[p.ntrace++] = nw;
}

namespace {

constexpr int kStages = 2;       // CTA tables: 0 the probe, 1 the passes
constexpr int kExtra = 3;        // + work outputs, select, one CTA per pair

// Offsets of one pair's network scratch inside its slab.
struct SlabLayout {
    size_t lw, rw, gh, d0, d1, d2, full, sel, hist, fa0, fa1, fb0, fb1, v0, v1, rin, ra, rb;
    size_t bytes;
};

SlabLayout slab_layout(const NetView &n, int Wm, int Hm, int Wf, int Hf) {
    SlabLayout L{};
    Carver cv(nullptr);
    int h1, w1, h, w;
    net_quarter(Hm, Wm, h1, w1, h, w);
    const size_t HW = (size_t)Wm * Hm, Hh = (size_t)(Hm / 2 + 1) * (Wm / 2 + 1);
    auto at = [&](size_t bytes) {
        const size_t o = cv.off;
        cv.take<unsigned char>(bytes);
        return o;
    };
    L.lw = at(HW * 4);
    L.rw = at(HW * 4);
    L.gh = at(Hh * 4);
    L.d0 = at((size_t)h * w * 4);
    L.d1 = at(Hh * 4);
    L.d2 = at(HW * 4);
    L.full = at((size_t)Wf * Hf * 8);
    L.sel = at(select_state_bytes());
    L.hist = at(select_hist_words() * 4);
    L.fa0 = at((size_t)n.C * h1 * w1 * 4);
    L.fa1 = at((size_t)n.C * h1 * w1 * 4);
    L.fb0 = at((size_t)n.C * h * w * 4);
    L.fb1 = at((size_t)n.C * h * w * 4);
    L.v0 = at((size_t)n.Cm * n.D * h * w * 4);
    L.v1 = at((size_t)n.Cm * n.D * h * w * 4);
    L.rin = at(2 * HW * 4);
    L.ra = at((size_t)n.Rc * HW * 4);
    L.rb = at((size_t)n.Rc * HW * 4);
    L.bytes = cv.off;
    return L;
}

}  // namespace
}  // namespace sv

using namespace sv;

struct sv_netbatch {
    const sv_net *net;
    NetView view;
    int n, dtype, probe_width, max_width, passes, precision;
    double target_peak, tol;
    RefineCfg rc;
    sv_batch_config cfg;
    std::vector<NetPair> init;                 // host copy of the pairs' fixed fields
    std::vector<long long> pre[kStages * NK_COUNT + kExtra];
    SlabLayout lay;
    size_t slab;
    // workspace layout
    size_t off_pairs, off_lt, off_rt, off_pre, off_slabs, off_refine, total;
    BatchPlan plan;
    // bound state
    char *ws;
    bool bound;
    std::vector<sv_pair_desc> desc;
    std::mutex mu;
    cudaGraphExec_t graph;
    int graph_dev;
    unsigned long long graph_kernels;
};

namespace {

int nb_check(const sv_netbatch *nb) {
    if (!nb) { set_error("NULL batch"); return SV_ERR_NULL; }
    return SV_OK;
}

// Every launch of one run, in stream order (no host synchronisation).
int nb_enqueue(sv_netbatch *nb, cudaStream_t st, bool refine) {
    char *ws = nb->ws;
    const int n = nb->n;
    NetPair *pairs = reinterpret_cast<NetPair *>(ws + nb->off_pairs);
    const void *const *lt = reinterpret_cast<const void *const *>(ws + nb->off_lt);
    const void *const *rt = reinterpret_cast<const void *const *>(ws + nb->off_rt);
    auto pre = [&](int k) {
        return reinterpret_cast<const long long *>(ws + nb->off_pre) + (size_t)k * (n + 1);
    };
    char *s0 = ws + nb->off_slabs;
    const SlabLayout &Ly = nb->lay;
    NetSlab s{};
    s.lw = reinterpret_cast<float *>(s0 + Ly.lw);
    s.rw = reinterpret_cast<float *>(s0 + Ly.rw);
    s.gh = reinterpret_cast<float *>(s0 + Ly.gh);
    s.d0 = reinterpret_cast<float *>(s0 + Ly.d0);
    s.d1 = reinterpret_cast<float *>(s0 + Ly.d1);
    s.d2 = reinterpret_cast<float *>(s0 + Ly.d2);
    s.full = reinterpret_cast<double *>(s0 + Ly.full);
    s.sel = reinterpret_cast<SelState *>(s0 + Ly.sel);
    s.hist = reinterpret_cast<unsigned *>(s0 + Ly.hist);
    s.f.fa[0] = reinterpret_cast<float *>(s0 + Ly.fa0);
    s.f.fa[1] = reinterpret_cast<float *>(s0 + Ly.fa1);
    s.f.fb[0] = reinterpret_cast<float *>(s0 + Ly.fb0);
    s.f.fb[1] = reinterpret_cast<float *>(s0 + Ly.fb1);
    s.f.v0 = reinterpret_cast<float *>(s0 + Ly.v0);
    s.f.v1 = reinterpret_cast<float *>(s0 + Ly.v1);
    s.f.rin = reinterpret_cast<float *>(s0 + Ly.rin);
    s.f.ra = reinterpret_cast<float *>(s0 + Ly.ra);
    s.f.rb = reinterpret_cast<float *>(s0 + Ly.rb);
    s.f.flag = nullptr;
    const long long slab = (long long)nb->slab;
    NetStageLaunch g[kStages];
    for (int k = 0; k < kStages; ++k) {
        for (int j = 0; j < NK_COUNT; ++j) {
            g[k].pre[j] = pre(k * NK_COUNT + j);
            g[k].total[j] = nb->pre[k * NK_COUNT + j][n];
        }
        g[k].pairs = pairs;
        g[k].n = n;
        g[k].slab = slab;
    }
    const int xo = kStages * NK_COUNT;
    const NetLaunch Lwo{pre(xo), pairs, n, slab}, Lsel{pre(xo + 1), pairs, n, slab},
        Lone{pre(xo + 2), pairs, n, slab};
    const long long twow = nb->pre[xo][n], tsel = nb->pre[xo + 1][n];
    const int tb = 128, nbk = (n + tb - 1) / tb;
    const long long sel_off = (long long)Ly.sel;
    int rc;
    // probe (stereonet.py:3900-3907)
    count_launch();
    k_nb_probe_init<<<nbk, tb, 0, st>>>(pairs, n);
    SV_LAUNCH_CHECK();
    if ((rc = launch_b_resize(g[0], lt, rt, nb->dtype, s, false, st))) return rc;
    if ((rc = launch_b_forward(nb->view, g[0], s, st))) return rc;
    // the width decisions from histograms of the rule's widths when every
    // pair's rule has at most kWidthBins + 1 widths (as the single-pair path)
    int kmax_all = 48;
    for (const NetPair &q : nb->init) {
        const int k = width_rule_kmax(WidthRule{q.W, nb->max_width, nb->target_peak, 1.0});
        kmax_all = k > kmax_all ? k : kmax_all;
    }
    const int by_rule = kmax_all - 48 <= kWidthBins;
    if (by_rule) rc = launch_b_width_probe(Lone, s, nb->target_peak, nb->max_width, st);
    else rc = launch_b_sel_probe(Lone, s, st);
    if (rc) return rc;
    count_launch();
    k_nb_decide<<<nbk, tb, 0, st>>>(pairs, n, s0, slab, sel_off, nb->target_peak, nb->max_width,
                                    0, by_rule);
    SV_LAUNCH_CHECK();
    // passes (stereonet.py:3918-3929)
    for (int pass = 1; pass <= nb->passes; ++pass) {
        const bool with_sel = pass < nb->passes;
        if ((rc = launch_b_resize(g[1], lt, rt, nb->dtype, s, with_sel, st))) return rc;
        if ((rc = launch_b_forward(nb->view, g[1], s, st))) return rc;
        if ((rc = launch_b_work_outputs(Lwo, twow, s, with_sel, nb->target_peak,
                                        by_rule ? nb->max_width : 0, st)))
            return rc;
        if (!with_sel) break;
        if (!by_rule && (rc = launch_b_sel_rest(Lsel, tsel, s, st))) return rc;
        count_launch();
        k_nb_decide<<<nbk, tb, 0, st>>>(pairs, n, s0, slab, sel_off, nb->target_peak,
                                        nb->max_width, pass, by_rule);
        SV_LAUNCH_CHECK();
    }
    if (!refine) return SV_OK;
    char *rws = ws + nb->off_refine;
    SV_CUDA_TRY(cudaMemsetAsync(rws, 0, sizeof(DevFlags) + 256, st));   // flag + queue
    const BatchTables t = batch_tables(nb->plan, n, rws, nb->rc, nb->dtype, nb->tol, nb->cfg);
    return launch_batch_refine(t, nb->plan.px_blocks, nb->plan.rows, nb->plan.tiles,
                               nb->plan.tasks, nb->rc.l16, nb->cfg.sgm_threads,
                               nb->cfg.sgm_ctas_per_sm, st);
}

void drop_graph(sv_netbatch *nb) {
    if (nb->graph) {
        cudaGraphExecDestroy(nb->graph);
        nb->graph = nullptr;
    }
}

}  // namespace

extern "C" {

int sv_netbatch_create(const sv_net *net, const int *W, const int *H, int n, int dtype,
                       double target_peak, int probe_width, int max_width, int passes,
                       int precision, double tol, const sv_refine_params *p, sv_netbatch **out) {
    if (!net || !W || !H || !p || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (n < 1) { set_error("no pairs"); return SV_ERR_PARAM; }
    if (precision != SV_FP32) {
        set_error("the batched network runs FP32 (precision %d)", precision);
        return SV_ERR_PARAM;
    }
    if (dtype != SV_U8 && dtype != SV_F32 && dtype != SV_F64) {
        set_error("unknown image dtype %d", dtype);
        return SV_ERR_PARAM;
    }
    if (probe_width < 1 || max_width < 1 || passes < 1 || !std::isfinite(target_peak) ||
        !std::isfinite(tol)) {
        set_error("bad arguments");
        return SV_ERR_PARAM;
    }
    RefineCfg c;
    int rc = check_refine(1, 1, p, true, &c);
    if (rc) return rc;
    if (slot_width(c.K) > 32) {
        set_error("batched refinement supports bands up to K = 30 (got K = %d)", c.K);
        return SV_ERR_SHAPE;
    }
    const NetView &v = net_view(net);
    sv_netbatch *nb = new sv_netbatch();
    nb->net = net;
    nb->view = v;
    nb->n = n;
    nb->dtype = dtype;
    nb->probe_width = probe_width;
    nb->max_width = max_width;
    nb->passes = passes;
    nb->precision = precision;
    nb->target_peak = target_peak;
    nb->tol = tol;
    nb->rc = c;
    sv_batch_config_default(&nb->cfg);
    nb->init.resize(n);
    for (auto &t : nb->pre) t.assign(n + 1, 0);
    int Wmax = 1, Hmax = 1, Wfm = 1, Hfm = 1;
    long long ctas[NK_COUNT];
    const int min_work = 48;
    for (int i = 0; i < n; ++i) {
        const int w = W[i], h = H[i];
        if (w < 2 || h < 2 || w > kMaxRowW) {
            set_error("pair %d: %dx%d outside 2..%d wide", i, w, h, kMaxRowW);
            delete nb;
            return SV_ERR_SHAPE;
        }
        NetPair &q = nb->init[i];
        memset(&q, 0, sizeof(q));
        q.W = w;
        q.H = h;
        q.pw = probe_width < w ? probe_width : w;
        const int ph = (int)(h * q.pw / (double)w + 0.5);
        q.ph = ph < 8 ? 8 : ph;
        // the largest work size a pass can choose (width_for's range)
        const int cap = max_width > min_work ? max_width : min_work;
        q.Wm = w <= cap ? w : cap;
        if (q.Wm >= w) {
            q.Hm = h;
        } else {
            const int hm = (int)(h * (q.Wm / (double)w) + 0.5);
            q.Hm = hm < 8 ? 8 : hm;
        }
        // every size the batch can run must pass the forward's shape check
        // (CostVolume.invalid_mask's IndexError, stereonet.py:837-839)
        const int chk_w[3] = {q.pw, w < min_work ? w : min_work, q.Wm};
        for (int k = 0; k < 3; ++k) {
            const int cw = chk_w[k];
            int h1, w1, hq, wq;
            net_quarter(8, cw, h1, w1, hq, wq);
            if (wq <= v.D - 2) {
                set_error("pair %d: a %d-wide pass has quarter width %d <= D-2 = %d (the "
                          "reference raises IndexError)", i, cw, wq, v.D - 2);
                delete nb;
                return SV_ERR_SHAPE;
            }
        }
        Wmax = std::max(Wmax, q.Wm);
        Hmax = std::max(Hmax, q.Hm);
        Wfm = std::max(Wfm, w);
        Hfm = std::max(Hfm, h);
        for (int k = 0; k < kStages; ++k) {
            if ((rc = net_stage_ctas(v, k ? q.Hm : q.ph, k ? q.Wm : q.pw, ctas))) {
                delete nb;
                return rc;
            }
            for (int j = 0; j < NK_COUNT; ++j)
                nb->pre[k * NK_COUNT + j][i + 1] = nb->pre[k * NK_COUNT + j][i] + ctas[j];
        }
        const int xo = kStages * NK_COUNT;
        nb->pre[xo][i + 1] = nb->pre[xo][i] + (long long)((w + 31) / 32) *
                                                  ((h + 8 * kWorkRowsBatched - 1) /
                                                   (8 * kWorkRowsBatched));
        nb->pre[xo + 1][i + 1] = nb->pre[xo + 1][i] + select_ctas((long)w * h);
        nb->pre[xo + 2][i + 1] = i + 1;
    }
    for (int k = 0; k < kStages * NK_COUNT + kExtra; ++k)
        if (nb->pre[k][n] >= (1ll << 31)) {
            set_error("batch too large: %lld CTAs in one launch", nb->pre[k][n]);
            delete nb;
            return SV_ERR_SHAPE;
        }
    nb->lay = slab_layout(v, Wmax, Hmax, Wfm, Hfm);
    nb->slab = align256(nb->lay.bytes);
    // workspace: pairs | left / right tables | CTA tables | slabs | refinement
    Carver cv(nullptr);
    nb->off_pairs = cv.off;
    cv.take<NetPair>(n);
    nb->off_lt = cv.off;
    cv.take<const void *>(n);
    nb->off_rt = cv.off;
    cv.take<const void *>(n);
    nb->off_pre = cv.off;
    cv.take<long long>((size_t)(kStages * NK_COUNT + kExtra) * (n + 1));
    nb->off_slabs = cv.off;
    cv.take<unsigned char>(nb->slab * (size_t)n);
    nb->off_refine = cv.off;
    std::vector<sv_pair_desc> d(n);
    for (int i = 0; i < n; ++i) {
        d[i] = sv_pair_desc{};
        d[i].W = W[i];
        d[i].H = H[i];
    }
    if ((rc = plan_batch(d.data(), n, c, nb->cfg.px_per_block, nullptr, &nb->plan))) {
        delete nb;
        return rc;
    }
    nb->total = nb->off_refine + nb->plan.total;
    *out = nb;
    return SV_OK;
}

size_t sv_netbatch_workspace_size(const sv_netbatch *nb) { return nb ? nb->total : 0; }

int sv_netbatch_bind(sv_netbatch *nb, const sv_pair_desc *pairs, void *workspace,
                     size_t workspace_bytes, void *stream) {
    int rc = nb_check(nb);
    if (rc) return rc;
    if (!pairs) { set_error("NULL pairs"); return SV_ERR_NULL; }
    if ((rc = check_ws(workspace, workspace_bytes, nb->total))) return rc;
    const int n = nb->n;
    char *ws = static_cast<char *>(workspace);
    std::vector<sv_pair_desc> d(pairs, pairs + n);
    std::vector<const void *> lt(n), rt(n);
    for (int i = 0; i < n; ++i) {
        if (d[i].W != nb->init[i].W || d[i].H != nb->init[i].H) {
            set_error("pair %d: %dx%d, the batch was planned for %dx%d", i, d[i].W, d[i].H,
                      nb->init[i].W, nb->init[i].H);
            return SV_ERR_SHAPE;
        }
        if (!d[i].left || !d[i].right || !d[i].out || !d[i].status) {
            set_error("pair %d: NULL pointer", i);
            return SV_ERR_NULL;
        }
        lt[i] = d[i].left;
        rt[i] = d[i].right;
        // the refinement reads the network disparity from the pair's slab
        d[i].disp0 = reinterpret_cast<const double *>(ws + nb->off_slabs + nb->slab * (size_t)i +
                                                      nb->lay.full);
    }
    std::lock_guard<std::mutex> lock(nb->mu);
    if ((rc = plan_batch(d.data(), n, nb->rc, nb->cfg.px_per_block, ws + nb->off_refine,
                         &nb->plan)))
        return rc;
    cudaStream_t st = (cudaStream_t)stream;
    SV_CUDA_TRY(cudaMemcpyAsync(ws + nb->off_pairs, nb->init.data(), sizeof(NetPair) * n,
                                cudaMemcpyHostToDevice, st));
    SV_CUDA_TRY(cudaMemcpyAsync(ws + nb->off_lt, lt.data(), sizeof(void *) * n,
                                cudaMemcpyHostToDevice, st));
    SV_CUDA_TRY(cudaMemcpyAsync(ws + nb->off_rt, rt.data(), sizeof(void *) * n,
                                cudaMemcpyHostToDevice, st));
    long long *pre = nullptr;
    std::vector<long long> flat;
    for (const auto &t : nb->pre) flat.insert(flat.end(), t.begin(), t.end());
    pre = flat.data();
    SV_CUDA_TRY(cudaMemcpyAsync(ws + nb->off_pre, pre, sizeof(long long) * flat.size(),
                                cudaMemcpyHostToDevice, st));
    if ((rc = upload_batch(nb->plan, n, ws + nb->off_refine, st))) return rc;
    SV_CUDA_TRY(cudaStreamSynchronize(st));        // the host tables above are temporaries
    nb->ws = ws;
    nb->desc = d;
    nb->bound = true;
    drop_graph(nb);
    return SV_OK;
}

// Enqueue the batch: the first run on a capturable stream records it into a
// CUDA graph, later runs replay the graph (one launch on the host).
static int nb_run(sv_netbatch *nb, void *stream, bool refine) {
    int rc = nb_check(nb);
    if (rc) return rc;
    if (!nb->bound) { set_error("sv_netbatch_bind first"); return SV_ERR_PARAM; }
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lock(nb->mu);
    if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread)
        return nb_enqueue(nb, st, refine);
    cudaStreamCaptureStatus cs;
    SV_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return nb_enqueue(nb, st, refine);
    int dev = 0;
    SV_CUDA_TRY(cudaGetDevice(&dev));
    const int key = refine ? 1 : 0;
    if (nb->graph && nb->graph_dev == dev * 2 + key) {
        SV_CUDA_TRY(cudaGraphLaunch(nb->graph, st));
        count_launches(nb->graph_kernels);
        return SV_OK;
    }
    drop_graph(nb);
    const unsigned long long before = launch_count_now();
    SV_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    rc = nb_enqueue(nb, st, refine);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    const unsigned long long kernels = launch_count_now() - before;
    uncount_launches(kernels);
    cudaGraphExec_t exec = nullptr;
    cudaError_t ei = cudaSuccess;
    if (!rc && e == cudaSuccess) ei = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (rc) return rc;
    if (e != cudaSuccess || ei != cudaSuccess) {
        set_error("%s failed: %s", e != cudaSuccess ? "stream capture" : "graph instantiation",
                  cudaGetErrorString(e != cudaSuccess ? e : ei));
        return SV_ERR_CUDA;
    }
    nb->graph = exec;
    nb->graph_dev = dev * 2 + key;
    nb->graph_kernels = kernels;
    SV_CUDA_TRY(cudaGraphLaunch(exec, st));
    count_launches(kernels);
    return SV_OK;
}

int sv_netbatch_run(sv_netbatch *nb, void *stream) { return nb_run(nb, stream, true); }

int sv_netbatch_predict(sv_netbatch *nb, void *stream) { return nb_run(nb, stream, false); }

int sv_netbatch_disparity(const sv_netbatch *nb, int i, const double **disp_full) {
    int rc = nb_check(nb);
    if (rc) return rc;
    if (!disp_full) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (!nb->bound || i < 0 || i >= nb->n) { set_error("pair %d not bound", i); return SV_ERR_PARAM; }
    *disp_full = reinterpret_cast<const double *>(nb->ws + nb->off_slabs + nb->slab * (size_t)i +
                                                  nb->lay.full);
    return SV_OK;
}

int sv_netbatch_trace(const sv_netbatch *nb, int *work_trace, int trace_len, int *work_size,
                      void *stream) {
    int rc = nb_check(nb);
    if (rc) return rc;
    if (!nb->bound) { set_error("sv_netbatch_bind first"); return SV_ERR_PARAM; }
    if (trace_len < 1) { set_error("trace_len < 1"); return SV_ERR_PARAM; }
    const int n = nb->n;
    std::vector<NetPair> h(n);
    cudaStream_t st = (cudaStream_t)stream;
    SV_CUDA_TRY(cudaMemcpyAsync(h.data(), nb->ws + nb->off_pairs, sizeof(NetPair) * n,
                                cudaMemcpyDeviceToHost, st));
    SV_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
        if (work_trace) {
            int *t = work_trace + (size_t)i * trace_len;
            int k = 0;
            for (; k < h[i].ntrace && k < trace_len - 1; ++k) t[k] = h[i].trace[k];
            for (; k < trace_len; ++k) t[k] = 0;
        }
        if (work_size) {
            work_size[2 * i] = h[i].Ww;
            work_size[2 * i + 1] = h[i].Hw;
        }
    }
    return SV_OK;
}

int sv_netbatch_data_status(const sv_netbatch *nb, void *stream) {
    int rc = nb_check(nb);
    if (rc) return rc;
    if (!nb->bound) { set_error("sv_netbatch_bind first"); return SV_ERR_PARAM; }
    return sv_workspace_status(nb->ws + nb->off_refine, stream);
}

void sv_netbatch_destroy(sv_netbatch *nb) {
    if (!nb) return;
    if (nb->graph) {
        cudaDeviceSynchronize();
        cudaGraphExecDestroy(nb->graph);
    }
    delete nb;
}

}  // extern "C"
