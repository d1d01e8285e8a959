// sv_net_api.cu -- extern "C" network entry points of include/sv_b200.h:
// checkpoint upload, StereoNet.forward, resize, predict_at_scale and the
// host-side control flow of predict_auto (stereonet.py:3872-3960).

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "sv_common.cuh"
#include "sv_network.cuh"
#include "sv_select.cuh"
#include "sv_tc.cuh"

// One captured predict_auto stage (a network pass, optionally with the peak
// selection that follows it), keyed by everything its kernels' arguments
// depend on.
struct sv_graph_key {
    int kind, W, H, dtype, work, with_sel, precision;
    const void *left, *right;
    void *disp_full, *disp_work, *ws;
    bool operator==(const sv_graph_key &o) const {
        return kind == o.kind && W == o.W && H == o.H && dtype == o.dtype && work == o.work &&
               with_sel == o.with_sel && precision == o.precision && left == o.left && right == o.right &&
               disp_full == o.disp_full && disp_work == o.disp_work && ws == o.ws;
    }
};

struct sv_graph_entry {
    sv_graph_key key;
    cudaGraphExec_t exec;
    unsigned long long kernels;
    int device;
    double *slot;             // mapped pinned slot the stage's peak lands in, or NULL
};

struct sv_net {
    sv::NetView view;
    float *dev = nullptr;     // all FP32 parameters, one allocation
    uint16_t *tc = nullptr;   // BF16 tensor-core operands of the six convolutions
    int arch[16];
    int n_arch;
    std::mutex graph_mu;      // guards graphs (the weights themselves are immutable)
    std::vector<sv_graph_entry> graphs;
};

namespace sv {

int lr_refine_census(const void *left, const void *right, int dtype, int W, int H,
                     const sv_refine_params *p, void *workspace, size_t workspace_bytes,
                     cudaStream_t st);
int lr_refine_after_census(const void *left, const void *right, int dtype, const double *disp0,
                           int W, int H, double tol, const sv_refine_params *p, double *out,
                           uint8_t *status, void *workspace, size_t workspace_bytes,
                           cudaStream_t st);

// A second stream of the calling thread on the current device (with a fork
// and a join event), for work that overlaps the caller's stream.
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

static int side_stream(SideStream **out) {
    constexpr int kDevs = 16;
    static thread_local SideStream per[kDevs];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) return SV_ERR_CUDA;
    SideStream &x = per[dev];
    if (!x.s) {
        SideStream y;
        if (cudaStreamCreateWithFlags(&y.s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&y.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&y.join, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            if (y.join) cudaEventDestroy(y.join);
            if (y.fork) cudaEventDestroy(y.fork);
            if (y.s) cudaStreamDestroy(y.s);
            return SV_ERR_CUDA;
        }
        x = y;
    }
    *out = &x;
    return SV_OK;
}

static long param_count(const int *a) {
    long C = a[0], Cm = a[1], Rc = a[3], nd = a[4];
    long n = C * 9 + C + 3 * (C * C * 9 + C);
    n += Cm * C * 27 + Cm + Cm * Cm * 27 + Cm + Cm * 27 + 1;
    long lv = 0, prev = 2;
    for (int i = 0; i < nd; ++i) { lv += Rc * prev * 9 + Rc; prev = Rc; }
    lv += prev * 9 + 1;
    return n + 2 * lv;
}

static void bind_view(sv_net *net) {
    NetView &v = net->view;
    const int *a = net->arch;
    v.C = a[0]; v.Cm = a[1]; v.D = a[2]; v.Rc = a[3]; v.ndil = a[4];
    for (int i = 0; i < v.ndil; ++i) v.dil[i] = a[5 + i];
    const float *p = net->dev;
    const int C = v.C, Cm = v.Cm, Rc = v.Rc;
    const int fic[4] = {1, C, C, C};
    for (int i = 0; i < 4; ++i) {
        v.fw[i] = p; p += C * fic[i] * 9;
        v.fb[i] = p; p += C;
    }
    const int cic[3] = {C, Cm, Cm}, coc[3] = {Cm, Cm, 1};
    for (int i = 0; i < 3; ++i) {
        v.cw[i] = p; p += coc[i] * cic[i] * 27;
        v.cb[i] = p; p += coc[i];
    }
    for (int lv = 0; lv < 2; ++lv) {
        int prev = 2;
        for (int i = 0; i < v.ndil; ++i) {
            v.rw[lv][i] = p; p += Rc * prev * 9;
            v.rb[lv][i] = p; p += Rc;
            prev = Rc;
        }
        v.rw[lv][v.ndil] = p; p += prev * 9;
        v.rb[lv][v.ndil] = p; p += 1;
    }
}

static void conv_out(int H, int W, int *h1, int *w1, int *h, int *w) {
    *h1 = (H - 1) / 2 + 1;
    *w1 = (W - 1) / 2 + 1;
    *h = (*h1 - 1) / 2 + 1;
    *w = (*w1 - 1) / 2 + 1;
}

// Forward scratch for an (H, W) input (sizes are monotone in H and W).
static size_t carve_fwd(Carver &cv, const NetView &n, int H, int W, DevFlags *flag, FwdBufs *b) {
    int h1, w1, h, w;
    conv_out(H, W, &h1, &w1, &h, &w);
    const size_t f1 = (size_t)n.C * h1 * w1, f2 = (size_t)n.C * h * w;
    const size_t vol = (size_t)n.Cm * n.D * h * w, HW = (size_t)H * W;
    size_t start = cv.off;
    FwdBufs t{};
    t.fa[0] = cv.take<float>(f1);
    t.fa[1] = cv.take<float>(f1);
    t.fb[0] = cv.take<float>(f2);
    t.fb[1] = cv.take<float>(f2);
    t.v0 = cv.take<float>(vol);
    t.v1 = cv.take<float>(vol);
    t.rin = cv.take<float>(2 * HW);
    t.ra = cv.take<float>((size_t)n.Rc * HW);
    t.rb = cv.take<float>((size_t)n.Rc * HW);
    t.flag = flag ? &flag->status : nullptr;
    if (b) *b = t;
    return cv.off - start;
}

static int check_net_shape(const NetView &n, int H, int W) {
    if (H < 2 || W < 2) {
        set_error("network input %dx%d too small", W, H);
        return SV_ERR_SHAPE;
    }
    int h1, w1, h, w;
    conv_out(H, W, &h1, &w1, &h, &w);
    // CostVolume.invalid_mask (stereonet.py:837-839) indexes past its list,
    // and the reference raises IndexError, when the quarter width <= D-2.
    if (w <= n.D - 2) {
        set_error("quarter-resolution width %d <= D-2 = %d (the reference raises IndexError)",
                  w, n.D - 2);
        return SV_ERR_SHAPE;
    }
    return SV_OK;
}

static int width_for(int W, double target_peak, int max_width, double pk) {
    double m = pk > 1.0e-6 ? pk : 1.0e-6;
    const double q = W * target_peak / m + 0.5;
    int w = q < 2147483647.0 ? (q > -2147483648.0 ? (int)q : -2147483647 - 1) : 2147483647;
    if (w > W) w = W;
    if (w > max_width) w = max_width;
    if (w < 48) w = 48;
    return w;
}

// Workspace of predict_auto / predict_at_scale for a W x H pair.
struct PredictWs {
    float *lw, *rw, *gh, *d0, *d1, *d2;
    double *probe64;
    SelState *sel;
    unsigned *hist;
    FwdBufs fwd;
};

static void predict_dims(int W, int H, int max_width, int probe_width, int *Wm, int *Hm) {
    const int cap = max_width > 48 ? max_width : 48;   // width_for's range
    int ww = W <= cap ? W : cap;
    int pw = probe_width < W ? probe_width : W;
    int ph = (int)(H * pw / (double)W + 0.5);
    if (ph < 8) ph = 8;
    *Wm = ww > pw ? ww : pw;
    int hm = H > 8 ? H : 8;
    *Hm = hm > ph ? hm : ph;
}

static size_t carve_predict(void *ws, const NetView &n, int Wm, int Hm, PredictWs *o) {
    Carver cv(ws);
    PredictWs p{};
    DevFlags *flag = cv.take<DevFlags>(1);
    const size_t HW = (size_t)Wm * Hm;
    int h1, w1, h, w;
    conv_out(Hm, Wm, &h1, &w1, &h, &w);
    p.lw = cv.take<float>(HW);
    p.rw = cv.take<float>(HW);
    p.gh = cv.take<float>(HW / 4 + 1);
    p.d0 = cv.take<float>((size_t)h * w);
    p.d1 = cv.take<float>(HW / 4 + 1);
    p.d2 = cv.take<float>(HW);
    p.probe64 = cv.take<double>(HW);
    p.sel = reinterpret_cast<SelState *>(cv.take<unsigned char>(select_state_bytes()));
    p.hist = cv.take<unsigned>(select_hist_words());
    carve_fwd(cv, n, Hm, Wm, flag, &p.fwd);
    p.fwd.qspread = cv.take<float>((size_t)h * w);   // the last pass's confidence maps
    p.fwd.qpmax = cv.take<float>((size_t)h * w);
    if (o) *o = p;
    return cv.off;
}

// predict (stereonet.py:5891-5897) on FP32 images already in lw/rw.
// gh_ready: the resize already wrote the half-resolution guide
// decide (optional): the width decision the network's output convolution
// runs over the map it writes (its state cleared by the stage's resize).
static int predict_f32(const sv_net *net, const PredictWs &w, int W, int H, int precision,
                       cudaStream_t st, bool gh_ready = false,
                       const SelFuse *decide = nullptr) {
    int rc = check_net_shape(net->view, H, W);
    if (rc) return rc;
    if (!gh_ready) {
        rc = launch_avgpool2(w.lw, H, W, w.gh, st);
        if (rc) return rc;
    }
    FwdBufs fb = w.fwd;
    fb.decide = decide;
    return launch_forward(net->view, w.lw, w.rw, H, W, w.gh, w.lw, w.d0, w.d1, w.d2, fb,
                          precision, st);
}

static int predict_at_scale_impl(const sv_net *net, const PredictWs &w, const void *left,
                                 const void *right, int dtype, int W, int H, int work,
                                 int precision, double *disp_full, double *disp_work, int *pWw,
                                 int *pHw, cudaStream_t st, const SelFuse *fuse = nullptr) {
    int rc;
    if (work >= W) {
        if (fuse) {
            set_error("a select fused into a native-resolution pass");
            return SV_ERR_PARAM;
        }
        rc = launch_to_f32_pair(left, right, dtype, (long)W * H, w.lw, w.rw, st);
        if (!rc) rc = predict_f32(net, w, W, H, precision, st);
        if (!rc) rc = launch_promote(w.d2, (long)W * H, disp_full, st);
        if (rc) return rc;
        SV_CUDA_TRY(cudaMemcpyAsync(disp_work, disp_full, sizeof(double) * W * H,
                                    cudaMemcpyDeviceToDevice, st));
        *pWw = W;
        *pHw = H;
        return SV_OK;
    }
    const double scale = work / (double)W;
    const int Ww = work;
    int Hw = (int)(H * scale + 0.5);
    if (Hw < 8) Hw = 8;
    rc = check_net_shape(net->view, Hw, Ww);
    if (!rc)
        rc = launch_resize_pair(left, right, dtype, W, H, Ww, Hw, w.lw, w.rw, st, w.gh, fuse);
    if (!rc) rc = predict_f32(net, w, Ww, Hw, precision, st, true);
    if (!rc)
        rc = launch_work_outputs(w.d2, Ww, Hw, W, H, 1.0 / scale, disp_work, disp_full, st,
                                 fuse);
    *pWw = Ww;
    *pHw = Hw;
    return rc;
}

#define SV_TRY(expr)                  \
    do {                              \
        int rc_ = (expr);             \
        if (rc_ != SV_OK) return rc_; \
    } while (0)

static void work_dims(int W, int H, int work, int *Ww, int *Hw) {
    if (work >= W) {
        *Ww = W;
        *Hw = H;
        return;
    }
    const double scale = work / (double)W;
    int hw = (int)(H * scale + 0.5);
    *Ww = work;
    *Hw = hw < 8 ? 8 : hw;
}

// Read back the selected peak (the one host synchronisation of a stage),
// through a pinned 8-byte slot per host thread (a copy into pageable memory
// is staged by the driver and returns later); the stack is the fallback if
// the slot cannot be had.
static int wait_slot(double *slot, cudaStream_t st, double *out);

// The peak of the stage just queued on st (floored like _peak): from its
// mapped slot when it published one, else copied out of the workspace.
static int fetch_peak(const PredictWs &w, cudaStream_t st, double *slot, double *peak,
                      bool floor = true) {
    double v = 0.0;
    if (slot) {
        SV_TRY(wait_slot(slot, st, &v));
    } else {
        struct Slot {
            double *p = nullptr;
            ~Slot() {
                if (p) cudaFreeHost(p);
            }
        };
        static thread_local Slot pinned;
        if (!pinned.p &&
            cudaMallocHost(reinterpret_cast<void **>(&pinned.p), sizeof(double)) != cudaSuccess) {
            pinned.p = nullptr;
            cudaGetLastError();
        }
        double local = 0.0;
        double *dst = pinned.p ? pinned.p : &local;
        SV_CUDA_TRY(cudaMemcpyAsync(dst,
                                    reinterpret_cast<const char *>(w.sel) + select_value_offset(),
                                    sizeof(double), cudaMemcpyDeviceToHost, st));
        SV_CUDA_TRY(cudaStreamSynchronize(st));
        v = *dst;
    }
    *peak = !floor || v > 0.5 ? v : 0.5;            // _peak's floor
    return SV_OK;
}

// A stage that ends with a peak selection publishes the value into a small
// mapped pinned host slot owned by its graph: the host polls the slot
// instead of queueing a device-to-host copy and synchronising the stream.
// Before each launch the slot holds kSlotEmpty, a NaN no selection returns.
constexpr uint64_t kSlotEmpty = 0x7ff4a5a5a5a5a5a5ull;

static void arm_slot(double *slot) {
    *reinterpret_cast<volatile uint64_t *>(slot) = kSlotEmpty;
}

// Wait for the stage launched on st to fill slot.  Bounded: a stream that
// drains (or fails) without filling it, or a minute without a value, is an
// error.
static int wait_slot(double *slot, cudaStream_t st, double *out) {
    const volatile uint64_t *p = reinterpret_cast<const volatile uint64_t *>(slot);
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned long i = 1;; ++i) {
        uint64_t b = *p;
        if (b != kSlotEmpty) {
            memcpy(out, &b, sizeof(b));
            return SV_OK;
        }
        if ((i & 1023) == 0) {
            const cudaError_t q = cudaStreamQuery(st);
            if (q == cudaSuccess) {             // the stage is done: its store is visible
                b = *p;
                if (b != kSlotEmpty) {
                    memcpy(out, &b, sizeof(b));
                    return SV_OK;
                }
                set_error("peak slot not written by the finished stage");
                return SV_ERR_TIMEOUT;
            }
            if (q != cudaErrorNotReady) {
                set_error("stage failed: %s", cudaGetErrorString(q));
                return SV_ERR_CUDA;
            }
            if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(60)) {
                set_error("peak selection did not finish within 60 s");
                return SV_ERR_TIMEOUT;
            }
        }
    }
}

// Run one predict_auto stage.  On a capturable stream the stage is recorded
// into a CUDA graph the first time (per shape, buffers and device) and
// replayed afterwards, so a network pass costs one launch on the host.  On
// the legacy default stream, or inside the caller's own capture, the
// kernels are enqueued directly.  enqueue(mirror) queues the stage; with
// publish, a graphed stage gets a mapped slot as mirror and *slot points at
// its host side (NULL otherwise: read the peak from the workspace).
constexpr size_t kMaxGraphs = 48;

template <typename F>
static int run_stage(sv_net *net, const sv_graph_key &key, cudaStream_t st, bool publish,
                     double **slot, F &&enqueue) {
    *slot = nullptr;
    if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread)
        return enqueue(nullptr);
    cudaStreamCaptureStatus cs;
    SV_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return enqueue(nullptr);
    int dev = 0;
    SV_CUDA_TRY(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lock(net->graph_mu);
        for (auto &g : net->graphs) {
            if (g.device == dev && g.key == key) {
                if (publish && g.slot) arm_slot(g.slot);
                SV_CUDA_TRY(cudaGraphLaunch(g.exec, st));
                count_launches(g.kernels);
                if (publish) *slot = g.slot;
                return SV_OK;
            }
        }
    }
    double *host = nullptr, *mirror = nullptr;
    if (publish) {
        void *h = nullptr, *d = nullptr;
        SV_CUDA_TRY(cudaHostAlloc(&h, 64, cudaHostAllocMapped | cudaHostAllocPortable));
        const cudaError_t e = cudaHostGetDevicePointer(&d, h, 0);
        if (e != cudaSuccess) {
            cudaFreeHost(h);
            set_error("mapped slot: %s", cudaGetErrorString(e));
            return SV_ERR_CUDA;
        }
        host = static_cast<double *>(h);
        mirror = static_cast<double *>(d);
    }
    const unsigned long long before = launch_count_now();
    {
        const cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            if (host) cudaFreeHost(host);
            set_error("stream capture failed: %s", cudaGetErrorString(e));
            return SV_ERR_CUDA;
        }
    }
    const int rc = enqueue(mirror);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    const unsigned long long kernels = launch_count_now() - before;
    uncount_launches(kernels);                       // they run at the launch below
    cudaGraphExec_t exec = nullptr;
    cudaError_t ei = cudaSuccess;
    if (!rc && e == cudaSuccess) ei = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (rc || e != cudaSuccess || ei != cudaSuccess) {
        if (host) cudaFreeHost(host);
        if (rc) return rc;
        set_error("%s failed: %s", e != cudaSuccess ? "stream capture" : "graph instantiation",
                  cudaGetErrorString(e != cudaSuccess ? e : ei));
        return SV_ERR_CUDA;
    }
    if (host) arm_slot(host);
    {
        const cudaError_t el = cudaGraphLaunch(exec, st);
        if (el != cudaSuccess) {
            cudaGraphExecDestroy(exec);
            if (host) cudaFreeHost(host);
            set_error("graph launch failed: %s", cudaGetErrorString(el));
            return SV_ERR_CUDA;
        }
    }
    count_launches(kernels);
    *slot = host;
    std::lock_guard<std::mutex> lock(net->graph_mu);
    if (net->graphs.size() >= kMaxGraphs) {
        sv_graph_entry &old = net->graphs.front();
        cudaGraphExecDestroy(old.exec);
        if (old.slot) {
            cudaDeviceSynchronize();                 // its last launch may still write the slot
            cudaFreeHost(old.slot);
        }
        net->graphs.erase(net->graphs.begin());
    }
    net->graphs.push_back({key, exec, kernels, dev, host});
    return SV_OK;
}

// Pack FeatureNet c1..c4 and CostFilter c1, c2 as BF16 tensor-core
// operands (their FP64 parameters sit at the FP32 copy's offsets).
static int pack_tc(sv_net *net, const double *params) {
    NetView &v = net->view;
    const float *w[6] = {v.fw[0], v.fw[1], v.fw[2], v.fw[3], v.cw[0], v.cw[1]};
    const int K[6] = {9, v.C * 9, v.C * 9, v.C * 9, v.C * 27, v.Cm * 27};
    const int OC[6] = {v.C, v.C, v.C, v.C, v.Cm, v.Cm};
    size_t total = 0, off[6];
    for (int l = 0; l < 6; ++l) {
        off[l] = total;
        total += tc_weight_elems(K[l]);
    }
    for (int l = 0; l < 6; ++l) v.tw[l] = nullptr;
    if (v.C > 16 || v.Cm > 16) return SV_OK;         // outside the kernel: FP32 only
    std::vector<uint16_t> h(total, 0);
    for (int l = 0; l < 6; ++l)
        tc_pack_weights(params + (w[l] - net->dev), OC[l], K[l], h.data() + off[l]);
    cudaError_t e = cudaMalloc(&net->tc, total * sizeof(uint16_t));
    if (e == cudaSuccess)
        e = cudaMemcpy(net->tc, h.data(), total * sizeof(uint16_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        set_error("BF16 weight upload failed: %s", cudaGetErrorString(e));
        return SV_ERR_CUDA;
    }
    for (int l = 0; l < 6; ++l) v.tw[l] = net->tc + off[l];
    return SV_OK;
}

const NetView &net_view(const sv_net *net) { return net->view; }

}  // namespace sv

using namespace sv;

extern "C" {

int sv_net_create(const int *arch, int n_arch, const double *params, long n_params,
                  sv_net **out) {
    if (!arch || !params || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (n_arch < 6 || n_arch > 13 || arch[4] < 1 || arch[4] > 8 || n_arch != 5 + arch[4]) {
        set_error("arch vector must be {feat_C, cost_C, D, refine_C, ndil, dil...}");
        return SV_ERR_NET;
    }
    long need = param_count(arch);
    if (need != n_params) {
        set_error("checkpoint has %ld parameters, the architecture needs %ld", n_params, need);
        return SV_ERR_NET;
    }
    sv_net *net = new sv_net();
    memcpy(net->arch, arch, sizeof(int) * n_arch);
    net->n_arch = n_arch;
    std::vector<float> f(n_params);
    for (long i = 0; i < n_params; ++i) f[i] = (float)params[i];
    cudaError_t e = cudaMalloc(&net->dev, sizeof(float) * n_params);
    if (e == cudaSuccess)
        e = cudaMemcpy(net->dev, f.data(), sizeof(float) * n_params, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        set_error("weight upload failed: %s", cudaGetErrorString(e));
        if (net->dev) cudaFree(net->dev);
        delete net;
        return SV_ERR_CUDA;
    }
    bind_view(net);
    if (pack_tc(net, params) != SV_OK) {
        sv_net_destroy(net);
        return SV_ERR_CUDA;
    }
    *out = net;
    return SV_OK;
}

void sv_net_destroy(sv_net *net) {
    if (!net) return;
    // a replayed pass may still be writing its slot
    if (!net->graphs.empty()) cudaDeviceSynchronize();
    for (auto &g : net->graphs) {
        cudaGraphExecDestroy(g.exec);
        if (g.slot) cudaFreeHost(g.slot);
    }
    if (net->dev) cudaFree(net->dev);
    if (net->tc) cudaFree(net->tc);
    delete net;
}

int sv_resize(const double *img, int W, int H, int W2, int H2, double *out, void *stream) {
    if (!img || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1 || W2 < 1 || H2 < 1) { set_error("bad shape"); return SV_ERR_SHAPE; }
    return launch_resize_f64(img, W, H, W2, H2, out, (cudaStream_t)stream);
}

int sv_avgpool2(const double *img, int C, int H, int W, double *out, void *stream) {
    if (!img || !out) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (C < 1 || H < 1 || W < 1) { set_error("bad shape"); return SV_ERR_SHAPE; }
    return launch_avgpool2_f64(img, C, H, W, out, (cudaStream_t)stream);
}

size_t sv_forward_workspace_size(const sv_net *net, int H, int W) {
    if (!net || H < 1 || W < 1) return 0;
    Carver cv(nullptr);
    cv.take<DevFlags>(1);
    carve_fwd(cv, net->view, H, W, nullptr, nullptr);
    return cv.off;
}

int sv_stereonet_forward(const sv_net *net, const float *left, const float *right, int H,
                         int W, const float *guide_half, const float *guide_full, float *d0,
                         float *d1, float *d2, int precision, void *workspace,
                         size_t workspace_bytes, void *stream) {
    if (!net || !left || !right || !guide_half || !guide_full || !d0 || !d1 || !d2) {
        set_error("NULL argument");
        return SV_ERR_NULL;
    }
    if (precision != SV_FP32 && precision != SV_BF16) {
        set_error("precision %d is neither SV_FP32 nor SV_BF16", precision);
        return SV_ERR_PARAM;
    }
    SV_TRY(check_net_shape(net->view, H, W));
    size_t need = sv_forward_workspace_size(net, H, W);
    if (!workspace || ((uintptr_t)workspace & 255) || workspace_bytes < need) {
        set_error("workspace needs %zu bytes, 256-aligned", need);
        return SV_ERR_WORKSPACE;
    }
    Carver cv(workspace);
    DevFlags *flag = cv.take<DevFlags>(1);
    FwdBufs b;
    carve_fwd(cv, net->view, H, W, flag, &b);
    return launch_forward(net->view, left, right, H, W, guide_half, guide_full, d0, d1, d2, b,
                          precision, (cudaStream_t)stream);
}

size_t sv_predict_workspace_size(const sv_net *net, int W, int H, int max_width) {
    if (!net || W < 1 || H < 1) return 0;
    int Wm, Hm;
    predict_dims(W, H, max_width, 64, &Wm, &Hm);
    return carve_predict(nullptr, net->view, Wm, Hm, nullptr);
}

static int predict_ws(const sv_net *net, int W, int H, int max_width, int probe_width,
                      void *ws, size_t bytes, PredictWs *w) {
    int Wm, Hm;
    predict_dims(W, H, max_width, probe_width, &Wm, &Hm);
    size_t need = carve_predict(nullptr, net->view, Wm, Hm, nullptr);
    if (!ws || ((uintptr_t)ws & 255) || bytes < need) {
        set_error("workspace needs %zu bytes, 256-aligned (have %zu)", need, bytes);
        return SV_ERR_WORKSPACE;
    }
    carve_predict(ws, net->view, Wm, Hm, w);
    return SV_OK;
}

int sv_predict_at_scale(const sv_net *net, const void *left, const void *right, int dtype,
                        int W, int H, int work_width, int precision, double *disp_full,
                        double *disp_work, int *Ww, int *Hw, void *workspace,
                        size_t workspace_bytes, void *stream) {
    if (!net || !left || !right || !disp_full || !disp_work || !Ww || !Hw) {
        set_error("NULL argument");
        return SV_ERR_NULL;
    }
    if (precision != SV_FP32 && precision != SV_BF16) {
        set_error("precision %d is neither SV_FP32 nor SV_BF16", precision);
        return SV_ERR_PARAM;
    }
    if (W < 1 || H < 1 || work_width < 1) { set_error("bad shape"); return SV_ERR_SHAPE; }
    PredictWs w;
    int mw = work_width > 48 ? work_width : 48;
    SV_TRY(predict_ws(net, W, H, mw, 64, workspace, workspace_bytes, &w));
    return predict_at_scale_impl(net, w, left, right, dtype, W, H, work_width, precision,
                                 disp_full, disp_work, Ww, Hw, (cudaStream_t)stream);
}

int sv_predict_confidence(const sv_net *net, int W, int H, int Ww, int Hw, int probe_width,
                          int max_width, const void *workspace, size_t workspace_bytes,
                          double *spread, double *pmax, void *stream) {
    if (!net || !spread || !pmax) { set_error("NULL argument"); return SV_ERR_NULL; }
    if (W < 1 || H < 1 || Ww < 2 || Hw < 2 || Ww > W || probe_width < 1 || max_width < 1) {
        set_error("bad sizes");
        return SV_ERR_SHAPE;
    }
    PredictWs w;
    SV_TRY(predict_ws(net, W, H, max_width, probe_width, const_cast<void *>(workspace),
                      workspace_bytes, &w));
    int h1, w1, hq, wq;
    conv_out(Hw, Ww, &h1, &w1, &hq, &wq);
    cudaStream_t st = (cudaStream_t)stream;
    // spread in full-resolution pixels: quarter -> work (x4) -> full (x W / Ww)
    SV_TRY(launch_upscale_disp(w.fwd.qspread, wq, hq, W, H, 4.0 * W / (double)Ww, spread, st));
    return launch_resize_f32(w.fwd.qpmax, wq, hq, W, H, pmax, st);
}

int sv_predict_refine(const sv_net *net, const void *left, const void *right, int dtype, int W,
                      int H, double target_peak, int probe_width, int max_width, int passes,
                      int precision, double *disp_full, double *disp_work, int *pWw, int *pHw,
                      int *work_trace, void *pworkspace, size_t pworkspace_bytes, double tol,
                      const sv_refine_params *p, double *out, uint8_t *status,
                      void *rworkspace, size_t rworkspace_bytes, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    SideStream *ss = nullptr;
    if (st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread) {
        // lr_refine's census needs the images alone: it runs on a second
        // stream beside predict_auto's small network launches, and the rest
        // of lr_refine waits for it
        if (side_stream(&ss) == SV_OK) {
            int rc = SV_OK;
            if (cudaEventRecord(ss->fork, st) != cudaSuccess ||
                cudaStreamWaitEvent(ss->s, ss->fork, 0) != cudaSuccess) {
                set_error("stream fork failed");
                return SV_ERR_CUDA;
            }
            rc = lr_refine_census(left, right, dtype, W, H, p, rworkspace, rworkspace_bytes,
                                  ss->s);
            if (cudaEventRecord(ss->join, ss->s) != cudaSuccess ||
                cudaStreamWaitEvent(st, ss->join, 0) != cudaSuccess) {
                set_error("stream join failed");
                return SV_ERR_CUDA;
            }
            if (rc) return rc;
        } else {
            ss = nullptr;
        }
    }
    const int rc = sv_predict_auto(net, left, right, dtype, W, H, target_peak, probe_width,
                                   max_width, passes, precision, disp_full, disp_work, pWw, pHw,
                                   work_trace, pworkspace, pworkspace_bytes, stream);
    if (rc) return rc;
    if (ss)
        return lr_refine_after_census(left, right, dtype, disp_full, W, H, tol, p, out, status,
                                      rworkspace, rworkspace_bytes, st);
    return sv_lr_refine(left, right, dtype, disp_full, W, H, tol, p, out, status, rworkspace,
                        rworkspace_bytes, stream);
}

int sv_predict_auto(const sv_net *net, const void *left, const void *right, int dtype, int W,
                    int H, double target_peak, int probe_width, int max_width, int passes,
                    int precision, double *disp_full, double *disp_work, int *pWw, int *pHw,
                    int *work_trace, void *workspace, size_t workspace_bytes, void *stream) {
    if (!net || !left || !right || !disp_full || !disp_work || !pWw || !pHw) {
        set_error("NULL argument");
        return SV_ERR_NULL;
    }
    if (precision != SV_FP32 && precision != SV_BF16) {
        set_error("precision %d is neither SV_FP32 nor SV_BF16", precision);
        return SV_ERR_PARAM;
    }
    if (W < 1 || H < 1 || probe_width < 1 || max_width < 1 || passes < 1 ||
        !std::isfinite(target_peak)) {
        set_error("bad arguments");
        return SV_ERR_PARAM;
    }
    cudaStream_t st = (cudaStream_t)stream;
    sv_net *mnet = const_cast<sv_net *>(net);       // only its graph cache changes
    PredictWs w;
    SV_TRY(predict_ws(net, W, H, max_width, probe_width, workspace, workspace_bytes, &w));
    // probe (stereonet.py:3900-3907)
    const int pw = probe_width < W ? probe_width : W;
    int ph = (int)(H * pw / (double)W + 0.5);
    if (ph < 8) ph = 8;
    // BF16 runs only where no work-width decision follows: the probe and the
    // passes whose 95% quantile picks the next width stay FP32, so the widths
    // are FP32's; the last permitted pass (no select after it) runs at the
    // requested precision.
    sv_graph_key key{0, W, H, dtype, pw * 65536 + ph, 1, SV_FP32, left, right, disp_full,
                     disp_work, workspace};
    // The width decisions: from a histogram of the widths the rule gives the
    // map's values (no value select) whenever the rule has at most
    // kWidthBins + 1 widths (every max_width up to 2095).
    const WidthRule probe_rule{W, max_width, target_peak, W / (double)pw};
    const WidthRule full_rule{W, max_width, target_peak, 1.0};
    const int kmax = width_rule_kmax(full_rule), nth = kmax - 48;
    const bool by_rule = nth <= kWidthBins;
    double *slot = nullptr;
    SV_TRY(run_stage(mnet, key, st, true, &slot, [&](double *mirror) -> int {
        int rc = check_net_shape(net->view, ph, pw);
        const long np = (long)pw * ph;
        const long long rank = (long long)(np * 0.95);
        if (by_rule) {
            // the probe's decision runs in the network's output convolution;
            // the stage's resize clears its state
            const WidthFuse f{probe_rule, nth, kmax, rank};
            const SelFuse sf{w.sel, w.hist, rank, &f, mirror};
            if (!rc)
                rc = launch_resize_pair(left, right, dtype, W, H, pw, ph, w.lw, w.rw, st, w.gh,
                                        &sf);
            if (!rc) rc = predict_f32(net, w, pw, ph, SV_FP32, st, true, &sf);
            return rc;
        }
        if (!rc) rc = launch_resize_pair(left, right, dtype, W, H, pw, ph, w.lw, w.rw, st, w.gh);
        if (!rc) rc = predict_f32(net, w, pw, ph, SV_FP32, st, true);
        if (!rc && np <= 16384) {
            rc = launch_select_small_f32(w.d2, np, rank, w.sel, st, mirror);
        } else if (!rc) {
            rc = launch_promote(w.d2, np, w.probe64, st);
            if (!rc) rc = launch_select(w.probe64, np, rank, w.sel, w.hist, st, mirror);
        }
        return rc;
    }));
    int work;
    if (by_rule) {
        double wv;
        SV_TRY(fetch_peak(w, st, slot, &wv, false));
        work = (int)wv;
    } else {
        double pk;
        SV_TRY(fetch_peak(w, st, slot, &pk));
        const double peak = pk * (W / (double)pw);
        work = width_for(W, target_peak, max_width, peak);
    }
    int nt = 0;
    if (work_trace) work_trace[nt++] = work;
    // passes (stereonet.py:3908-3929): the peak after pass i is needed only
    // when another pass may follow
    for (int pass = 1;; ++pass) {
        const bool with_sel = pass < passes;
        const int prec = with_sel ? SV_FP32 : precision;
        sv_graph_key k{1, W, H, dtype, work, with_sel ? 1 : 0, prec, left, right, disp_full,
                       disp_work, workspace};
        int Ww, Hw;
        SV_TRY(run_stage(mnet, k, st, with_sel, &slot, [&](double *mirror) -> int {
            const long nf = (long)W * H;
            const long long rank = (long long)((long)W * H * 0.95);
            if (by_rule) {
                // the whole decision runs inside the pass when it resamples
                const bool fuse = with_sel && work < W;
                const WidthFuse f{full_rule, nth, kmax, rank};
                const SelFuse sf{w.sel, w.hist, rank, &f, mirror};
                int rc = predict_at_scale_impl(net, w, left, right, dtype, W, H, work, prec,
                                               disp_full, disp_work, &Ww, &Hw, st,
                                               fuse ? &sf : nullptr);
                if (!rc && with_sel && !fuse)
                    rc = launch_width_map<double>(disp_full, nf, f, w.sel, w.hist, st, mirror);
                return rc;
            }
            // the select's pass 0 runs inside the pass when it resamples
            const bool fuse = with_sel && work < W && nf > select_small_cap();
            const SelFuse sf{w.sel, w.hist, rank};
            int rc = predict_at_scale_impl(net, w, left, right, dtype, W, H, work, prec,
                                           disp_full, disp_work, &Ww, &Hw, st,
                                           fuse ? &sf : nullptr);
            if (!rc && fuse)
                rc = launch_select_after_pass0(disp_full, nf, w.sel, w.hist, st, mirror);
            else if (!rc && with_sel)
                rc = launch_select(disp_full, nf, rank, w.sel, w.hist, st, mirror);
            return rc;
        }));
        work_dims(W, H, work, &Ww, &Hw);
        *pWw = Ww;
        *pHw = Hw;
        if (!with_sel) break;
        int nw;
        if (by_rule) {
            double wv;
            SV_TRY(fetch_peak(w, st, slot, &wv, false));
            nw = (int)wv;
        } else {
            double np_;
            SV_TRY(fetch_peak(w, st, slot, &np_));
            nw = width_for(W, target_peak, max_width, np_);
        }
        if (std::abs(nw - work) <= 0.08 * work) break;
        work = nw;
        if (work_trace) work_trace[nt++] = work;
    }
    if (work_trace) work_trace[nt] = 0;
    return SV_OK;
}

// Self-test of the host side of a stage's peak hand-off: arm a mapped slot
// that no kernel will write, and poll it while the stream has nothing queued.
// The poll must give up with SV_ERR_TIMEOUT instead of waiting forever.
int sv_selftest_slot_wait(void *stream) {
    void *h = nullptr;
    SV_CUDA_TRY(cudaHostAlloc(&h, 64, cudaHostAllocMapped | cudaHostAllocPortable));
    double *slot = static_cast<double *>(h);
    arm_slot(slot);
    double v = 0.0;
    const int rc = wait_slot(slot, (cudaStream_t)stream, &v);
    cudaFreeHost(h);
    return rc;
}

// Self-test of the device side: one CTA holding tensor memory waits, at most
// `limit` polls, on an mbarrier nothing arrives at (launch_selftest_wait).
int sv_selftest_wait_timeout(unsigned limit, int *flag_done, void *stream) {
    if (!flag_done) { set_error("NULL argument"); return SV_ERR_NULL; }
    return launch_selftest_wait(limit, flag_done, flag_done + 1, (cudaStream_t)stream);
}

}  // extern "C"

// ------------------------------------------- network-level LR consistency
#include "sv_post.cuh"

namespace {

size_t dtype_size(int dtype) {
    return dtype == SV_U8 ? 1 : dtype == SV_F32 ? 4 : dtype == SV_F64 ? 8 : 0;
}

struct ConsistWs {
    unsigned char *ml, *mr;
    double *dl, *dwork, *drm, *dr;
    uint8_t *valid;
    int *scratch;
    unsigned long long *kept;
    void *pws;
};

size_t carve_consist(void *ws, const sv_net *net, int W, int H, int dtype, int max_width,
                     size_t *pneed, ConsistWs *o) {
    Carver cv(ws);
    ConsistWs c{};
    const size_t N = (size_t)W * H, es = dtype_size(dtype);
    c.ml = cv.take<unsigned char>(N * es);
    c.mr = cv.take<unsigned char>(N * es);
    c.dl = cv.take<double>(N);
    c.dwork = cv.take<double>(N > 4096 ? N : 4096);
    c.drm = cv.take<double>(N);
    c.dr = cv.take<double>(N);
    c.valid = cv.take<uint8_t>(N);
    c.scratch = cv.take<int>(N);
    c.kept = cv.take<unsigned long long>(1);
    const size_t pn = sv_predict_workspace_size(net, W, H, max_width);
    c.pws = cv.take<unsigned char>(pn);
    if (pneed) *pneed = pn;
    if (o) *o = c;
    return cv.off;
}

}  // namespace

extern "C" {

size_t sv_predict_consistent_workspace_size(const sv_net *net, int W, int H, int dtype,
                                            int max_width) {
    if (!net || W < 1 || H < 1 || !dtype_size(dtype)) return 0;
    return carve_consist(nullptr, net, W, H, dtype, max_width < 48 ? 48 : max_width, nullptr,
                         nullptr);
}

int sv_predict_consistent(const sv_net *net, const void *left, const void *right, int dtype,
                          int W, int H, int work_width, double target_peak, int probe_width,
                          int max_width, int passes, double tol, int precision,
                          double *disp_out, long long *kept, void *workspace,
                          size_t workspace_bytes, void *stream) {
    if (!net || !left || !right || !disp_out || !kept) {
        set_error("NULL argument");
        return SV_ERR_NULL;
    }
    if (W < 1 || H < 1 || !dtype_size(dtype)) { set_error("bad shape or dtype"); return SV_ERR_SHAPE; }
    if (!std::isfinite(tol)) { set_error("tol must be finite"); return SV_ERR_PARAM; }
    const int mw = work_width > 0 ? (work_width > 48 ? work_width : 48) : max_width;
    const size_t need = sv_predict_consistent_workspace_size(net, W, H, dtype, mw);
    if (!workspace || ((uintptr_t)workspace & 255) || workspace_bytes < need) {
        set_error("workspace needs %zu bytes, 256-aligned", need);
        return SV_ERR_WORKSPACE;
    }
    ConsistWs c;
    size_t pn = 0;
    carve_consist(workspace, net, W, H, dtype, mw < 48 ? 48 : mw, &pn, &c);
    cudaStream_t st = (cudaStream_t)stream;
    int Ww = 0, Hw = 0;
    // predict_consistent, stereonet.py:5048-5076
    if (work_width <= 0)
        SV_TRY(sv_predict_auto(net, left, right, dtype, W, H, target_peak, probe_width, max_width,
                               passes, precision, c.dl, c.dwork, &Ww, &Hw, nullptr, c.pws, pn,
                               stream));
    else
        SV_TRY(sv_predict_at_scale(net, left, right, dtype, W, H, work_width, precision, c.dl,
                                   c.dwork, &Ww, &Hw, c.pws, pn, stream));
    const int es = (int)dtype_size(dtype);
    SV_TRY(launch_mirror(left, es, W, H, c.ml, st));
    SV_TRY(launch_mirror(right, es, W, H, c.mr, st));
    SV_TRY(sv_predict_at_scale(net, c.mr, c.ml, dtype, W, H, Ww, precision, c.drm, c.dwork, &Ww,
                               &Hw, c.pws, pn, stream));
    SV_TRY(launch_mirror(c.drm, 8, W, H, c.dr, st));
    SV_TRY(launch_lr_consistency(c.dl, c.dr, W, H, tol, c.valid, c.kept, st));
    SV_TRY(launch_fill_invalid(c.dl, c.valid, W, H, c.scratch, disp_out, st));
    unsigned long long k = 0;
    SV_CUDA_TRY(cudaMemcpyAsync(&k, c.kept, sizeof(k), cudaMemcpyDeviceToHost, st));
    SV_CUDA_TRY(cudaStreamSynchronize(st));
    *kept = (long long)k;
    return SV_OK;
}

}  // extern "C"
