// C ABI of libpivb200.so: analyzer and frame handles, the multipass driver (multipass.rs:152-259)
// on one CUDA stream with no host synchronisation between passes, and the stage hooks.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/piv_b200.h"
#include "common.cuh"
#include "kernels.h"

using namespace pivb200;

namespace {

thread_local std::string g_last_error;

}  // namespace

void pivb200::set_last_error(const char* msg) { g_last_error = msg; }

namespace {

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                          \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess) return fail(PIV_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

// Grid::new (grid.rs:20-44), f32 step arithmetic as the reference.
int make_grid(int64_t h, int64_t w, int64_t window, float overlap, PivGridC* g) {
    if (!(overlap >= 0.0f && overlap < 1.0f)) return fail(PIV_ERR_CONFIG, "overlap %g must be in [0, 1)", overlap);
    if (window <= 0 || window > w || window > h)
        return fail(PIV_ERR_IMAGE_TOO_SMALL, "image (%lldx%lld) is smaller than the %lld px interrogation window",
                    (long long)h, (long long)w, (long long)window);
    const float st = std::round((float)window * (1.0f - overlap));
    int64_t step = st > 0.0f ? (int64_t)st : 0;
    if (step < 1) step = 1;
    g->window = window;
    g->step = step;
    g->nx = (w - window) / step + 1;
    g->ny = (h - window) / step + 1;
    g->x0 = (w - window - (g->nx - 1) * step) / 2;
    g->y0 = (h - window - (g->ny - 1) * step) / 2;
    return PIV_OK;
}

GridP to_gp(const PivGridC& g) {
    return GridP{(int32_t)g.window, (int32_t)g.step, (int32_t)g.nx, (int32_t)g.ny, (int32_t)g.x0, (int32_t)g.y0};
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct PassBuf {
    PivGridC grid;
    int64_t cells;
    float4* origins;
    uint8_t* status;
    float* raw_dx;
    float* raw_dy;
    float* raw_ppr;
    uint8_t* raw_flags;
    uint8_t* f1;
    uint8_t* f2;
    float* dx;
    float* dy;
    uint8_t* flags;
    float4* corners;  // deformed windows: predictor at the 4 corner pixels (2 float4 per cell)
};

std::mutex g_init_mu;
std::vector<int> g_inited_devices;

int ensure_device_init(int dev) {
    std::lock_guard<std::mutex> lk(g_init_mu);
    for (int d : g_inited_devices)
        if (d == dev) return PIV_OK;
    CUDA_TRY(corr_init_device());
    CUDA_TRY(corr_tc_init_device());
    g_inited_devices.push_back(dev);
    return PIV_OK;
}

}  // namespace

struct PivAnalyzer {
    std::vector<int32_t> windows;
    float overlap = 0.5f;
    int32_t final_iterations = 2;
    float min_mean = 0.0f, min_std = 0.0f;
    float ppr_threshold = 1.3f, median_threshold = 2.0f, median_eps = 0.1f;
    int32_t replace = 1;
    int32_t deform = 0;
    int32_t precision = PIV_PRECISION_FP32;
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t cur = nullptr;
    // per-pair workspace, sized for (H, W)
    int64_t H = 0, W = 0;
    int K = 0;                                // pairs the workspace holds
    std::vector<std::vector<PassBuf>> pairs;  // [pair][pass]
    void* arena = nullptr;
    unsigned long long* d_counts = nullptr;
    long long launches = 0;
    // stage timing: per pass, pending (start, end) event pairs and the events to reuse
    bool profiling = false;
    std::vector<std::vector<std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<cudaEvent_t> spare;

    // correlation launch variant chosen per window size (0 until autotuned), uniform / deformed
    int variant[2][129] = {};
    // with tensor cores allowed: window sizes where the autotuner found the FP32 kernel faster
    bool fp32_faster[2][129] = {};  // [uniform / deformed windows][window]
    // launch choices change (autotune, variant pinning): cached pass graphs are stale
    uint64_t epoch = 0;
    // the passes of the last repeated call, as a CUDA graph replayed while its key holds
    cudaGraphExec_t gexec = nullptr;
    std::vector<uintptr_t> gkey, pending_key;
    long long gnl = 0;  // kernels in the graph

    bool mask_trivial() const { return min_mean <= 0.0f && min_std <= 0.0f; }
    std::vector<int32_t> pass_windows() const {
        std::vector<int32_t> v = windows;
        for (int i = 1; i < final_iterations; ++i) v.push_back(windows.back());
        return v;
    }
};

struct PivFrame {
    PivAnalyzer* an = nullptr;
    int device = 0;
    int64_t H = 0, W = 0;
    float* image = nullptr;
    float* base = nullptr;  // background-subtracted intensity; aliases image when no blur/normalize
    float* base_store = nullptr;
    float* tmp = nullptr;
    long long* sum = nullptr;
    long long* sumsq = nullptr;
    int* scales = nullptr;
    unsigned int* words = nullptr;  // maxbits[2] + histogram scratch
    bool stats_valid = false;
    bool nonneg = false;
    void* d_raw = nullptr;
    size_t d_raw_bytes = 0;
    float* d_bg = nullptr;
};

struct PivBatch {
    PivAnalyzer* an = nullptr;  // private analyzer: its workspace is never resized by other calls
    int64_t H = 0, W = 0;
    int K = 0;
    bool sequential = false;
    int32_t dtype = PIV_DTYPE_U16;
    PivPreprocessC pre{};
    size_t frame_bytes = 0;
    void* raw = nullptr;
    const float* background = nullptr;  // device image subtracted from every frame (caller-owned)
    std::vector<PivFrame*> frames;
    int64_t cells = 0;
    void* out = nullptr;
    float* dx = nullptr;
    float* dy = nullptr;
    float* ppr = nullptr;
    uint8_t* flags = nullptr;
    unsigned long long* sums = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;  // kernel launches of the eager run
    int runs = 0;
    // asynchronous host submission: pinned summary counters, the copy streams (uploads and
    // downloads overlap graph replays on the compute stream) and their ordering events
    unsigned long long* hsums = nullptr;
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t uploaded = nullptr, computed = nullptr, hdone = nullptr;
    bool pending = false;
};

namespace {

bool split_precision(int32_t p) { return p == PIV_PRECISION_BF16X3 || p == PIV_PRECISION_FP16X3; }

int check_cfg(const PivConfigC* c) {
    // multipass.rs:91-119
    if (!c) return fail(PIV_ERR_ARGUMENT, "null config");
    if (c->n_windows <= 0 || !c->windows) return fail(PIV_ERR_CONFIG, "at least one window size is required");
    for (int i = 0; i < c->n_windows; ++i)
        if (c->windows[i] < 8 || c->windows[i] % 2 != 0)
            return fail(PIV_ERR_CONFIG, "window size %d must be even and >= 8", c->windows[i]);
    if (!(c->overlap >= 0.0f && c->overlap < 1.0f)) return fail(PIV_ERR_CONFIG, "overlap %g must be in [0, 1)", c->overlap);
    if (c->final_iterations < 1) return fail(PIV_ERR_CONFIG, "final_iterations must be at least 1");
    if (c->deform != 0 && c->deform != 1) return fail(PIV_ERR_CONFIG, "deform must be 0 or 1");
    if (c->precision != PIV_PRECISION_FP32 && c->precision != PIV_PRECISION_BF16X3 &&
        c->precision != PIV_PRECISION_FP16X3)
        return fail(PIV_ERR_CONFIG, "precision must be PIV_PRECISION_FP32, _BF16X3 or _FP16X3");
    for (int i = 0; i < c->n_windows; ++i)
        if (!corr_supported(c->windows[i]))
            return fail(PIV_ERR_UNSUPPORTED, "window size %d is not supported on the GPU (8, 12, 16, 24, 32, 48, 64, 96, 128)",
                        c->windows[i]);
    return PIV_OK;
}

int use_device(PivAnalyzer* an) {
    CUDA_TRY(cudaSetDevice(an->device));
    return PIV_OK;
}

// Per-pair workspace for up to K pairs of (H, W) frames: for every pass, origins, signal status,
// raw field, two flag snapshots and the validated field; 8 summary counters per pair.
int ensure_workspace(PivAnalyzer* an, int64_t H, int64_t W, int K) {
    if (an->arena && an->H == H && an->W == W && an->K >= K) return PIV_OK;
    if (an->arena) {
        CUDA_TRY(cudaStreamSynchronize(an->cur));
        CUDA_TRY(cudaFree(an->arena));
        an->arena = nullptr;
    }
    an->pairs.clear();
    const auto wins = an->pass_windows();
    std::vector<PassBuf> proto;
    size_t per_pair = 0;
    for (int32_t n : wins) {
        PassBuf pb{};
        int st = make_grid(H, W, n, an->overlap, &pb.grid);
        if (st) return st;
        pb.cells = pb.grid.nx * pb.grid.ny;
        if (pb.cells > (int64_t)1 << 30) return fail(PIV_ERR_UNSUPPORTED, "too many windows in one pass");
        const size_t c = (size_t)pb.cells;
        per_pair += align256(16 * c) + align256(c) + 3 * align256(4 * c) + 3 * align256(c) + 2 * align256(4 * c) + align256(c) +
                    (an->deform ? align256(32 * c) : 0);
        proto.push_back(pb);
    }
    const size_t total = align256(sizeof(unsigned long long) * 8 * (size_t)K) + per_pair * (size_t)K;
    CUDA_TRY(cudaMalloc(&an->arena, total));
    char* p = (char*)an->arena;
    auto take = [&](size_t bytes) {
        void* r = p;
        p += align256(bytes);
        return r;
    };
    an->d_counts = (unsigned long long*)take(sizeof(unsigned long long) * 8 * (size_t)K);
    for (int k = 0; k < K; ++k) {
        std::vector<PassBuf> passes = proto;
        for (auto& pb : passes) {
            const size_t c = (size_t)pb.cells;
            pb.origins = (float4*)take(16 * c);
            pb.status = (uint8_t*)take(c);
            pb.raw_dx = (float*)take(4 * c);
            pb.raw_dy = (float*)take(4 * c);
            pb.raw_ppr = (float*)take(4 * c);
            pb.raw_flags = (uint8_t*)take(c);
            pb.f1 = (uint8_t*)take(c);
            pb.f2 = (uint8_t*)take(c);
            pb.dx = (float*)take(4 * c);
            pb.dy = (float*)take(4 * c);
            pb.flags = (uint8_t*)take(c);
            pb.corners = an->deform ? (float4*)take(32 * c) : nullptr;
        }
        an->pairs.push_back(passes);
    }
    an->H = H;
    an->W = W;
    an->K = K;
    return PIV_OK;
}

StatsView stats_of(const PivFrame* f) { return StatsView{f->sum, f->sumsq, f->scales, (int)f->H, (int)f->W}; }

bool needs_stats(const PivAnalyzer* an, const PivFrame* f) { return !an->mask_trivial() || !f->nonneg; }

int alloc_stats(PivFrame* f) {
    if (f->sum) return PIV_OK;
    const size_t cells = (size_t)(f->H + 1) * (size_t)(f->W + 1);
    CUDA_TRY(cudaMalloc(&f->sum, sizeof(long long) * cells));
    CUDA_TRY(cudaMalloc(&f->sumsq, sizeof(long long) * cells));
    return PIV_OK;
}

// The multipass loop (multipass.rs:152-192) for K pairs of equal size at once: every pass is
// placement -> correlation -> validation, each stage ONE launch covering all K pairs, on the
// analyzer's stream; the predictor of pair k is its own previous pass's validated field.
int run_passes_eager(PivAnalyzer* an, const PivFrame* const* a, const PivFrame* const* b, int K, bool tune) {
    if (K <= 0) return fail(PIV_ERR_ARGUMENT, "no pairs");
    for (int k = 0; k < K; ++k) {
        if (!a[k] || !b[k]) return fail(PIV_ERR_ARGUMENT, "null frame");
        if (a[k]->H != b[k]->H || a[k]->W != b[k]->W)
            return fail(PIV_ERR_SHAPE_MISMATCH, "frames have different shapes: (%lld, %lld) vs (%lld, %lld)",
                        (long long)a[k]->H, (long long)a[k]->W, (long long)b[k]->H, (long long)b[k]->W);
        if (a[k]->H != a[0]->H || a[k]->W != a[0]->W)
            return fail(PIV_ERR_SHAPE_MISMATCH, "all pairs of a batch must have the same frame size");
    }
    const int64_t H = a[0]->H, W = a[0]->W;
    int st = use_device(an);
    if (st) return st;
    st = ensure_workspace(an, H, W, K);
    if (st) return st;
    std::vector<int> use_stats(K);
    for (int k = 0; k < K; ++k) {
        use_stats[k] = needs_stats(an, a[k]) || needs_stats(an, b[k]);
        if (use_stats[k] && !(a[k]->stats_valid && b[k]->stats_valid))
            return fail(PIV_ERR_ARGUMENT, "frame statistics missing for the signal mask");
    }
    const size_t npass = an->pairs[0].size();
    std::vector<PlaceParams> pps(K);
    std::vector<CorrParams> cps(K);
    std::vector<ValidateParams> vps(K);
    for (size_t i = 0; i < npass; ++i) {
        for (int k = 0; k < K; ++k) {
            PassBuf& pb = an->pairs[k][i];
            PlaceParams& pp = pps[k];
            pp = PlaceParams{};
            pp.grid = to_gp(pb.grid);
            pp.H = (int)H;
            pp.W = (int)W;
            pp.has_pred = i > 0;
            if (i > 0) {
                pp.pgrid = to_gp(an->pairs[k][i - 1].grid);
                pp.pdx = an->pairs[k][i - 1].dx;
                pp.pdy = an->pairs[k][i - 1].dy;
            }
            pp.origins = pb.origins;
            pp.status = pb.status;
            // Deformed windows need a predictor; the first pass is the uniform placement.
            pp.corners = (an->deform && i > 0) ? pb.corners : nullptr;
            pp.use_stats = use_stats[k];
            if (use_stats[k]) {
                pp.sa = stats_of(a[k]);
                pp.sb = stats_of(b[k]);
            }
            pp.min_mean = an->min_mean;
            pp.min_std = an->min_std;
            cps[k] = CorrParams{a[k]->image, b[k]->image, (int)H, (int)W, pb.origins, pb.status, (int)pb.cells,
                                pb.raw_dx, pb.raw_dy, pb.raw_ppr, pb.raw_flags, pp.corners, (int)pb.grid.x0,
                                (int)pb.grid.y0, (int)pb.grid.step, (int)pb.grid.nx};
            vps[k] = ValidateParams{(int)pb.grid.nx, (int)pb.grid.ny, pb.raw_dx, pb.raw_dy, pb.raw_ppr, pb.raw_flags,
                                    pb.f1, pb.f2, pb.dx, pb.dy, pb.flags, (float)an->windows[0] / 2.0f,
                                    an->ppr_threshold, an->median_threshold, an->median_eps, an->replace};
        }
        int nl = 0;
        CUDA_TRY(launch_place_items(pps.data(), K, an->cur, &nl));
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        if (an->profiling) {
            for (cudaEvent_t* ev : {&ev0, &ev1}) {
                if (!an->spare.empty()) {
                    *ev = an->spare.back();
                    an->spare.pop_back();
                } else {
                    CUDA_TRY(cudaEventCreate(ev));
                }
            }
            CUDA_TRY(cudaEventRecord(ev0, an->cur));
        }
        const int nwin = (int)an->pairs[0][i].grid.window;
        const int kind = cps[0].corners ? 1 : 0;
        const bool tc_ok = split_precision(an->precision) && corr_tc_supported(nwin);
        const bool f16 = an->precision == PIV_PRECISION_FP16X3;
        if (tune) {
            // Time every launch variant of this window size on this pass's data (all compute the
            // same results) and keep the fastest for later calls. With tensor cores allowed, the
            // tensor-core kernel is timed too, and the FP32 kernel (higher precision) is kept
            // for this size when it is faster.
            cudaEvent_t t0, t1;
            CUDA_TRY(cudaEventCreate(&t0));
            CUDA_TRY(cudaEventCreate(&t1));
            float best = 1e30f;
            int best_v = 0;
            for (int v = 0; v < corr_num_variants(nwin, kind); ++v) {
                CUDA_TRY(launch_correlate_items(nwin, v, cps.data(), K, an->cur, &nl));
                CUDA_TRY(cudaEventRecord(t0, an->cur));
                for (int r = 0; r < 3; ++r) CUDA_TRY(launch_correlate_items(nwin, v, cps.data(), K, an->cur, &nl));
                CUDA_TRY(cudaEventRecord(t1, an->cur));
                CUDA_TRY(cudaEventSynchronize(t1));
                float ms = 0.0f;
                CUDA_TRY(cudaEventElapsedTime(&ms, t0, t1));
                if (ms < best) {
                    best = ms;
                    best_v = v;
                }
            }
            an->variant[kind][nwin] = best_v;
            ++an->epoch;
            if (tc_ok) {
                CUDA_TRY(launch_correlate_tc_items(nwin, f16, cps.data(), K, an->cur, &nl));
                CUDA_TRY(cudaEventRecord(t0, an->cur));
                for (int r = 0; r < 3; ++r) CUDA_TRY(launch_correlate_tc_items(nwin, f16, cps.data(), K, an->cur, &nl));
                CUDA_TRY(cudaEventRecord(t1, an->cur));
                CUDA_TRY(cudaEventSynchronize(t1));
                float ms = 0.0f;
                CUDA_TRY(cudaEventElapsedTime(&ms, t0, t1));
                an->fp32_faster[kind][nwin] = best < ms;
            }
            cudaEventDestroy(t0);
            cudaEventDestroy(t1);
        }
        const bool tensor = tc_ok && !an->fp32_faster[kind][nwin];
        if (tensor)
            CUDA_TRY(launch_correlate_tc_items(nwin, f16, cps.data(), K, an->cur, &nl));
        else
            CUDA_TRY(launch_correlate_items(nwin, an->variant[kind][nwin], cps.data(), K, an->cur, &nl));
        if (an->profiling) {
            CUDA_TRY(cudaEventRecord(ev1, an->cur));
            if (an->pending.size() < npass) an->pending.resize(npass);
            an->pending[i].push_back({ev0, ev1});
        }
        CUDA_TRY(launch_validate_items(vps.data(), K, an->cur, &nl));
        an->launches += nl;
    }
    std::vector<SummaryItem> sums(K);
    for (int k = 0; k < K; ++k) {
        const PassBuf& last = an->pairs[k].back();
        sums[k] = SummaryItem{last.flags, (int)last.cells, an->d_counts + 8 * (size_t)k};
    }
    int nl = 0;
    CUDA_TRY(launch_summary_items(sums.data(), K, an->cur, &nl));
    an->launches += nl;
    return PIV_OK;
}

// All passes of K pairs on the analyzer's stream. A call that repeats the previous call's launch
// sequence exactly (same frames and their buffers, sizes, workspace and launch choices: the key)
// is captured once as a CUDA graph, and later calls with that key replay it, which removes the
// per-kernel launch cost that dominates small frames. The graph reads the frames' current
// contents, so new samples in the same frames need no new capture. Tuning, profiling and a
// stream that the caller is capturing run eagerly.
int run_passes(PivAnalyzer* an, const PivFrame* const* a, const PivFrame* const* b, int K, bool tune = false) {
    if (tune || an->profiling || K <= 0) {
        an->pending_key.clear();
        return run_passes_eager(an, a, b, K, tune);
    }
    for (int k = 0; k < K; ++k)
        if (!a[k] || !b[k] || a[k]->H != a[0]->H || a[k]->W != a[0]->W || b[k]->H != a[0]->H || b[k]->W != a[0]->W)
            return run_passes_eager(an, a, b, K, tune);  // reports the error
    int st = use_device(an);
    if (st) return st;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(an->cur, &cap));
    if (cap != cudaStreamCaptureStatusNone) return run_passes_eager(an, a, b, K, tune);
    st = ensure_workspace(an, a[0]->H, a[0]->W, K);
    if (st) return st;
    std::vector<uintptr_t> key = {(uintptr_t)K, (uintptr_t)a[0]->H, (uintptr_t)a[0]->W, (uintptr_t)an->arena,
                                  (uintptr_t)an->epoch};
    for (int k = 0; k < K; ++k)
        for (const PivFrame* f : {a[k], b[k]})
            for (uintptr_t v : {(uintptr_t)f, (uintptr_t)f->image, (uintptr_t)f->sum, (uintptr_t)f->sumsq,
                                (uintptr_t)f->scales, (uintptr_t)needs_stats(an, f), (uintptr_t)f->stats_valid})
                key.push_back(v);
    if (an->gexec && key == an->gkey) {
        CUDA_TRY(cudaGraphLaunch(an->gexec, an->cur));
        an->launches += an->gnl;
        return PIV_OK;
    }
    if (key != an->pending_key) {  // first call with this key: eager
        an->pending_key = key;
        return run_passes_eager(an, a, b, K, tune);
    }
    // second call with the same key: capture, then replay
    CUDA_TRY(cudaStreamBeginCapture(an->cur, cudaStreamCaptureModeRelaxed));
    const long long l0 = an->launches;
    st = run_passes_eager(an, a, b, K, tune);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(an->cur, &graph);
    const long long nl = an->launches - l0;
    an->launches = l0;
    if (st) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (ce != cudaSuccess) return fail(PIV_ERR_CUDA, "pass graph capture: %s", cudaGetErrorString(ce));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return fail(PIV_ERR_CUDA, "pass graph instantiation: %s", cudaGetErrorString(ie));
    if (an->gexec) cudaGraphExecDestroy(an->gexec);
    an->gexec = exec;
    an->gkey = key;
    an->gnl = nl;
    CUDA_TRY(cudaGraphLaunch(exec, an->cur));
    an->launches += nl;
    return PIV_OK;
}

int run_passes(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, bool tune = false) {
    return run_passes(an, &a, &b, 1, tune);
}

// After a synchronisation: a tensor-core kernel whose bounded wait ran out leaves its results
// undefined and sets the device's error word.
int check_device_error(int dev) {
    if (corr_tc_error(dev)) return fail(PIV_ERR_CUDA, "a tensor-core correlation wait timed out on device %d", dev);
    return PIV_OK;
}

int copy_summary(PivAnalyzer* an, PivSummaryC* s) {
    if (!s) return PIV_OK;
    unsigned long long c[5];
    CUDA_TRY(cudaMemcpyAsync(c, an->d_counts, sizeof(c), cudaMemcpyDeviceToHost, an->cur));
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    s->no_signal = (int64_t)c[0];
    s->low_ppr = (int64_t)c[1];
    s->median_outliers = (int64_t)c[2];
    s->out_of_range = (int64_t)c[3];
    s->replaced = (int64_t)c[4];
    return PIV_OK;
}

size_t dtype_size(int32_t dtype) {
    switch (dtype) {
        case PIV_DTYPE_U8: return 1;
        case PIV_DTYPE_U16: return 2;
        case PIV_DTYPE_F32: return 4;
        default: return 0;
    }
}

int prepare_common(PivAnalyzer* an, PivFrame* f, const void* raw_dev, int32_t dtype, const PivPreprocessC* pre,
                   const float* bg_dev) {
    PivPreprocessC dflt{1.0f, 4, 0.02f, 0.0};
    if (!pre) pre = &dflt;
    if (pre->clip_percentile > 0.0 && dtype == PIV_DTYPE_F32)
        return fail(PIV_ERR_UNSUPPORTED, "percentile clipping needs integer (u8/u16) samples");
    if (pre->normalize_radius > 16) return fail(PIV_ERR_UNSUPPORTED, "normalize_radius > 16 is not supported");
    if (pre->smooth_sigma > 0.0f && std::ceil(3.0f * pre->smooth_sigma) > 32.0f)
        return fail(PIV_ERR_UNSUPPORTED, "smooth_sigma > 32/3 is not supported");
    const bool chain = pre->smooth_sigma > 0.0f || pre->normalize_radius > 0;
    f->nonneg = dtype != PIV_DTYPE_F32 || bg_dev != nullptr;
    const size_t n = (size_t)f->H * (size_t)f->W;
    if (chain && !f->base_store) CUDA_TRY(cudaMalloc(&f->base_store, sizeof(float) * n));
    if (pre->smooth_sigma > 0.0f && pre->normalize_radius > 0 && !f->tmp) CUDA_TRY(cudaMalloc(&f->tmp, sizeof(float) * n));
    f->base = chain ? f->base_store : f->image;
    const bool stats = needs_stats(an, f);
    if (stats) {
        int st = alloc_stats(f);
        if (st) return st;
    }
    PrepParams pp{};
    pp.H = (int)f->H;
    pp.W = (int)f->W;
    pp.raw = raw_dev;
    pp.raw_type = dtype == PIV_DTYPE_U8 ? RAW_U8 : (dtype == PIV_DTYPE_U16 ? RAW_U16 : RAW_F32);
    pp.background = bg_dev;
    pp.clip_percentile_on = pre->clip_percentile > 0.0;
    pp.clip_percentile = pre->clip_percentile;
    pp.hist = f->words + 4;
    pp.base = f->base;
    pp.image = f->image;
    pp.tmp = f->tmp;
    pp.smooth_sigma = pre->smooth_sigma;
    pp.normalize_radius = pre->normalize_radius;
    pp.normalize_eps = pre->normalize_eps;
    pp.build_stats = stats;
    pp.sum = f->sum;
    pp.sumsq = f->sumsq;
    pp.scales = f->scales;
    pp.maxbits = f->words;
    int nl = 0;
    CUDA_TRY(launch_prepare(pp, an->cur, &nl));
    an->launches += nl;
    f->stats_valid = stats;
    return PIV_OK;
}

int stage_raw(PivFrame* f, size_t bytes) {
    if (f->d_raw_bytes >= bytes) return PIV_OK;
    if (f->d_raw) CUDA_TRY(cudaFree(f->d_raw));
    f->d_raw = nullptr;
    f->d_raw_bytes = 0;
    CUDA_TRY(cudaMalloc(&f->d_raw, bytes));
    f->d_raw_bytes = bytes;
    return PIV_OK;
}

__global__ void background_kernel(const void* frames, int dtype, long long count, long long npix, int mode, float* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (long long k = 0; k < count; ++k) {
            float v;
            if (dtype == PIV_DTYPE_U8)
                v = __fdiv_rn((float)((const uint8_t*)frames)[k * npix + i], 255.0f);
            else if (dtype == PIV_DTYPE_U16)
                v = __fdiv_rn((float)((const uint16_t*)frames)[k * npix + i], 65535.0f);
            else
                v = ((const float*)frames)[k * npix + i];
            if (k == 0)
                acc = v;
            else if (mode == 0)
                acc = fminf(acc, v);
            else
                acc = __fadd_rn(acc, v);
        }
        if (mode == 1) acc = __fdiv_rn(acc, (float)count);
        out[i] = acc;
    }
}

}  // namespace

extern "C" {

int32_t piv_abi_version(void) { return PIV_B200_ABI_VERSION; }

const char* piv_last_error(void) { return g_last_error.c_str(); }

int32_t piv_grid(int64_t height, int64_t width, int64_t window, float overlap, PivGridC* out) {
    if (!out) return fail(PIV_ERR_ARGUMENT, "null output");
    return make_grid(height, width, window, overlap, out);
}

int32_t piv_check_config(const PivConfigC* cfg) { return check_cfg(cfg); }

int32_t piv_analyzer_create(const PivConfigC* cfg, PivAnalyzer** out) {
    if (!out) return fail(PIV_ERR_ARGUMENT, "null output");
    *out = nullptr;
    int st = check_cfg(cfg);
    if (st) return st;
    int dev = cfg->device;
    if (dev < 0) CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaSetDevice(dev));
    st = ensure_device_init(dev);
    if (st) return st;
    PivAnalyzer* an = new PivAnalyzer();
    an->windows.assign(cfg->windows, cfg->windows + cfg->n_windows);
    an->overlap = cfg->overlap;
    an->final_iterations = cfg->final_iterations;
    an->min_mean = cfg->min_mean;
    an->min_std = cfg->min_std;
    an->ppr_threshold = cfg->ppr_threshold;
    an->median_threshold = cfg->median_threshold;
    an->median_eps = cfg->median_eps;
    an->replace = cfg->replace;
    an->deform = cfg->deform;
    an->precision = cfg->precision;
    an->device = dev;
    cudaError_t e = cudaStreamCreateWithFlags(&an->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete an;
        return fail(PIV_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    an->cur = an->own;
    *out = an;
    return PIV_OK;
}

void piv_analyzer_destroy(PivAnalyzer* an) {
    if (!an) return;
    cudaSetDevice(an->device);
    // Only the analyzer's own stream is known to be alive here; cudaFree waits for the device.
    if (an->own) cudaStreamSynchronize(an->own);
    for (auto& v : an->pending)
        for (auto& pr : v) {
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
    for (cudaEvent_t e : an->spare) cudaEventDestroy(e);
    if (an->gexec) {
        cudaDeviceSynchronize();  // a replay may still run on a caller's stream
        cudaGraphExecDestroy(an->gexec);
    }
    if (an->arena) cudaFree(an->arena);
    if (an->own) cudaStreamDestroy(an->own);
    delete an;
}

int32_t piv_num_passes(const PivAnalyzer* an) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    return (int32_t)an->pass_windows().size();
}

int32_t piv_output_grid(const PivAnalyzer* an, int64_t height, int64_t width, PivGridC* out) {
    if (!an || !out) return fail(PIV_ERR_ARGUMENT, "null argument");
    return make_grid(height, width, an->windows.back(), an->overlap, out);
}

int32_t piv_pass_grid(const PivAnalyzer* an, int64_t height, int64_t width, int32_t pass, PivGridC* out) {
    if (!an || !out) return fail(PIV_ERR_ARGUMENT, "null argument");
    const auto w = an->pass_windows();
    if (pass < 0 || pass >= (int32_t)w.size()) return fail(PIV_ERR_ARGUMENT, "pass %d out of range", pass);
    return make_grid(height, width, w[pass], an->overlap, out);
}

int32_t piv_analyzer_set_stream(PivAnalyzer* an, void* stream) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    an->cur = stream ? (cudaStream_t)stream : an->own;
    return PIV_OK;
}

int32_t piv_analyzer_sync(PivAnalyzer* an) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    int st = use_device(an);
    if (st) return st;
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    return check_device_error(an->device);
}

int64_t piv_analyzer_launches(const PivAnalyzer* an) { return an ? an->launches : 0; }

int32_t piv_analyzer_autotune(PivAnalyzer* an, const PivFrame* a, const PivFrame* b) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    int st = run_passes(an, a, b, true);
    if (st) return st;
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    return PIV_OK;
}

int32_t piv_analyzer_variant(const PivAnalyzer* an, int32_t window, char* name, int32_t capacity) {
    if (!an || !name || capacity <= 0) return fail(PIV_ERR_ARGUMENT, "bad argument");
    if (!corr_supported(window)) return fail(PIV_ERR_UNSUPPORTED, "window size %d", window);
    const int kind = an->deform ? 1 : 0;
    if (split_precision(an->precision) && corr_tc_supported(window) && !an->fp32_faster[kind][window])
        snprintf(name, (size_t)capacity, "%d/tensor-core/%s", window,
                 an->precision == PIV_PRECISION_FP16X3 ? "fp16x3" : "bf16x3");
    else
        snprintf(name, (size_t)capacity, "%s", corr_variant_name(window, an->variant[kind][window], kind));
    return PIV_OK;
}

int32_t piv_num_variants(int32_t window) { return corr_supported(window) ? corr_num_variants(window, false) : 0; }

int32_t piv_analyzer_set_variant(PivAnalyzer* an, int32_t window, int32_t v) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    if (!corr_supported(window)) return fail(PIV_ERR_UNSUPPORTED, "window size %d", window);
    const int kind = an->deform ? 1 : 0;
    if (v < 0 || v >= corr_num_variants(window, kind))
        return fail(PIV_ERR_ARGUMENT, "variant %d out of range for window %d", v, window);
    an->variant[kind][window] = v;
    an->fp32_faster[kind][window] = true;  // an explicit FP32 launch variant
    ++an->epoch;
    return PIV_OK;
}

int32_t piv_analyzer_set_profiling(PivAnalyzer* an, int32_t enable) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    an->profiling = enable != 0;
    return PIV_OK;
}

int32_t piv_analyzer_profile(PivAnalyzer* an, int32_t pass, double* correlate_ms, int64_t* launches) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    int st = use_device(an);
    if (st) return st;
    double ms = 0.0;
    int64_t n = 0;
    if (pass >= 0 && pass < (int32_t)an->pending.size()) {
        CUDA_TRY(cudaStreamSynchronize(an->cur));
        for (auto& pr : an->pending[pass]) {
            float t = 0.0f;
            CUDA_TRY(cudaEventElapsedTime(&t, pr.first, pr.second));
            ms += t;
            ++n;
            an->spare.push_back(pr.first);
            an->spare.push_back(pr.second);
        }
        an->pending[pass].clear();
    }
    if (correlate_ms) *correlate_ms = ms;
    if (launches) *launches = n;
    return PIV_OK;
}

int32_t piv_frame_create(PivAnalyzer* an, int64_t height, int64_t width, PivFrame** out) {
    if (!an || !out) return fail(PIV_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    if (height <= 0 || width <= 0 || height > (1 << 16) || width > (1 << 16))
        return fail(PIV_ERR_ARGUMENT, "frame size %lldx%lld out of range", (long long)height, (long long)width);
    int st = use_device(an);
    if (st) return st;
    PivFrame* f = new PivFrame();
    f->an = an;
    f->device = an->device;
    f->H = height;
    f->W = width;
    const size_t n = (size_t)height * (size_t)width;
    cudaError_t e = cudaMalloc(&f->image, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMalloc(&f->words, sizeof(unsigned int) * (4 + 512 + 4));
    if (e == cudaSuccess) e = cudaMalloc(&f->scales, sizeof(int) * 2);
    if (e != cudaSuccess) {
        piv_frame_destroy(f);
        return fail(PIV_ERR_CUDA, "frame allocation: %s", cudaGetErrorString(e));
    }
    f->base = f->image;
    *out = f;
    return PIV_OK;
}

void piv_frame_destroy(PivFrame* f) {
    if (!f) return;
    // A frame may outlive its analyzer: touch nothing of it. cudaFree synchronises the device.
    cudaSetDevice(f->device);
    cudaFree(f->image);
    cudaFree(f->base_store);
    cudaFree(f->tmp);
    cudaFree(f->sum);
    cudaFree(f->sumsq);
    cudaFree(f->scales);
    cudaFree(f->words);
    cudaFree(f->d_raw);
    cudaFree(f->d_bg);
    delete f;
}

int32_t piv_frame_prepare_device(PivAnalyzer* an, PivFrame* f, const void* raw_dev, int32_t dtype,
                                 const PivPreprocessC* pre, const float* background_dev) {
    if (!an || !f || !raw_dev) return fail(PIV_ERR_ARGUMENT, "null argument");
    if (!dtype_size(dtype)) return fail(PIV_ERR_ARGUMENT, "unknown dtype %d", dtype);
    int st = use_device(an);
    if (st) return st;
    return prepare_common(an, f, raw_dev, dtype, pre, background_dev);
}

int32_t piv_frame_prepare(PivAnalyzer* an, PivFrame* f, const void* raw, int32_t dtype, const PivPreprocessC* pre,
                          const float* background) {
    if (!an || !f || !raw) return fail(PIV_ERR_ARGUMENT, "null argument");
    const size_t es = dtype_size(dtype);
    if (!es) return fail(PIV_ERR_ARGUMENT, "unknown dtype %d", dtype);
    int st = use_device(an);
    if (st) return st;
    const size_t n = (size_t)f->H * (size_t)f->W;
    st = stage_raw(f, es * n);
    if (st) return st;
    CUDA_TRY(cudaMemcpyAsync(f->d_raw, raw, es * n, cudaMemcpyHostToDevice, an->cur));
    const float* bg = nullptr;
    if (background) {
        if (!f->d_bg) CUDA_TRY(cudaMalloc(&f->d_bg, sizeof(float) * n));
        CUDA_TRY(cudaMemcpyAsync(f->d_bg, background, sizeof(float) * n, cudaMemcpyHostToDevice, an->cur));
        bg = f->d_bg;
    }
    return prepare_common(an, f, f->d_raw, dtype, pre, bg);
}

int32_t piv_frame_set_prepared(PivAnalyzer* an, PivFrame* f, const float* image, const float* base) {
    if (!an || !f || !image) return fail(PIV_ERR_ARGUMENT, "null argument");
    int st = use_device(an);
    if (st) return st;
    const size_t n = (size_t)f->H * (size_t)f->W;
    CUDA_TRY(cudaMemcpyAsync(f->image, image, sizeof(float) * n, cudaMemcpyHostToDevice, an->cur));
    f->nonneg = false;  // unknown: statistics are always built
    st = alloc_stats(f);
    if (st) return st;
    const float* bsrc = f->image;
    if (base) {
        if (!f->base_store) CUDA_TRY(cudaMalloc(&f->base_store, sizeof(float) * n));
        CUDA_TRY(cudaMemcpyAsync(f->base_store, base, sizeof(float) * n, cudaMemcpyHostToDevice, an->cur));
        bsrc = f->base_store;
    }
    f->base = const_cast<float*>(bsrc);
    int nl = 0;
    CUDA_TRY(launch_stats(bsrc, (int)f->H, (int)f->W, f->sum, f->sumsq, f->scales, f->words, an->cur, &nl));
    an->launches += nl;
    f->stats_valid = true;
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    return PIV_OK;
}

int32_t piv_frame_set_prepared_tables(PivAnalyzer* an, PivFrame* f, const float* image, const double* sum,
                                      const double* sumsq) {
    if (!an || !f || !image || !sum || !sumsq) return fail(PIV_ERR_ARGUMENT, "null argument");
    if (!f->words) return fail(PIV_ERR_ARGUMENT, "frame has no scratch");
    int st = use_device(an);
    if (st) return st;
    const size_t n = (size_t)f->H * (size_t)f->W;
    const size_t cells = (size_t)(f->H + 1) * (size_t)(f->W + 1);
    CUDA_TRY(cudaMemcpyAsync(f->image, image, sizeof(float) * n, cudaMemcpyHostToDevice, an->cur));
    f->nonneg = false;  // unknown: statistics are always used
    st = alloc_stats(f);
    if (st) return st;
    // the f64 tables land in the int64 tables' storage (8 bytes per entry) and are converted there
    static_assert(sizeof(double) == sizeof(long long), "8-byte entries");
    CUDA_TRY(cudaMemcpyAsync(f->sum, sum, sizeof(double) * cells, cudaMemcpyHostToDevice, an->cur));
    CUDA_TRY(cudaMemcpyAsync(f->sumsq, sumsq, sizeof(double) * cells, cudaMemcpyHostToDevice, an->cur));
    unsigned long long* maxbits2 = reinterpret_cast<unsigned long long*>(f->words);  // words[0..3]
    unsigned int* nonfinite = f->words + 4;
    int nl = 0;
    CUDA_TRY(launch_tables_to_fixed(f->sum, f->sumsq, (int)f->H, (int)f->W, f->scales, maxbits2, nonfinite, an->cur,
                                    &nl));
    an->launches += nl;
    unsigned int bad = 0;
    CUDA_TRY(cudaMemcpyAsync(&bad, nonfinite, sizeof(bad), cudaMemcpyDeviceToHost, an->cur));
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    f->base = f->image;  // the tables stand for the base image, which is not needed itself
    if (bad) {
        f->stats_valid = false;
        return fail(PIV_ERR_ARGUMENT, "the integral tables hold a non-finite entry");
    }
    f->stats_valid = true;
    return PIV_OK;
}

int32_t piv_frame_download(PivAnalyzer* an, const PivFrame* f, float* image) {
    if (!an || !f || !image) return fail(PIV_ERR_ARGUMENT, "null argument");
    int st = use_device(an);
    if (st) return st;
    CUDA_TRY(cudaMemcpyAsync(image, f->image, sizeof(float) * f->H * f->W, cudaMemcpyDeviceToHost, an->cur));
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    return PIV_OK;
}

const float* piv_frame_image_device(const PivFrame* f) { return f ? f->image : nullptr; }

int32_t piv_background_device(PivAnalyzer* an, const void* frames_dev, int32_t dtype, int64_t count, int64_t height,
                              int64_t width, int32_t mode, float* out_dev) {
    if (!an || !frames_dev || !out_dev || count <= 0) return fail(PIV_ERR_ARGUMENT, "bad argument");
    if (!dtype_size(dtype)) return fail(PIV_ERR_ARGUMENT, "unknown dtype %d", dtype);
    int st = use_device(an);
    if (st) return st;
    const long long npix = (long long)height * width;
    background_kernel<<<(int)std::min<long long>((npix + 255) / 256, 148 * 16), 256, 0, an->cur>>>(
        frames_dev, dtype, count, npix, mode, out_dev);
    CUDA_TRY(cudaGetLastError());
    an->launches += 1;
    return PIV_OK;
}

int32_t piv_analyze_device(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, float* dx, float* dy,
                           float* peak_ratio, uint8_t* flags, uint64_t* summary_dev) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    int st = run_passes(an, a, b);
    if (st) return st;
    const PassBuf& last = an->pairs[0].back();
    const size_t c = (size_t)last.cells;
    if (dx) CUDA_TRY(cudaMemcpyAsync(dx, last.dx, 4 * c, cudaMemcpyDeviceToDevice, an->cur));
    if (dy) CUDA_TRY(cudaMemcpyAsync(dy, last.dy, 4 * c, cudaMemcpyDeviceToDevice, an->cur));
    if (peak_ratio) CUDA_TRY(cudaMemcpyAsync(peak_ratio, last.raw_ppr, 4 * c, cudaMemcpyDeviceToDevice, an->cur));
    if (flags) CUDA_TRY(cudaMemcpyAsync(flags, last.flags, c, cudaMemcpyDeviceToDevice, an->cur));
    if (summary_dev)
        CUDA_TRY(cudaMemcpyAsync(summary_dev, an->d_counts, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, an->cur));
    return PIV_OK;
}

int32_t piv_analyze(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, float* dx, float* dy, float* peak_ratio,
                    uint8_t* flags, PivSummaryC* summary) {
    if (!an) return fail(PIV_ERR_ARGUMENT, "null analyzer");
    int st = run_passes(an, a, b);
    if (st) return st;
    const PassBuf& last = an->pairs[0].back();
    const size_t c = (size_t)last.cells;
    if (dx) CUDA_TRY(cudaMemcpyAsync(dx, last.dx, 4 * c, cudaMemcpyDeviceToHost, an->cur));
    if (dy) CUDA_TRY(cudaMemcpyAsync(dy, last.dy, 4 * c, cudaMemcpyDeviceToHost, an->cur));
    if (peak_ratio) CUDA_TRY(cudaMemcpyAsync(peak_ratio, last.raw_ppr, 4 * c, cudaMemcpyDeviceToHost, an->cur));
    if (flags) CUDA_TRY(cudaMemcpyAsync(flags, last.flags, c, cudaMemcpyDeviceToHost, an->cur));
    st = copy_summary(an, summary);
    if (st) return st;
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    return check_device_error(an->device);
}

int32_t piv_analyze_traced(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, PivTraceC* tr, PivSummaryC* summary) {
    if (!an || !tr) return fail(PIV_ERR_ARGUMENT, "null argument");
    int st = run_passes(an, a, b);
    if (st) return st;
    size_t off = 0;
    for (const PassBuf& pb : an->pairs[0]) {
        const size_t c = (size_t)pb.cells;
        auto d2h = [&](void* dst, const void* src, size_t es) -> cudaError_t {
            if (!dst) return cudaSuccess;
            return cudaMemcpyAsync((char*)dst + off * es, src, es * c, cudaMemcpyDeviceToHost, an->cur);
        };
        if (tr->origins) CUDA_TRY(cudaMemcpyAsync(tr->origins + 4 * off, pb.origins, 16 * c, cudaMemcpyDeviceToHost, an->cur));
        CUDA_TRY(d2h(tr->raw_dx, pb.raw_dx, 4));
        CUDA_TRY(d2h(tr->raw_dy, pb.raw_dy, 4));
        CUDA_TRY(d2h(tr->raw_peak_ratio, pb.raw_ppr, 4));
        CUDA_TRY(d2h(tr->raw_flags, pb.raw_flags, 1));
        CUDA_TRY(d2h(tr->dx, pb.dx, 4));
        CUDA_TRY(d2h(tr->dy, pb.dy, 4));
        CUDA_TRY(d2h(tr->peak_ratio, pb.raw_ppr, 4));
        CUDA_TRY(d2h(tr->flags, pb.flags, 1));
        off += c;
    }
    st = copy_summary(an, summary);
    if (st) return st;
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    return PIV_OK;
}

namespace {

int place_windows(PivAnalyzer* an, int64_t height, int64_t width, const PivGridC* grid, const PivGridC* pred_grid,
                  const float* pred_dx, const float* pred_dy, float* origins, float* corners) {
    if (!an || !grid || !origins) return fail(PIV_ERR_ARGUMENT, "null argument");
    if (grid->nx <= 0 || grid->ny <= 0 || grid->window <= 0 || grid->step <= 0)
        return fail(PIV_ERR_ARGUMENT, "empty grid");
    if (pred_grid && (pred_grid->nx <= 0 || pred_grid->ny <= 0 || pred_grid->step <= 0))
        return fail(PIV_ERR_ARGUMENT, "empty predictor grid");
    int st = use_device(an);
    if (st) return st;
    const size_t c = (size_t)(grid->nx * grid->ny);
    const size_t pc = pred_grid ? (size_t)(pred_grid->nx * pred_grid->ny) : 0;
    void* buf = nullptr;
    CUDA_TRY(cudaMalloc(&buf, align256(16 * c) + align256(c) + 2 * align256(4 * pc + 4) + align256(32 * c)));
    char* p = (char*)buf;
    float4* d_org = (float4*)p;
    p += align256(16 * c);
    uint8_t* d_st = (uint8_t*)p;
    p += align256(c);
    float* d_pdx = (float*)p;
    p += align256(4 * pc + 4);
    float* d_pdy = (float*)p;
    p += align256(4 * pc + 4);
    float4* d_corners = (float4*)p;
    PlaceParams pp{};
    pp.grid = to_gp(*grid);
    pp.H = (int)height;
    pp.W = (int)width;
    pp.has_pred = pred_grid && pred_dx && pred_dy;
    cudaError_t e = cudaSuccess;
    if (pp.has_pred) {
        pp.pgrid = to_gp(*pred_grid);
        e = cudaMemcpyAsync(d_pdx, pred_dx, 4 * pc, cudaMemcpyHostToDevice, an->cur);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_pdy, pred_dy, 4 * pc, cudaMemcpyHostToDevice, an->cur);
        pp.pdx = d_pdx;
        pp.pdy = d_pdy;
    }
    pp.origins = d_org;
    pp.status = d_st;
    pp.corners = corners ? d_corners : nullptr;
    pp.use_stats = 0;
    if (e == cudaSuccess) e = launch_place(pp, an->cur);
    an->launches += 1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(origins, d_org, 16 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && corners) e = cudaMemcpyAsync(corners, d_corners, 32 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess) e = cudaStreamSynchronize(an->cur);
    cudaFree(buf);
    if (e != cudaSuccess) return fail(PIV_ERR_CUDA, "place: %s", cudaGetErrorString(e));
    return PIV_OK;
}

}  // namespace

int32_t piv_place_windows(PivAnalyzer* an, int64_t height, int64_t width, const PivGridC* grid,
                          const PivGridC* pred_grid, const float* pred_dx, const float* pred_dy, float* origins) {
    return place_windows(an, height, width, grid, pred_grid, pred_dx, pred_dy, origins, nullptr);
}

int32_t piv_place_windows_deform(PivAnalyzer* an, int64_t height, int64_t width, const PivGridC* grid,
                                 const PivGridC* pred_grid, const float* pred_dx, const float* pred_dy, float* origins,
                                 float* corners) {
    if (!corners) return fail(PIV_ERR_ARGUMENT, "null corners");
    return place_windows(an, height, width, grid, pred_grid, pred_dx, pred_dy, origins, corners);
}

int32_t piv_correlate_origins(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, int64_t window,
                              const float* origins, int64_t ncells, float* dx, float* dy, float* peak_ratio,
                              uint8_t* flags) {
    if (!an || !a || !b || !origins || ncells < 0) return fail(PIV_ERR_ARGUMENT, "bad argument");
    if (a->H != b->H || a->W != b->W) return fail(PIV_ERR_SHAPE_MISMATCH, "frames have different shapes");
    if (!corr_supported((int)window)) return fail(PIV_ERR_UNSUPPORTED, "window size %lld", (long long)window);
    if (window > a->W || window > a->H) return fail(PIV_ERR_IMAGE_TOO_SMALL, "window larger than image");
    // Host-side bounds check of the origins (the kernel also clamps every index).
    for (int64_t k = 0; k < ncells; ++k)
        for (int j = 0; j < 4; ++j) {
            const float v = origins[4 * k + j];
            const float lim = (float)((j % 2 == 0 ? a->W : a->H) - window);
            if (!(v >= 0.0f && v <= lim)) return fail(PIV_ERR_ARGUMENT, "origin %lld out of the image", (long long)k);
        }
    int st = use_device(an);
    if (st) return st;
    const bool use_stats = needs_stats(an, a) || needs_stats(an, b);
    if (use_stats && !(a->stats_valid && b->stats_valid)) return fail(PIV_ERR_ARGUMENT, "frame statistics missing");
    const size_t c = (size_t)ncells;
    void* buf = nullptr;
    CUDA_TRY(cudaMalloc(&buf, align256(16 * c) + align256(c) + 3 * align256(4 * c) + align256(c) + 256));
    char* p = (char*)buf;
    float4* d_org = (float4*)p;
    p += align256(16 * c);
    uint8_t* d_st = (uint8_t*)p;
    p += align256(c);
    float* d_dx = (float*)p;
    p += align256(4 * c);
    float* d_dy = (float*)p;
    p += align256(4 * c);
    float* d_ppr = (float*)p;
    p += align256(4 * c);
    uint8_t* d_fl = (uint8_t*)p;
    cudaError_t e = cudaMemcpyAsync(d_org, origins, 16 * c, cudaMemcpyHostToDevice, an->cur);
    PlaceParams pp{};
    pp.grid.window = (int)window;
    pp.H = (int)a->H;
    pp.W = (int)a->W;
    pp.status = d_st;
    pp.use_stats = use_stats;
    if (use_stats) {
        pp.sa = stats_of(a);
        pp.sb = stats_of(b);
    }
    pp.min_mean = an->min_mean;
    pp.min_std = an->min_std;
    if (e == cudaSuccess) e = launch_mask(pp, d_org, (int)ncells, an->cur);
    CorrParams cp{a->image, b->image, (int)a->H, (int)a->W, d_org, d_st, (int)ncells, d_dx, d_dy, d_ppr, d_fl};
    if (e == cudaSuccess)
        e = (split_precision(an->precision) && corr_tc_supported((int)window))
                ? launch_correlate_tc_items((int)window, an->precision == PIV_PRECISION_FP16X3, &cp, 1, an->cur, nullptr)
                : launch_correlate((int)window, cp, an->cur);
    an->launches += 2;
    if (e == cudaSuccess && dx) e = cudaMemcpyAsync(dx, d_dx, 4 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && dy) e = cudaMemcpyAsync(dy, d_dy, 4 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && peak_ratio) e = cudaMemcpyAsync(peak_ratio, d_ppr, 4 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && flags) e = cudaMemcpyAsync(flags, d_fl, c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess) e = cudaStreamSynchronize(an->cur);
    cudaFree(buf);
    if (e != cudaSuccess) return fail(PIV_ERR_CUDA, "correlate: %s", cudaGetErrorString(e));
    return check_device_error(an->device);
}

int32_t piv_correlate_deform(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, const PivGridC* grid,
                             const float* origins, const float* corners, float* dx, float* dy, float* peak_ratio,
                             uint8_t* flags) {
    if (!an || !a || !b || !grid || !origins || !corners) return fail(PIV_ERR_ARGUMENT, "bad argument");
    if (a->H != b->H || a->W != b->W) return fail(PIV_ERR_SHAPE_MISMATCH, "frames have different shapes");
    const int64_t window = grid->window;
    if (!corr_supported((int)window)) return fail(PIV_ERR_UNSUPPORTED, "window size %lld", (long long)window);
    if (grid->nx <= 0 || grid->ny <= 0 || grid->step <= 0 || grid->x0 < 0 || grid->y0 < 0 ||
        grid->x0 + (grid->nx - 1) * grid->step + window > a->W || grid->y0 + (grid->ny - 1) * grid->step + window > a->H)
        return fail(PIV_ERR_ARGUMENT, "grid does not fit the image");
    const int64_t ncells = grid->nx * grid->ny;
    for (int64_t k = 0; k < ncells; ++k) {
        for (int j = 0; j < 4; ++j) {
            const float v = origins[4 * k + j];
            const float lim = (float)((j % 2 == 0 ? a->W : a->H) - window);
            if (!(v >= 0.0f && v <= lim)) return fail(PIV_ERR_ARGUMENT, "origin %lld out of the image", (long long)k);
        }
        for (int j = 0; j < 8; ++j)
            if (!std::isfinite(corners[8 * k + j])) return fail(PIV_ERR_ARGUMENT, "corner %lld not finite", (long long)k);
    }
    int st = use_device(an);
    if (st) return st;
    const bool use_stats = needs_stats(an, a) || needs_stats(an, b);
    if (use_stats && !(a->stats_valid && b->stats_valid)) return fail(PIV_ERR_ARGUMENT, "frame statistics missing");
    const size_t c = (size_t)ncells;
    void* buf = nullptr;
    CUDA_TRY(cudaMalloc(&buf, align256(16 * c) + align256(32 * c) + align256(c) + 3 * align256(4 * c) + align256(c) + 256));
    char* p = (char*)buf;
    float4* d_org = (float4*)p;
    p += align256(16 * c);
    float4* d_cor = (float4*)p;
    p += align256(32 * c);
    uint8_t* d_st = (uint8_t*)p;
    p += align256(c);
    float* d_dx = (float*)p;
    p += align256(4 * c);
    float* d_dy = (float*)p;
    p += align256(4 * c);
    float* d_ppr = (float*)p;
    p += align256(4 * c);
    uint8_t* d_fl = (uint8_t*)p;
    cudaError_t e = cudaMemcpyAsync(d_org, origins, 16 * c, cudaMemcpyHostToDevice, an->cur);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_cor, corners, 32 * c, cudaMemcpyHostToDevice, an->cur);
    PlaceParams pp{};
    pp.grid.window = (int)window;
    pp.H = (int)a->H;
    pp.W = (int)a->W;
    pp.status = d_st;
    pp.use_stats = use_stats;
    if (use_stats) {
        pp.sa = stats_of(a);
        pp.sb = stats_of(b);
    }
    pp.min_mean = an->min_mean;
    pp.min_std = an->min_std;
    if (e == cudaSuccess) e = launch_mask(pp, d_org, (int)ncells, an->cur);
    CorrParams cp{a->image, b->image, (int)a->H, (int)a->W, d_org, d_st, (int)ncells, d_dx, d_dy, d_ppr, d_fl,
                  d_cor, (int)grid->x0, (int)grid->y0, (int)grid->step, (int)grid->nx};
    if (e == cudaSuccess) e = launch_correlate_items((int)window, an->variant[1][window], &cp, 1, an->cur, nullptr);
    an->launches += 2;
    if (e == cudaSuccess && dx) e = cudaMemcpyAsync(dx, d_dx, 4 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && dy) e = cudaMemcpyAsync(dy, d_dy, 4 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && peak_ratio) e = cudaMemcpyAsync(peak_ratio, d_ppr, 4 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && flags) e = cudaMemcpyAsync(flags, d_fl, c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess) e = cudaStreamSynchronize(an->cur);
    cudaFree(buf);
    if (e != cudaSuccess) return fail(PIV_ERR_CUDA, "correlate: %s", cudaGetErrorString(e));
    return PIV_OK;
}

int32_t piv_flow_stats_device(int64_t ny, int64_t nx, int64_t step, double dt_s, const float* dx, const float* dy,
                              const uint8_t* flags, float* vorticity, PivFlowStatsC* stats, void* stream) {
    if (!dx || !dy || !flags || !stats) return fail(PIV_ERR_ARGUMENT, "null pointer");
    if (ny <= 0 || nx <= 0 || ny * nx > 0x7fffffffll) return fail(PIV_ERR_ARGUMENT, "bad field shape");
    if (step <= 0 || !(dt_s > 0.0)) return fail(PIV_ERR_ARGUMENT, "step and dt_s must be positive");
    FlowStatsHost h{};
    CUDA_TRY(flow_stats_device((int)ny, (int)nx, (float)step, dt_s, dx, dy, flags, vorticity, &h, (cudaStream_t)stream));
    stats->vorticity_mean = h.vorticity_mean;
    stats->vorticity_abs_mean = h.vorticity_abs_mean;
    stats->ke_mean = h.ke_mean;
    stats->ke_sum = h.ke_sum;
    stats->coverage = h.coverage;
    stats->n_usable = h.n_usable;
    stats->n_vorticity = h.n_vorticity;
    return PIV_OK;
}

int32_t piv_temporal_smooth_device(int64_t nt, int64_t ny, int64_t nx, const float* dx, const float* dy,
                                   const uint8_t* usable, const uint8_t* gate, int32_t median, int32_t window,
                                   int32_t min_support, const int32_t* leave_out, int32_t n_leave_out, float* out_dx,
                                   float* out_dy, uint16_t* support, void* stream) {
    if (!dx || !dy || !usable || !gate || !out_dx || !out_dy || !support) return fail(PIV_ERR_ARGUMENT, "null pointer");
    if (nt <= 0 || ny <= 0 || nx <= 0 || nt * ny * nx > 0x7fffffffll) return fail(PIV_ERR_ARGUMENT, "bad shape");
    if (window < 1 || window % 2 == 0 || window > 63) return fail(PIV_ERR_ARGUMENT, "window must be odd, 1..63");
    if (n_leave_out < 0 || (n_leave_out > 0 && !leave_out)) return fail(PIV_ERR_ARGUMENT, "bad leave_out list");
    // smooth.rs:59-73: the offsets, centre first, then each side outwards skipping left-out ones
    std::vector<int> off;
    auto left = [&](int o) {
        for (int i = 0; i < n_leave_out; ++i)
            if (leave_out[i] == o) return true;
        return false;
    };
    if (!left(0)) off.push_back(0);
    for (int sign : {-1, 1}) {
        int k = 1, taken = 0;
        while (taken < window / 2) {
            if (!left(sign * k)) {
                off.push_back(sign * k);
                ++taken;
            }
            ++k;
        }
    }
    CUDA_TRY(temporal_smooth_device((int)nt, (int)ny, (int)nx, dx, dy, usable, gate, median != 0, off.data(),
                                    (int)off.size(), min_support, out_dx, out_dy, support, (cudaStream_t)stream));
    return PIV_OK;
}

int32_t piv_spatial_smooth_device(int64_t nt, int64_t ny, int64_t nx, const float* dx, const float* dy,
                                  const uint8_t* gate, float sigma, float min_weight, int32_t leave_out, float* out_dx,
                                  float* out_dy, uint16_t* support, void* stream) {
    if (!dx || !dy || !gate || !out_dx || !out_dy || !support) return fail(PIV_ERR_ARGUMENT, "null pointer");
    if (nt <= 0 || ny <= 0 || nx <= 0 || nt * ny * nx > 0x7fffffffll) return fail(PIV_ERR_ARGUMENT, "bad shape");
    if (!(sigma > 0.0f && sigma <= 12.0f)) return fail(PIV_ERR_ARGUMENT, "sigma must be in (0, 12]");
    CUDA_TRY(spatial_smooth_device((int)nt, (int)ny, (int)nx, dx, dy, gate, sigma, min_weight, leave_out, out_dx, out_dy,
                                   support, (cudaStream_t)stream));
    return PIV_OK;
}

int32_t piv_tc_selftest(int32_t device, int32_t a_mn, int32_t n, int32_t k, const float* a, const float* b, float* d) {
    if (!a || !b || !d) return fail(PIV_ERR_ARGUMENT, "null pointer");
    if (n < 16 || n > 256 || n % 16 || k < 16 || k > 256 || k % 16)
        return fail(PIV_ERR_ARGUMENT, "n and k must be multiples of 16 in [16, 256]");
    int dev = device;
    if (dev < 0) CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaSetDevice(dev));
    int st = ensure_device_init(dev);
    if (st) return st;
    CUDA_TRY(tc_selftest(a_mn != 0, n, k, a, b, d));
    CUDA_TRY(cudaDeviceSynchronize());
    return check_device_error(dev);
}

int32_t piv_tc_wait_probe(int32_t device, int32_t log2_iters, int32_t* timed_out, float* ms) {
    if (!timed_out || !ms) return fail(PIV_ERR_ARGUMENT, "null pointer");
    if (log2_iters < 0 || log2_iters > 18) return fail(PIV_ERR_ARGUMENT, "log2_iters must be in [0, 18]");
    int dev = device;
    if (dev < 0) CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaSetDevice(dev));
    unsigned int t = 0;
    CUDA_TRY(tc_wait_probe(log2_iters, &t, ms));
    *timed_out = t != 0;
    return PIV_OK;
}

int32_t piv_validate_field(PivAnalyzer* an, int64_t ny, int64_t nx, const float* dx, const float* dy,
                           const float* peak_ratio, const uint8_t* flags, float* out_dx, float* out_dy,
                           uint8_t* out_flags, PivSummaryC* summary) {
    if (!an || !dx || !dy || !peak_ratio || !flags) return fail(PIV_ERR_ARGUMENT, "null argument");
    if (ny <= 0 || nx <= 0) return fail(PIV_ERR_ARGUMENT, "empty field");
    int st = use_device(an);
    if (st) return st;
    const size_t c = (size_t)(ny * nx);
    void* buf = nullptr;
    CUDA_TRY(cudaMalloc(&buf, 5 * align256(4 * c) + 4 * align256(c) + 256));
    char* p = (char*)buf;
    auto take = [&](size_t bytes) {
        void* r = p;
        p += align256(bytes);
        return r;
    };
    float* d_dx = (float*)take(4 * c);
    float* d_dy = (float*)take(4 * c);
    float* d_ppr = (float*)take(4 * c);
    float* o_dx = (float*)take(4 * c);
    float* o_dy = (float*)take(4 * c);
    uint8_t* f0 = (uint8_t*)take(c);
    uint8_t* f1 = (uint8_t*)take(c);
    uint8_t* f2 = (uint8_t*)take(c);
    uint8_t* fo = (uint8_t*)take(c);
    unsigned long long* cnt = (unsigned long long*)take(64);
    cudaError_t e = cudaMemcpyAsync(d_dx, dx, 4 * c, cudaMemcpyHostToDevice, an->cur);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_dy, dy, 4 * c, cudaMemcpyHostToDevice, an->cur);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ppr, peak_ratio, 4 * c, cudaMemcpyHostToDevice, an->cur);
    if (e == cudaSuccess) e = cudaMemcpyAsync(f0, flags, c, cudaMemcpyHostToDevice, an->cur);
    ValidateParams vp{(int)nx, (int)ny, d_dx, d_dy, d_ppr, f0, f1, f2, o_dx, o_dy, fo, (float)an->windows[0] / 2.0f,
                      an->ppr_threshold, an->median_threshold, an->median_eps, an->replace};
    if (e == cudaSuccess) e = launch_validate(vp, an->cur);
    if (e == cudaSuccess) e = launch_summary(fo, (int)c, cnt, an->cur);
    an->launches += kValidateLaunches + kSummaryLaunches;
    unsigned long long hc[5] = {0, 0, 0, 0, 0};
    if (e == cudaSuccess && out_dx) e = cudaMemcpyAsync(out_dx, o_dx, 4 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && out_dy) e = cudaMemcpyAsync(out_dy, o_dy, 4 * c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess && out_flags) e = cudaMemcpyAsync(out_flags, fo, c, cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, an->cur);
    if (e == cudaSuccess) e = cudaStreamSynchronize(an->cur);
    cudaFree(buf);
    if (e != cudaSuccess) return fail(PIV_ERR_CUDA, "validate: %s", cudaGetErrorString(e));
    if (summary) {
        summary->no_signal = (int64_t)hc[0];
        summary->low_ppr = (int64_t)hc[1];
        summary->median_outliers = (int64_t)hc[2];
        summary->out_of_range = (int64_t)hc[3];
        summary->replaced = (int64_t)hc[4];
    }
    return PIV_OK;
}

int32_t piv_analyze_batch_device(PivAnalyzer* an, const PivFrame* const* a, const PivFrame* const* b, int32_t count,
                                 float* dx, float* dy, float* peak_ratio, uint8_t* flags, uint64_t* summaries_dev) {
    if (!an || !a || !b) return fail(PIV_ERR_ARGUMENT, "null argument");
    int st = run_passes(an, a, b, count);
    if (st) return st;
    for (int k = 0; k < count; ++k) {
        const PassBuf& last = an->pairs[k].back();
        const size_t c = (size_t)last.cells;
        if (dx) CUDA_TRY(cudaMemcpyAsync(dx + k * c, last.dx, 4 * c, cudaMemcpyDeviceToDevice, an->cur));
        if (dy) CUDA_TRY(cudaMemcpyAsync(dy + k * c, last.dy, 4 * c, cudaMemcpyDeviceToDevice, an->cur));
        if (peak_ratio) CUDA_TRY(cudaMemcpyAsync(peak_ratio + k * c, last.raw_ppr, 4 * c, cudaMemcpyDeviceToDevice, an->cur));
        if (flags) CUDA_TRY(cudaMemcpyAsync(flags + k * c, last.flags, c, cudaMemcpyDeviceToDevice, an->cur));
    }
    if (summaries_dev)
        CUDA_TRY(cudaMemcpyAsync(summaries_dev, an->d_counts, 8 * sizeof(unsigned long long) * (size_t)count,
                                 cudaMemcpyDeviceToDevice, an->cur));
    return PIV_OK;
}

namespace {

// One run of a batch: prepare every frame from the slab, all passes of all pairs, outputs.
int batch_record(PivBatch* bt) {
    PivAnalyzer* an = bt->an;
    const int nf = (int)bt->frames.size();
    for (int i = 0; i < nf; ++i) {
        int st = prepare_common(an, bt->frames[i], (const char*)bt->raw + (size_t)i * bt->frame_bytes, bt->dtype, &bt->pre,
                                bt->background);
        if (st) return st;
    }
    std::vector<const PivFrame*> fa(bt->K), fb(bt->K);
    for (int k = 0; k < bt->K; ++k) {
        fa[k] = bt->sequential ? bt->frames[k] : bt->frames[2 * k];
        fb[k] = bt->sequential ? bt->frames[k + 1] : bt->frames[2 * k + 1];
    }
    return piv_analyze_batch_device(an, fa.data(), fb.data(), bt->K, bt->dx, bt->dy, bt->ppr, bt->flags,
                                    (uint64_t*)bt->sums);
}

}  // namespace

namespace {
// A private analyzer with the parent's configuration and chosen launch variants (no workspace,
// no stream yet): its workspace is never resized by the parent's calls.
PivAnalyzer* clone_config(const PivAnalyzer* parent) {
    PivAnalyzer* an = new PivAnalyzer();
    an->windows = parent->windows;
    an->overlap = parent->overlap;
    an->final_iterations = parent->final_iterations;
    an->min_mean = parent->min_mean;
    an->min_std = parent->min_std;
    an->ppr_threshold = parent->ppr_threshold;
    an->median_threshold = parent->median_threshold;
    an->median_eps = parent->median_eps;
    an->replace = parent->replace;
    an->deform = parent->deform;
    an->precision = parent->precision;
    an->device = parent->device;
    for (int k = 0; k < 2; ++k)
        for (int i = 0; i < 129; ++i) an->variant[k][i] = parent->variant[k][i];
    for (int k = 0; k < 2; ++k)
        for (int i = 0; i < 129; ++i) an->fp32_faster[k][i] = parent->fp32_faster[k][i];
    return an;
}
}  // namespace

int32_t piv_batch_create(const PivAnalyzer* parent, int64_t height, int64_t width, int32_t pairs, int32_t sequential,
                         int32_t dtype, const PivPreprocessC* pre, PivBatch** out) {
    if (!parent || !out || pairs <= 0) return fail(PIV_ERR_ARGUMENT, "bad argument");
    *out = nullptr;
    const size_t es = dtype_size(dtype);
    if (!es) return fail(PIV_ERR_ARGUMENT, "unknown dtype %d", dtype);
    PivGridC g;
    int st = make_grid(height, width, parent->windows.back(), parent->overlap, &g);
    if (st) return st;
    for (int32_t n : parent->windows) {
        st = make_grid(height, width, n, parent->overlap, &g);
        if (st) return st;
    }
    make_grid(height, width, parent->windows.back(), parent->overlap, &g);
    CUDA_TRY(cudaSetDevice(parent->device));
    PivBatch* bt = new PivBatch();
    PivAnalyzer* an = clone_config(parent);
    bt->an = an;
    bt->H = height;
    bt->W = width;
    bt->K = pairs;
    bt->sequential = sequential != 0;
    bt->dtype = dtype;
    bt->pre = pre ? *pre : PivPreprocessC{1.0f, 4, 0.02f, 0.0};
    bt->frame_bytes = es * (size_t)height * (size_t)width;
    bt->cells = g.nx * g.ny;
    const int nf = bt->sequential ? pairs + 1 : 2 * pairs;
    const size_t c = (size_t)bt->cells * (size_t)pairs;
    cudaError_t e = cudaStreamCreateWithFlags(&an->own, cudaStreamNonBlocking);
    an->cur = an->own;
    if (e == cudaSuccess) e = cudaMalloc(&bt->raw, bt->frame_bytes * (size_t)nf);
    if (e == cudaSuccess)
        e = cudaMalloc(&bt->out, align256(4 * c) * 3 + align256(c) + align256(8 * sizeof(unsigned long long) * pairs));
    if (e != cudaSuccess) {
        piv_batch_destroy(bt);
        return fail(PIV_ERR_CUDA, "batch allocation: %s", cudaGetErrorString(e));
    }
    char* p = (char*)bt->out;
    bt->dx = (float*)p;
    p += align256(4 * c);
    bt->dy = (float*)p;
    p += align256(4 * c);
    bt->ppr = (float*)p;
    p += align256(4 * c);
    bt->flags = (uint8_t*)p;
    p += align256(c);
    bt->sums = (unsigned long long*)p;
    for (int i = 0; i < nf; ++i) {
        PivFrame* f = nullptr;
        st = piv_frame_create(an, height, width, &f);
        if (st) {
            piv_batch_destroy(bt);
            return st;
        }
        bt->frames.push_back(f);
    }
    *out = bt;
    return PIV_OK;
}

void piv_batch_destroy(PivBatch* bt) {
    if (!bt) return;
    if (bt->an) {
        cudaSetDevice(bt->an->device);
        // The batch's kernels may run on a stream it borrowed (piv_batch_set_stream), which may
        // already be gone; waiting for the device needs no stream handle.
        cudaDeviceSynchronize();
        bt->an->cur = bt->an->own;
    }
    for (cudaStream_t st : {bt->up, bt->down})
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    for (cudaEvent_t ev : {bt->uploaded, bt->computed, bt->hdone})
        if (ev) cudaEventDestroy(ev);
    if (bt->hsums) cudaFreeHost(bt->hsums);
    for (PivFrame* f : bt->frames) piv_frame_destroy(f);
    cudaFree(bt->raw);
    cudaFree(bt->out);
    piv_analyzer_destroy(bt->an);
    delete bt;
}

// ---------------------------------------------------------------------------------------------
// Pipelined pairs: `depth` slots, each a private analyzer (workspace) with its own frames, and
// three streams shared by the slots. A submitted pair's uploads go on the upload stream, its
// preparation and passes on the compute stream (after the uploads), its downloads on the
// download stream (after the passes). The copies of one pair overlap the kernels of the others,
// while the kernels of different pairs run one after another as in a single analyzer, so they
// never compete for the SMs. A slot is reused only after its previous pair fully completed.
// ---------------------------------------------------------------------------------------------
struct PivPipeline {
    struct Slot {
        PivAnalyzer* an = nullptr;
        PivFrame* fa = nullptr;
        PivFrame* fb = nullptr;
        unsigned long long* sums = nullptr;  // pinned: 5 counters of the slot's last pair
        cudaEvent_t uploaded = nullptr;       // on the upload stream
        cudaEvent_t prepared = nullptr;       // on the preparation stream
        cudaEvent_t computed = nullptr;       // on the compute stream
        cudaEvent_t done = nullptr;           // on the download stream
        uint64_t ticket = 0;  // 0: idle
    };
    // Preparation has its own stream so that a pair's frames are prepared while the previous pair
    // is analysed (the slots' frames and workspaces are separate, and a slot is reused only after
    // its previous pair has been waited for).
    cudaStream_t up = nullptr, prep = nullptr, comp = nullptr, down = nullptr;
    const float* background = nullptr;  // device image subtracted from every frame (caller-owned)
    int device = 0;
    int64_t H = 0, W = 0;
    int32_t dtype = PIV_DTYPE_U16;
    PivPreprocessC pre{};
    std::vector<Slot> slots;
    size_t next = 0;
    uint64_t tickets = 0;
    std::map<uint64_t, PivSummaryC> finished;  // pairs whose slot was reused before their wait
};

namespace {
int retire_slot(PivPipeline* pl, PivPipeline::Slot& s, PivSummaryC* out) {
    CUDA_TRY(cudaEventSynchronize(s.done));
    int st = check_device_error(pl->device);
    if (st) return st;
    PivSummaryC r{(int64_t)s.sums[0], (int64_t)s.sums[1], (int64_t)s.sums[2], (int64_t)s.sums[3], (int64_t)s.sums[4]};
    if (out) *out = r;
    else pl->finished[s.ticket] = r;
    s.ticket = 0;
    return PIV_OK;
}
}  // namespace

int32_t piv_pipeline_create(const PivAnalyzer* parent, int64_t height, int64_t width, int32_t dtype,
                            const PivPreprocessC* pre, int32_t depth, PivPipeline** out) {
    if (!parent || !out) return fail(PIV_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    if (depth < 1 || depth > 8) return fail(PIV_ERR_ARGUMENT, "depth must be in [1, 8]");
    if (!dtype_size(dtype)) return fail(PIV_ERR_ARGUMENT, "unknown dtype %d", dtype);
    PivGridC g;
    for (int32_t n : parent->windows) {
        int st = make_grid(height, width, n, parent->overlap, &g);
        if (st) return st;
    }
    CUDA_TRY(cudaSetDevice(parent->device));
    PivPipeline* pl = new PivPipeline();
    pl->device = parent->device;
    pl->H = height;
    pl->W = width;
    pl->dtype = dtype;
    pl->pre = pre ? *pre : PivPreprocessC{1.0f, 4, 0.02f, 0.0};
    pl->slots.resize((size_t)depth);
    {
        cudaError_t e = cudaStreamCreateWithFlags(&pl->up, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&pl->prep, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&pl->comp, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&pl->down, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            piv_pipeline_destroy(pl);
            return fail(PIV_ERR_CUDA, "pipeline streams: %s", cudaGetErrorString(e));
        }
    }
    const size_t raw_bytes = dtype_size(dtype) * (size_t)height * (size_t)width;
    for (auto& s : pl->slots) {
        s.an = clone_config(parent);
        s.an->cur = pl->comp;
        cudaError_t e = cudaEventCreateWithFlags(&s.uploaded, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.prepared, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.computed, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaHostAlloc((void**)&s.sums, 8 * sizeof(unsigned long long), cudaHostAllocDefault);
        int st = e == cudaSuccess ? PIV_OK : fail(PIV_ERR_CUDA, "pipeline slot: %s", cudaGetErrorString(e));
        if (!st) st = piv_frame_create(s.an, height, width, &s.fa);
        if (!st) st = piv_frame_create(s.an, height, width, &s.fb);
        if (!st) st = stage_raw(s.fa, raw_bytes);
        if (!st) st = stage_raw(s.fb, raw_bytes);
        if (st) {
            piv_pipeline_destroy(pl);
            return st;
        }
    }
    *out = pl;
    return PIV_OK;
}

void piv_pipeline_destroy(PivPipeline* pl) {
    if (!pl) return;
    cudaSetDevice(pl->device);
    for (cudaStream_t st : {pl->up, pl->prep, pl->comp, pl->down})
        if (st) cudaStreamSynchronize(st);
    for (auto& s : pl->slots) {
        if (s.fa) piv_frame_destroy(s.fa);
        if (s.fb) piv_frame_destroy(s.fb);
        for (cudaEvent_t ev : {s.uploaded, s.prepared, s.computed, s.done})
            if (ev) cudaEventDestroy(ev);
        if (s.sums) cudaFreeHost(s.sums);
        piv_analyzer_destroy(s.an);
    }
    for (cudaStream_t st : {pl->up, pl->prep, pl->comp, pl->down})
        if (st) cudaStreamDestroy(st);
    delete pl;
}

int32_t piv_pipeline_submit(PivPipeline* pl, const void* frame_a, const void* frame_b, float* dx, float* dy,
                            float* peak_ratio, uint8_t* flags, uint64_t* ticket) {
    if (!pl || !frame_a || !frame_b || !ticket) return fail(PIV_ERR_ARGUMENT, "null argument");
    CUDA_TRY(cudaSetDevice(pl->device));
    PivPipeline::Slot& s = pl->slots[pl->next % pl->slots.size()];
    if (s.ticket) {
        int st = retire_slot(pl, s, nullptr);
        if (st) return st;
    }
    const size_t raw_bytes = dtype_size(pl->dtype) * (size_t)pl->H * (size_t)pl->W;
    CUDA_TRY(cudaMemcpyAsync(s.fa->d_raw, frame_a, raw_bytes, cudaMemcpyHostToDevice, pl->up));
    CUDA_TRY(cudaMemcpyAsync(s.fb->d_raw, frame_b, raw_bytes, cudaMemcpyHostToDevice, pl->up));
    CUDA_TRY(cudaEventRecord(s.uploaded, pl->up));
    CUDA_TRY(cudaStreamWaitEvent(pl->prep, s.uploaded, 0));
    s.an->cur = pl->prep;
    int st = prepare_common(s.an, s.fa, s.fa->d_raw, pl->dtype, &pl->pre, pl->background);
    if (!st) st = prepare_common(s.an, s.fb, s.fb->d_raw, pl->dtype, &pl->pre, pl->background);
    s.an->cur = pl->comp;
    if (st) return st;
    CUDA_TRY(cudaEventRecord(s.prepared, pl->prep));
    CUDA_TRY(cudaStreamWaitEvent(pl->comp, s.prepared, 0));
    st = run_passes(s.an, s.fa, s.fb);
    if (st) return st;
    CUDA_TRY(cudaEventRecord(s.computed, pl->comp));
    CUDA_TRY(cudaStreamWaitEvent(pl->down, s.computed, 0));
    const PassBuf& last = s.an->pairs[0].back();
    const size_t c = (size_t)last.cells;
    cudaStream_t cs = pl->down;
    if (dx) CUDA_TRY(cudaMemcpyAsync(dx, last.dx, 4 * c, cudaMemcpyDeviceToHost, cs));
    if (dy) CUDA_TRY(cudaMemcpyAsync(dy, last.dy, 4 * c, cudaMemcpyDeviceToHost, cs));
    if (peak_ratio) CUDA_TRY(cudaMemcpyAsync(peak_ratio, last.raw_ppr, 4 * c, cudaMemcpyDeviceToHost, cs));
    if (flags) CUDA_TRY(cudaMemcpyAsync(flags, last.flags, c, cudaMemcpyDeviceToHost, cs));
    CUDA_TRY(cudaMemcpyAsync(s.sums, s.an->d_counts, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, cs));
    CUDA_TRY(cudaEventRecord(s.done, cs));
    s.ticket = ++pl->tickets;
    pl->next++;
    *ticket = s.ticket;
    return PIV_OK;
}

int32_t piv_pipeline_set_background(PivPipeline* pl, const float* background_dev) {
    if (!pl) return fail(PIV_ERR_ARGUMENT, "null pipeline");
    for (const auto& s : pl->slots)
        if (s.ticket) return fail(PIV_ERR_ARGUMENT, "pairs are in flight: wait for them before changing the background");
    pl->background = background_dev;
    return PIV_OK;
}

int32_t piv_pipeline_wait(PivPipeline* pl, uint64_t ticket, PivSummaryC* summary) {
    if (!pl) return fail(PIV_ERR_ARGUMENT, "null pipeline");
    CUDA_TRY(cudaSetDevice(pl->device));
    auto it = pl->finished.find(ticket);
    if (it != pl->finished.end()) {
        if (summary) *summary = it->second;
        pl->finished.erase(it);
        return PIV_OK;
    }
    for (auto& s : pl->slots)
        if (s.ticket == ticket) {
            PivSummaryC r{};
            int st = retire_slot(pl, s, &r);
            if (st) return st;
            if (summary) *summary = r;
            return PIV_OK;
        }
    return fail(PIV_ERR_ARGUMENT, "unknown or already collected ticket %llu", (unsigned long long)ticket);
}

void* piv_batch_input_device(PivBatch* bt) { return bt ? bt->raw : nullptr; }

int64_t piv_batch_input_bytes(const PivBatch* bt) {
    return bt ? (int64_t)(bt->frame_bytes * bt->frames.size()) : 0;
}

int32_t piv_batch_run(PivBatch* bt) {
    if (!bt) return fail(PIV_ERR_ARGUMENT, "null batch");
    PivAnalyzer* an = bt->an;
    int st = use_device(an);
    if (st) return st;
    if (bt->exec) {
        CUDA_TRY(cudaGraphLaunch(bt->exec, an->cur));
        ++bt->runs;
        return PIV_OK;
    }
    // First run: eager (allocates the workspace and frame buffers), then capture the same work.
    const long long l0 = an->launches;
    st = batch_record(bt);
    if (st) return st;
    bt->kernels = an->launches - l0;
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    CUDA_TRY(cudaStreamBeginCapture(an->cur, cudaStreamCaptureModeRelaxed));
    st = batch_record(bt);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(an->cur, &graph);
    if (st) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (ce != cudaSuccess) return fail(PIV_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    bt->graph = graph;
    CUDA_TRY(cudaGraphInstantiate(&bt->exec, bt->graph, 0));
    ++bt->runs;
    return PIV_OK;
}

void* piv_batch_stream(PivBatch* bt) { return bt ? (void*)bt->an->cur : nullptr; }

int32_t piv_batch_set_background(PivBatch* bt, const float* background_dev) {
    if (!bt) return fail(PIV_ERR_ARGUMENT, "null batch");
    if (bt->pending) return fail(PIV_ERR_ARGUMENT, "the batch has a submission that has not been collected");
    if (background_dev == bt->background) return PIV_OK;
    CUDA_TRY(cudaSetDevice(bt->an->device));
    CUDA_TRY(cudaDeviceSynchronize());  // a replay may still read the old pointer
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    bt->exec = nullptr;  // the next run records the batch again with the new image
    bt->graph = nullptr;
    bt->background = background_dev;
    return PIV_OK;
}

int32_t piv_batch_set_stream(PivBatch* bt, void* stream) {
    if (!bt) return fail(PIV_ERR_ARGUMENT, "null batch");
    if (bt->pending) return fail(PIV_ERR_ARGUMENT, "the batch has a submission that has not been collected");
    bt->an->cur = stream ? (cudaStream_t)stream : bt->an->own;
    return PIV_OK;
}

int32_t piv_batch_sync(PivBatch* bt) {
    if (!bt) return fail(PIV_ERR_ARGUMENT, "null batch");
    CUDA_TRY(cudaSetDevice(bt->an->device));
    CUDA_TRY(cudaStreamSynchronize(bt->an->cur));
    return PIV_OK;
}

int32_t piv_batch_outputs_device(PivBatch* bt, float** dx, float** dy, float** peak_ratio, uint8_t** flags,
                                 uint64_t** summaries) {
    if (!bt) return fail(PIV_ERR_ARGUMENT, "null batch");
    if (dx) *dx = bt->dx;
    if (dy) *dy = bt->dy;
    if (peak_ratio) *peak_ratio = bt->ppr;
    if (flags) *flags = bt->flags;
    if (summaries) *summaries = (uint64_t*)bt->sums;
    return PIV_OK;
}

int32_t piv_batch_run_host(PivBatch* bt, const void* raw, float* dx, float* dy, float* peak_ratio, uint8_t* flags,
                           PivSummaryC* summaries) {
    if (!bt || !raw) return fail(PIV_ERR_ARGUMENT, "null argument");
    PivAnalyzer* an = bt->an;
    int st = use_device(an);
    if (st) return st;
    CUDA_TRY(cudaMemcpyAsync(bt->raw, raw, bt->frame_bytes * bt->frames.size(), cudaMemcpyHostToDevice, an->cur));
    st = piv_batch_run(bt);
    if (st) return st;
    const size_t c = (size_t)bt->cells * (size_t)bt->K;
    if (dx) CUDA_TRY(cudaMemcpyAsync(dx, bt->dx, 4 * c, cudaMemcpyDeviceToHost, an->cur));
    if (dy) CUDA_TRY(cudaMemcpyAsync(dy, bt->dy, 4 * c, cudaMemcpyDeviceToHost, an->cur));
    if (peak_ratio) CUDA_TRY(cudaMemcpyAsync(peak_ratio, bt->ppr, 4 * c, cudaMemcpyDeviceToHost, an->cur));
    if (flags) CUDA_TRY(cudaMemcpyAsync(flags, bt->flags, c, cudaMemcpyDeviceToHost, an->cur));
    std::vector<unsigned long long> hs;
    if (summaries) {
        hs.resize(8 * (size_t)bt->K);
        CUDA_TRY(cudaMemcpyAsync(hs.data(), bt->sums, sizeof(unsigned long long) * hs.size(), cudaMemcpyDeviceToHost,
                                 an->cur));
    }
    CUDA_TRY(cudaStreamSynchronize(an->cur));
    if (summaries)
        for (int k = 0; k < bt->K; ++k) {
            summaries[k].no_signal = (int64_t)hs[8 * k + 0];
            summaries[k].low_ppr = (int64_t)hs[8 * k + 1];
            summaries[k].median_outliers = (int64_t)hs[8 * k + 2];
            summaries[k].out_of_range = (int64_t)hs[8 * k + 3];
            summaries[k].replaced = (int64_t)hs[8 * k + 4];
        }
    return PIV_OK;
}

int32_t piv_batch_submit_host(PivBatch* bt, const void* raw, float* dx, float* dy, float* peak_ratio, uint8_t* flags) {
    if (!bt || !raw) return fail(PIV_ERR_ARGUMENT, "null argument");
    if (bt->pending) return fail(PIV_ERR_ARGUMENT, "the previous submission of this batch has not been collected");
    PivAnalyzer* an = bt->an;
    int st = use_device(an);
    if (st) return st;
    if (!bt->hsums) {
        CUDA_TRY(cudaHostAlloc((void**)&bt->hsums, sizeof(unsigned long long) * 8 * (size_t)bt->K, cudaHostAllocDefault));
        CUDA_TRY(cudaStreamCreateWithFlags(&bt->up, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&bt->down, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&bt->uploaded, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&bt->computed, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&bt->hdone, cudaEventDisableTiming));
    }
    // upload stream -> compute stream (graph replay) -> download stream; the previous submission
    // was collected, so the input slab and the outputs are free
    CUDA_TRY(cudaMemcpyAsync(bt->raw, raw, bt->frame_bytes * bt->frames.size(), cudaMemcpyHostToDevice, bt->up));
    CUDA_TRY(cudaEventRecord(bt->uploaded, bt->up));
    CUDA_TRY(cudaStreamWaitEvent(an->cur, bt->uploaded, 0));
    st = piv_batch_run(bt);
    if (st) return st;
    CUDA_TRY(cudaEventRecord(bt->computed, an->cur));
    CUDA_TRY(cudaStreamWaitEvent(bt->down, bt->computed, 0));
    const size_t c = (size_t)bt->cells * (size_t)bt->K;
    cudaStream_t ds = bt->down;
    if (dx) CUDA_TRY(cudaMemcpyAsync(dx, bt->dx, 4 * c, cudaMemcpyDeviceToHost, ds));
    if (dy) CUDA_TRY(cudaMemcpyAsync(dy, bt->dy, 4 * c, cudaMemcpyDeviceToHost, ds));
    if (peak_ratio) CUDA_TRY(cudaMemcpyAsync(peak_ratio, bt->ppr, 4 * c, cudaMemcpyDeviceToHost, ds));
    if (flags) CUDA_TRY(cudaMemcpyAsync(flags, bt->flags, c, cudaMemcpyDeviceToHost, ds));
    CUDA_TRY(cudaMemcpyAsync(bt->hsums, bt->sums, sizeof(unsigned long long) * 8 * (size_t)bt->K, cudaMemcpyDeviceToHost,
                             ds));
    CUDA_TRY(cudaEventRecord(bt->hdone, ds));
    bt->pending = true;
    return PIV_OK;
}

int32_t piv_batch_wait_host(PivBatch* bt, PivSummaryC* summaries) {
    if (!bt) return fail(PIV_ERR_ARGUMENT, "null batch");
    if (!bt->pending) return fail(PIV_ERR_ARGUMENT, "nothing submitted");
    int st = use_device(bt->an);
    if (st) return st;
    CUDA_TRY(cudaEventSynchronize(bt->hdone));
    bt->pending = false;
    st = check_device_error(bt->an->device);
    if (st) return st;
    if (summaries)
        for (int k = 0; k < bt->K; ++k) {
            const unsigned long long* h = bt->hsums + 8 * (size_t)k;
            summaries[k] = PivSummaryC{(int64_t)h[0], (int64_t)h[1], (int64_t)h[2], (int64_t)h[3], (int64_t)h[4]};
        }
    return PIV_OK;
}

int64_t piv_batch_kernels(const PivBatch* bt) { return bt ? bt->kernels : 0; }

// ---------------------------------------------------------------------------------------------
// Serving form: continuous batching of independent requests on one stream.
// ---------------------------------------------------------------------------------------------
}  // extern "C"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    PivAnalyzer cfg;  // configuration only (no stream of its own)
    PivPreprocessC pre{};
    int32_t dtype = 0;
    int64_t H = 0, W = 0;
    const void* host_a = nullptr;
    const void* host_b = nullptr;
    float* out_dx = nullptr;
    float* out_dy = nullptr;
    float* out_ppr = nullptr;
    uint8_t* out_flags = nullptr;
    size_t bytes = 0;
    void* mem = nullptr;
    PivFrame fa, fb;
    std::vector<PassBuf> passes;
    unsigned long long* d_counts = nullptr;
    unsigned long long h_counts[8] = {};
    // Pinned staging of the downloads (the summary counts, and every output that is not in pinned
    // host memory itself): a copy into pageable memory would block the scheduler thread until the
    // GPU reached it. Unpacked into the caller's buffers when the request retires.
    uint8_t* stage = nullptr;
    int stage_class = 0;
    size_t stage_off[4] = {};  // offsets of dx, dy, peak_ratio, flags in `stage` (0: copied directly)
    bool use_stats = false;
    int next_pass = 0;
    cudaEvent_t done_ev = nullptr;
    bool final_launched = false;
    bool done = false;
    std::atomic<bool> cancel{false};  // set by piv_server_cancel; read by the scheduler
    int status = PIV_OK;
    std::string error;
    Clock::time_point t_submit, t_done;
};

// Device footprint of a request and the layout of its single allocation.
size_t request_bytes(const Request& r, bool stats, bool chain, bool both, size_t es) {
    const size_t hw = (size_t)r.H * (size_t)r.W;
    size_t b = 2 * align256(es * hw) + 2 * align256(4 * hw);
    if (chain) b += 2 * align256(4 * hw);
    if (both) b += 2 * align256(4 * hw);
    if (stats) b += 4 * align256(8 * (size_t)(r.H + 1) * (size_t)(r.W + 1));
    b += 2 * align256(4 * (4 + 512 + 4)) + 2 * align256(8);
    for (const PassBuf& pb : r.passes) {
        const size_t c = (size_t)pb.cells;
        b += align256(16 * c) + align256(c) + 3 * align256(4 * c) + 3 * align256(c) + 2 * align256(4 * c) + align256(c) +
             (r.cfg.deform ? align256(32 * c) : 0);
    }
    return b + align256(8 * sizeof(unsigned long long));
}

}  // namespace

struct PivServer {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t budget = 0;
    int max_in_flight = 1;
    std::mutex mu;
    std::condition_variable cv_submit, cv_done;
    std::deque<Request*> queue;
    std::vector<Request*> active;
    std::map<uint64_t, Request*> by_id;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    int64_t in_use = 0;
    cudaMemPool_t pool = nullptr;  // the server's own pool: requests' memory, kept when freed
    // Copy streams: an admitted request's uploads run on `up` and its result downloads on `down`,
    // so they overlap the kernels that other requests run on `stream`.
    cudaStream_t up = nullptr, down = nullptr;
    // Pinned host blocks of 2^k bytes for the download staging, reused across requests (the
    // scheduler takes and returns them; piv_server_reserve pins the first slabs ahead of time).
    std::mutex pinned_mu;
    std::vector<void*> pinned_free[48];
    std::vector<void*> pinned_all;
    bool pinned_grow(int k);  // pinned_mu held
    uint8_t* pinned_get(size_t bytes, int* cls);
    void pinned_put(uint8_t* p, int cls) {
        std::lock_guard<std::mutex> lk(pinned_mu);
        pinned_free[cls].push_back(p);
    }
    PivServerStatsC stats{};
    int variant[2][129] = {};
    // FP32 windows of several sizes and kinds in one fused correlation launch per step (on by
    // default; piv_server_set_fused(0) launches per (size, kind) instead)
    bool fused = true;
    std::vector<cudaEvent_t> step_events;  // completion of recent steps (bounded run-ahead)
    // Admission waits for a retirement after an allocation failed while requests were in flight.
    bool admission_blocked = false;
    // Host-side fault injection: the next fail_allocs admissions fail as an out-of-memory
    // allocation would, without calling the allocator.
    int fail_allocs = 0;
    // Manual stepping: the scheduler admits and launches only while granted steps remain.
    bool manual = false;
    int64_t granted = 0, stepped = 0;
    std::condition_variable cv_step;

    void loop();
    int admit(Request* r, std::string* err);
    void launch_step(std::vector<Request*>& work);
    void cancel_active();
    void retire();
};

namespace {

constexpr int kAdmitOutOfMemory = -1;

// Allocates the request's device memory on the server stream and queues the uploads and frame
// preparation (preprocess.rs:138-158) for both frames. Returns kAdmitOutOfMemory, with nothing
// allocated or queued, when the allocation fails for lack of memory (or an injected failure).
int admit_request(PivServer* sv, Request* r, bool inject_failure) {
    const size_t es = dtype_size(r->dtype);
    const size_t hw = (size_t)r->H * (size_t)r->W;
    const bool chain = r->pre.smooth_sigma > 0.0f || r->pre.normalize_radius > 0;
    const bool both = r->pre.smooth_sigma > 0.0f && r->pre.normalize_radius > 0;
    if (inject_failure) return kAdmitOutOfMemory;
    const cudaError_t ae = cudaMallocFromPoolAsync(&r->mem, r->bytes, sv->pool, sv->up);
    if (ae == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // not a sticky error: clear it and report
        r->mem = nullptr;
        return kAdmitOutOfMemory;
    }
    if (ae != cudaSuccess) return fail(PIV_ERR_CUDA, "cudaMallocFromPoolAsync: %s", cudaGetErrorString(ae));
    char* p = (char*)r->mem;
    auto take = [&](size_t bytes) {
        void* q = p;
        p += align256(bytes);
        return q;
    };
    for (PivFrame* f : {&r->fa, &r->fb}) {
        f->an = &r->cfg;
        f->device = sv->device;
        f->H = r->H;
        f->W = r->W;
        f->d_raw = take(es * hw);
        f->d_raw_bytes = es * hw;
        f->image = (float*)take(4 * hw);
        f->base = f->image;
        if (chain) f->base_store = (float*)take(4 * hw);
        if (both) f->tmp = (float*)take(4 * hw);
        if (r->use_stats) {
            f->sum = (long long*)take(8 * (size_t)(r->H + 1) * (size_t)(r->W + 1));
            f->sumsq = (long long*)take(8 * (size_t)(r->H + 1) * (size_t)(r->W + 1));
        }
        f->words = (unsigned int*)take(4 * (4 + 512 + 4));
        f->scales = (int*)take(8);
    }
    for (PassBuf& pb : r->passes) {
        const size_t c = (size_t)pb.cells;
        pb.origins = (float4*)take(16 * c);
        pb.status = (uint8_t*)take(c);
        pb.raw_dx = (float*)take(4 * c);
        pb.raw_dy = (float*)take(4 * c);
        pb.raw_ppr = (float*)take(4 * c);
        pb.raw_flags = (uint8_t*)take(c);
        pb.f1 = (uint8_t*)take(c);
        pb.f2 = (uint8_t*)take(c);
        pb.dx = (float*)take(4 * c);
        pb.dy = (float*)take(4 * c);
        pb.flags = (uint8_t*)take(c);
        pb.corners = r->cfg.deform ? (float4*)take(32 * c) : nullptr;
    }
    r->d_counts = (unsigned long long*)take(8 * sizeof(unsigned long long));
    r->cfg.cur = sv->stream;
    // allocation and uploads on the upload stream; the preparation on the server stream waits for them
    CUDA_TRY(cudaMemcpyAsync(r->fa.d_raw, r->host_a, es * hw, cudaMemcpyHostToDevice, sv->up));
    CUDA_TRY(cudaMemcpyAsync(r->fb.d_raw, r->host_b, es * hw, cudaMemcpyHostToDevice, sv->up));
    cudaEvent_t uploaded = nullptr;
    CUDA_TRY(cudaEventCreateWithFlags(&uploaded, cudaEventDisableTiming));
    cudaError_t ue = cudaEventRecord(uploaded, sv->up);
    if (ue == cudaSuccess) ue = cudaStreamWaitEvent(sv->stream, uploaded, 0);
    cudaEventDestroy(uploaded);
    CUDA_TRY(ue);
    int st = prepare_common(&r->cfg, &r->fa, r->fa.d_raw, r->dtype, &r->pre, nullptr);
    if (!st) st = prepare_common(&r->cfg, &r->fb, r->fb.d_raw, r->dtype, &r->pre, nullptr);
    return st;
}

}  // namespace

// Called with the lock released. Returns PIV_OK, kAdmitOutOfMemory, or another status with
// *err set.
int PivServer::admit(Request* r, std::string* err) {
    bool inject = false;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (fail_allocs > 0) {
            --fail_allocs;
            inject = true;
        }
    }
    const int st = admit_request(this, r, inject);
    if (st && st != kAdmitOutOfMemory) *err = g_last_error;
    return st;
}

// Pins a slab of at least 8 MiB and splits it into blocks of class k: a cudaHostAlloc costs far
// more than the copies a block serves (with one allocation per block, the download setup of a
// saturated 1 200-request run took 150-169 ms of scheduler time; with slabs 68-96 ms).
bool PivServer::pinned_grow(int k) {
    const size_t block = (size_t)1 << k;
    const size_t slab = std::max(block, (size_t)8 << 20);
    void* p = nullptr;
    if (cudaHostAlloc(&p, slab, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    pinned_all.push_back(p);
    for (size_t off = 0; off + block <= slab; off += block) pinned_free[k].push_back((uint8_t*)p + off);
    return true;
}

uint8_t* PivServer::pinned_get(size_t bytes, int* cls) {
    int k = 16;
    while (k < 47 && ((size_t)1 << k) < bytes) ++k;
    *cls = k;
    std::lock_guard<std::mutex> lk(pinned_mu);
    if (pinned_free[k].empty() && !pinned_grow(k)) return nullptr;
    uint8_t* p = (uint8_t*)pinned_free[k].back();
    pinned_free[k].pop_back();
    return p;
}

namespace {
bool is_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}
}  // namespace

// Requests cancelled while admitted stop at the step boundary: their completion event covers the
// work already queued for them, after which retire() gives their memory back.
void PivServer::cancel_active() {
    for (Request* r : active) {
        if (r->final_launched || !r->cancel.load()) continue;
        r->status = PIV_ERR_CANCELLED;
        r->error = "cancelled";
        if (cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming) == cudaSuccess)
            cudaEventRecord(r->done_ev, stream);
        else
            r->done_ev = nullptr;
        r->final_launched = true;
    }
}

// One step: the next pass of every admitted request (multipass.rs:194-259 and validate.rs:51),
// batched across requests: one placement launch, one correlation launch per window size, one
// validation chain; requests whose last pass this is get their summary and their results copied
// to host memory, followed by a completion event. Correlation launches are keyed by window size
// and window kind (uniform shift / deformed).
void PivServer::launch_step(std::vector<Request*>& work) {
    std::vector<PlaceParams> pps;
    std::map<std::pair<int, int>, std::vector<CorrParams>> cps;
    std::vector<ValidateParams> vps;
    for (Request* r : work) {
        const int i = r->next_pass;
        PassBuf& pb = r->passes[i];
        PlaceParams pp{};
        pp.grid = to_gp(pb.grid);
        pp.H = (int)r->H;
        pp.W = (int)r->W;
        pp.has_pred = i > 0;
        if (i > 0) {
            pp.pgrid = to_gp(r->passes[i - 1].grid);
            pp.pdx = r->passes[i - 1].dx;
            pp.pdy = r->passes[i - 1].dy;
        }
        pp.origins = pb.origins;
        pp.status = pb.status;
        pp.corners = (r->cfg.deform && i > 0) ? pb.corners : nullptr;
        pp.use_stats = r->use_stats;
        if (r->use_stats) {
            pp.sa = stats_of(&r->fa);
            pp.sb = stats_of(&r->fb);
        }
        pp.min_mean = r->cfg.min_mean;
        pp.min_std = r->cfg.min_std;
        pps.push_back(pp);
        // 0 / 1: FP32 uniform / deformed windows; 2 / 3: tensor cores, BF16 / FP16 split, uniform;
        // 4 / 5: the same with deformed windows
        const bool tc = split_precision(r->cfg.precision) && corr_tc_supported((int)pb.grid.window);
        const int kind = tc ? (r->cfg.precision == PIV_PRECISION_FP16X3 ? 3 : 2) + (pp.corners ? 2 : 0)
                            : (pp.corners ? 1 : 0);
        cps[{(int)pb.grid.window, kind}].push_back(
            CorrParams{r->fa.image, r->fb.image, (int)r->H, (int)r->W, pb.origins, pb.status, (int)pb.cells, pb.raw_dx,
                       pb.raw_dy, pb.raw_ppr, pb.raw_flags, pp.corners, (int)pb.grid.x0, (int)pb.grid.y0,
                       (int)pb.grid.step, (int)pb.grid.nx});
        vps.push_back(ValidateParams{(int)pb.grid.nx, (int)pb.grid.ny, pb.raw_dx, pb.raw_dy, pb.raw_ppr, pb.raw_flags, pb.f1,
                                     pb.f2, pb.dx, pb.dy, pb.flags, (float)r->cfg.windows[0] / 2.0f, r->cfg.ppr_threshold,
                                     r->cfg.median_threshold, r->cfg.median_eps, r->cfg.replace});
    }
    int nl = 0;
    cudaError_t e = launch_place_items(pps.data(), (int)pps.size(), stream, &nl);
    // FP32 windows of 8, 16, 32 and 64 px, uniform or deformed, of all requests: one fused
    // launch; other sizes and the tensor-core kinds: one launch per (size, kind)
    std::vector<CorrParams> fused_items;
    std::vector<int> fused_kinds;
    for (auto& kv : cps) {
        const int fk = (kv.first.second < 2 && fused && variant[kv.first.second][kv.first.first] == 0)
                           ? fused_kind(kv.first.first, kv.first.second == 1)
                           : -1;
        if (fk < 0) continue;
        for (const CorrParams& cp : kv.second) {
            fused_items.push_back(cp);
            fused_kinds.push_back(fk);
        }
        kv.second.clear();
    }
    if (e == cudaSuccess && !fused_items.empty())
        e = launch_correlate_fused(fused_items.data(), fused_kinds.data(), (int)fused_items.size(), stream, &nl);
    for (auto& kv : cps)
        if (e == cudaSuccess && !kv.second.empty())
            e = kv.first.second >= 2
                    ? launch_correlate_tc_items(kv.first.first, kv.first.second == 3 || kv.first.second == 5,
                                                kv.second.data(), (int)kv.second.size(), stream, &nl)
                    : launch_correlate_items(kv.first.first, variant[kv.first.second][kv.first.first], kv.second.data(),
                                             (int)kv.second.size(), stream, &nl);
    if (e == cudaSuccess) e = launch_validate_items(vps.data(), (int)vps.size(), stream, &nl);
    std::vector<SummaryItem> sums;
    for (Request* r : work) {
        r->next_pass++;
        if (r->next_pass == (int)r->passes.size()) {
            const PassBuf& last = r->passes.back();
            sums.push_back(SummaryItem{last.flags, (int)last.cells, r->d_counts});
        }
    }
    if (e == cudaSuccess && !sums.empty()) e = launch_summary_items(sums.data(), (int)sums.size(), stream, &nl);
    // downloads of the requests that finished in this step, on the download stream after the step
    if (e == cudaSuccess && !sums.empty()) {
        cudaEvent_t computed = nullptr;
        e = cudaEventCreateWithFlags(&computed, cudaEventDisableTiming);
        if (e == cudaSuccess) {
            e = cudaEventRecord(computed, stream);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(down, computed, 0);
            cudaEventDestroy(computed);
        }
    }
    for (Request* r : work) {
        if (r->next_pass != (int)r->passes.size() || e != cudaSuccess) continue;
        const PassBuf& last = r->passes.back();
        const size_t c = (size_t)last.cells;
        void* const outs[4] = {r->out_dx, r->out_dy, r->out_ppr, r->out_flags};
        const void* const srcs[4] = {last.dx, last.dy, last.raw_ppr, last.flags};
        const size_t sizes[4] = {4 * c, 4 * c, 4 * c, c};
        size_t need = 256;  // the summary counts, then each staged output 256-byte aligned
        for (int o = 0; o < 4; ++o) {
            r->stage_off[o] = 0;
            if (outs[o] && !is_pinned(outs[o])) {
                r->stage_off[o] = need;
                need += align256(sizes[o]);
            }
        }
        r->stage = pinned_get(need, &r->stage_class);
        if (!r->stage)  // no pinned host memory to be had: copy directly (slower, still correct)
            for (int o = 0; o < 4; ++o) r->stage_off[o] = 0;
        for (int o = 0; o < 4 && e == cudaSuccess; ++o)
            if (outs[o])
                e = cudaMemcpyAsync(r->stage_off[o] ? r->stage + r->stage_off[o] : outs[o], srcs[o], sizes[o],
                                    cudaMemcpyDeviceToHost, down);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(r->stage ? (void*)r->stage : (void*)r->h_counts, r->d_counts, sizeof(r->h_counts),
                                cudaMemcpyDeviceToHost, down);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(r->done_ev, down);
        r->final_launched = true;
    }
    stats.steps++;
    stats.kernel_launches += nl;
    if (e != cudaSuccess) {
        for (Request* r : work) {
            r->status = PIV_ERR_CUDA;
            r->error = cudaGetErrorString(e);
            r->final_launched = true;
        }
    }
}

// Requests whose completion event has fired: results are in host memory, memory goes back.
void PivServer::retire() {
    std::vector<Request*> keep;
    bool any = false;
    for (Request* r : active) {
        bool fin = false;
        if (r->final_launched) {
            if (!r->done_ev) {
                fin = true;  // failed before recording
            } else {
                const cudaError_t q = cudaEventQuery(r->done_ev);
                if (q == cudaSuccess) fin = true;
                else if (q != cudaErrorNotReady) {
                    r->status = PIV_ERR_CUDA;
                    r->error = cudaGetErrorString(q);
                    fin = true;
                }
            }
        }
        if (!fin) {
            keep.push_back(r);
            continue;
        }
        if (r->stage) {  // unpack the staged downloads (they completed with the completion event)
            if (!r->done_ev) cudaStreamSynchronize(down);  // failed before recording: copies may be queued
            if (r->status == PIV_OK) {
                void* const outs[4] = {r->out_dx, r->out_dy, r->out_ppr, r->out_flags};
                const size_t c = (size_t)r->passes.back().cells;
                const size_t sizes[4] = {4 * c, 4 * c, 4 * c, c};
                for (int o = 0; o < 4; ++o)
                    if (outs[o] && r->stage_off[o]) std::memcpy(outs[o], r->stage + r->stage_off[o], sizes[o]);
                std::memcpy(r->h_counts, r->stage, sizeof(r->h_counts));
            }
            pinned_put(r->stage, r->stage_class);
            r->stage = nullptr;
        }
        r->t_done = Clock::now();
        if (r->done_ev) cudaEventDestroy(r->done_ev);
        r->done_ev = nullptr;
        if (r->mem) cudaFreeAsync(r->mem, stream);
        r->mem = nullptr;
        in_use -= (int64_t)r->bytes;
        std::lock_guard<std::mutex> lk(mu);
        r->done = true;
        if (r->status == PIV_OK) stats.completed++;
        else if (r->status == PIV_ERR_CANCELLED) stats.cancelled++;
        else stats.failed++;
        stats.in_flight--;
        stats.memory_in_use_bytes = in_use;
        admission_blocked = false;
        any = true;
    }
    active.swap(keep);
    if (any) cv_done.notify_all();
}

void PivServer::loop() {
    cudaSetDevice(device);
    for (;;) {
        bool may_step = true;
        // admission at a step boundary (FIFO while slots and memory allow)
        {
            std::unique_lock<std::mutex> lk(mu);
            if (queue.empty() && active.empty()) {
                if (stop) break;
                if (manual && granted > 0) {  // a granted step with nothing to do
                    --granted;
                    ++stepped;
                    cv_step.notify_all();
                }
                cv_submit.wait_for(lk, std::chrono::milliseconds(50));
                continue;
            }
            may_step = !manual || granted > 0;
            while (may_step && !admission_blocked && !queue.empty() && (int)active.size() < max_in_flight &&
                   in_use + (int64_t)queue.front()->bytes <= budget) {
                Request* r = queue.front();
                queue.pop_front();
                stats.queued--;
                lk.unlock();
                std::string err;
                const int st = admit(r, &err);
                lk.lock();
                if (st == kAdmitOutOfMemory && !active.empty()) {
                    // the device is short of memory although the budget allows the request: try
                    // again once an admitted request has finished and given its memory back
                    queue.push_front(r);
                    stats.queued++;
                    stats.deferred++;
                    admission_blocked = true;
                    break;
                }
                if (st) {
                    r->status = st == kAdmitOutOfMemory ? PIV_ERR_CUDA : st;
                    r->error = st == kAdmitOutOfMemory
                                   ? "device memory for the request could not be allocated (out of memory)"
                                   : err;
                    if (r->mem) {
                        cudaStreamSynchronize(up);  // queued uploads may still read host memory
                        cudaStreamSynchronize(stream);
                        cudaFreeAsync(r->mem, stream);
                        r->mem = nullptr;
                    }
                    r->done = true;
                    r->t_done = Clock::now();
                    stats.failed++;
                    cv_done.notify_all();
                    continue;
                }
                in_use += (int64_t)r->bytes;
                stats.admitted++;
                stats.in_flight++;
                active.push_back(r);
            }
            stats.memory_in_use_bytes = in_use;
        }
        cancel_active();
        std::vector<Request*> work;
        if (may_step)
            for (Request* r : active)
                if (r->next_pass < (int)r->passes.size() && !r->final_launched) work.push_back(r);
        if (!work.empty()) {
            launch_step(work);
            {
                std::lock_guard<std::mutex> lk(mu);
                stats.last_step_requests = (int64_t)work.size();
                stats.max_step_requests = std::max<int64_t>(stats.max_step_requests, (int64_t)work.size());
                if (manual) {
                    --granted;
                    ++stepped;
                    cv_step.notify_all();
                }
            }
            // bounded run-ahead: keep at most two steps queued on the device
            cudaEvent_t ev;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
                cudaEventRecord(ev, stream);
                step_events.push_back(ev);
                while (step_events.size() > 2) {
                    cudaEventSynchronize(step_events.front());
                    cudaEventDestroy(step_events.front());
                    step_events.erase(step_events.begin());
                }
            }
        } else {
            if (may_step && manual) {
                // a granted step with no pass to launch (everything admitted has launched its
                // last pass): it is used up
                std::lock_guard<std::mutex> lk(mu);
                if (granted > 0) {
                    --granted;
                    ++stepped;
                    cv_step.notify_all();
                }
            }
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
        retire();
    }
    for (cudaEvent_t ev : step_events) cudaEventDestroy(ev);
    step_events.clear();
}

extern "C" {

int32_t piv_server_create(const PivServerConfigC* cfg, PivServer** out) {
    if (!cfg || !out) return fail(PIV_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    if (cfg->memory_budget_bytes <= 0 || cfg->max_in_flight <= 0) return fail(PIV_ERR_ARGUMENT, "bad server config");
    int dev = cfg->device;
    if (dev < 0) CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaSetDevice(dev));
    int st = ensure_device_init(dev);
    if (st) return st;
    // A pool of the server's own that keeps freed request memory instead of returning it to the
    // driver (piv_server_reserve grows it ahead of time).
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    CUDA_TRY(cudaMemPoolCreate(&pool, &props));
    uint64_t threshold = UINT64_MAX;
    cudaError_t e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    if (e != cudaSuccess) {
        cudaMemPoolDestroy(pool);
        return fail(PIV_ERR_CUDA, "server pool: %s", cudaGetErrorString(e));
    }
    PivServer* sv = new PivServer();
    sv->device = dev;
    sv->pool = pool;
    sv->budget = cfg->memory_budget_bytes;
    sv->max_in_flight = cfg->max_in_flight;
    e = cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->up, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->down, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        for (cudaStream_t q : {sv->stream, sv->up, sv->down})
            if (q) cudaStreamDestroy(q);
        cudaMemPoolDestroy(pool);
        delete sv;
        return fail(PIV_ERR_CUDA, "server stream: %s", cudaGetErrorString(e));
    }
    sv->worker = std::thread([sv] { sv->loop(); });
    *out = sv;
    return PIV_OK;
}

void piv_server_destroy(PivServer* sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        sv->manual = false;  // finish what is queued without waiting for granted steps
    }
    sv->cv_submit.notify_all();
    sv->cv_step.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    cudaSetDevice(sv->device);
    for (cudaStream_t q : {sv->up, sv->stream, sv->down}) cudaStreamSynchronize(q);
    for (auto& kv : sv->by_id) delete kv.second;
    for (cudaStream_t q : {sv->up, sv->stream, sv->down}) cudaStreamDestroy(q);
    for (void* p : sv->pinned_all) cudaFreeHost(p);
    if (sv->pool) cudaMemPoolDestroy(sv->pool);  // every request's memory has been freed into it
    delete sv;
}

int32_t piv_server_reserve(PivServer* sv, int64_t bytes, int64_t* reserved_bytes) {
    if (!sv) return fail(PIV_ERR_ARGUMENT, "null server");
    if (bytes < 0) return fail(PIV_ERR_ARGUMENT, "negative reservation");
    CUDA_TRY(cudaSetDevice(sv->device));
    int st = PIV_OK;
    if (bytes > 0) {
        // Allocate the reservation in chunks on a stream of its own, free it again and wait: the
        // pool keeps the memory (release threshold at its maximum) and serves later admissions on
        // the server stream from it once the frees have completed.
        constexpr int64_t kChunk = 1ll << 30;
        cudaStream_t s = nullptr;
        CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        std::vector<void*> chunks;
        cudaError_t e = cudaSuccess;
        for (int64_t left = bytes; left > 0 && e == cudaSuccess;) {
            const int64_t n = std::min(left, kChunk);
            void* p = nullptr;
            e = cudaMallocFromPoolAsync(&p, (size_t)n, sv->pool, s);
            if (e == cudaSuccess) chunks.push_back(p);
            left -= n;
        }
        if (e != cudaSuccess) {
            cudaGetLastError();  // an out-of-memory allocation is not a sticky error
            st = fail(PIV_ERR_CUDA, "piv_server_reserve: %s after %zu chunk(s)", cudaGetErrorString(e), chunks.size());
        }
        for (void* p : chunks) cudaFreeAsync(p, s);
        const cudaError_t se = cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        if (se != cudaSuccess && st == PIV_OK) st = fail(PIV_ERR_CUDA, "piv_server_reserve: %s", cudaGetErrorString(se));
    }
    if (bytes > 0) {
        // and one staging slab for each download size up to 1 MiB (final fields up to 80 k cells),
        // so that the first requests do not wait for host memory to be pinned either
        std::lock_guard<std::mutex> lk(sv->pinned_mu);
        for (int k = 16; k <= 20; ++k)
            if (sv->pinned_free[k].empty()) sv->pinned_grow(k);
    }
    if (reserved_bytes) {
        uint64_t held = 0;
        CUDA_TRY(cudaMemPoolGetAttribute(sv->pool, cudaMemPoolAttrReservedMemCurrent, &held));
        *reserved_bytes = (int64_t)held;
    }
    return st;
}

int32_t piv_server_submit(PivServer* sv, const PivRequestC* q, uint64_t* id) {
    if (!sv || !q || !id) return fail(PIV_ERR_ARGUMENT, "null argument");
    int st = check_cfg(&q->config);
    if (st) return st;
    const size_t es = dtype_size(q->dtype);
    if (!es) return fail(PIV_ERR_ARGUMENT, "unknown dtype %d", q->dtype);
    if (!q->frame_a || !q->frame_b) return fail(PIV_ERR_ARGUMENT, "null frame");
    if (q->preprocess.clip_percentile > 0.0 && q->dtype == PIV_DTYPE_F32)
        return fail(PIV_ERR_UNSUPPORTED, "percentile clipping needs integer (u8/u16) samples");
    Request* r = new Request();
    PivAnalyzer& c = r->cfg;
    c.windows.assign(q->config.windows, q->config.windows + q->config.n_windows);
    c.overlap = q->config.overlap;
    c.final_iterations = q->config.final_iterations;
    c.min_mean = q->config.min_mean;
    c.min_std = q->config.min_std;
    c.ppr_threshold = q->config.ppr_threshold;
    c.median_threshold = q->config.median_threshold;
    c.median_eps = q->config.median_eps;
    c.replace = q->config.replace;
    c.deform = q->config.deform;
    c.precision = q->config.precision;
    c.device = sv->device;
    r->pre = q->preprocess;
    r->dtype = q->dtype;
    r->H = q->height;
    r->W = q->width;
    r->host_a = q->frame_a;
    r->host_b = q->frame_b;
    r->out_dx = q->dx;
    r->out_dy = q->dy;
    r->out_ppr = q->peak_ratio;
    r->out_flags = q->flags;
    for (int32_t n : c.pass_windows()) {
        PassBuf pb{};
        st = make_grid(r->H, r->W, n, c.overlap, &pb.grid);
        if (st) {
            delete r;
            return st;
        }
        pb.cells = pb.grid.nx * pb.grid.ny;
        r->passes.push_back(pb);
    }
    const bool chain = r->pre.smooth_sigma > 0.0f || r->pre.normalize_radius > 0;
    const bool both = r->pre.smooth_sigma > 0.0f && r->pre.normalize_radius > 0;
    r->fa.nonneg = r->fb.nonneg = r->dtype != PIV_DTYPE_F32;
    r->use_stats = !c.mask_trivial() || r->dtype == PIV_DTYPE_F32;
    r->bytes = request_bytes(*r, r->use_stats, chain, both, es);
    if ((int64_t)r->bytes > sv->budget) {
        const size_t b = r->bytes;
        delete r;
        return fail(PIV_ERR_UNSUPPORTED, "request needs %zu bytes of device memory, above the budget", b);
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        r->id = sv->next_id++;
        sv->by_id[r->id] = r;
        sv->queue.push_back(r);
        sv->stats.submitted++;
        sv->stats.queued++;
    }
    sv->cv_submit.notify_all();
    *id = r->id;
    return PIV_OK;
}

namespace {

// Waits for request `id` (forever when timeout_ms < 0); on completion fills the summary and
// latency, forgets the request and returns its status.
int32_t server_wait(PivServer* sv, uint64_t id, double timeout_ms, PivSummaryC* summary, double* latency_ms) {
    if (!sv) return fail(PIV_ERR_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->by_id.find(id);
    if (it == sv->by_id.end()) return fail(PIV_ERR_ARGUMENT, "unknown request %llu", (unsigned long long)id);
    Request* r = it->second;
    if (timeout_ms < 0.0) {
        sv->cv_done.wait(lk, [r] { return r->done; });
    } else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                     [r] { return r->done; })) {
        return fail(PIV_ERR_TIMEOUT, "request %llu not done within %g ms", (unsigned long long)id, timeout_ms);
    }
    sv->by_id.erase(it);
    lk.unlock();
    const int st = r->status;
    if (st) fail(st, "request %llu: %s", (unsigned long long)id, r->error.c_str());
    if (summary) {
        summary->no_signal = (int64_t)r->h_counts[0];
        summary->low_ppr = (int64_t)r->h_counts[1];
        summary->median_outliers = (int64_t)r->h_counts[2];
        summary->out_of_range = (int64_t)r->h_counts[3];
        summary->replaced = (int64_t)r->h_counts[4];
    }
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    delete r;
    return st;
}

}  // namespace

int32_t piv_server_wait(PivServer* sv, uint64_t id, PivSummaryC* summary, double* latency_ms) {
    return server_wait(sv, id, -1.0, summary, latency_ms);
}

int32_t piv_server_wait_timeout(PivServer* sv, uint64_t id, double timeout_ms, PivSummaryC* summary,
                                double* latency_ms) {
    if (!(timeout_ms >= 0.0)) return fail(PIV_ERR_ARGUMENT, "timeout_ms must be >= 0");
    return server_wait(sv, id, timeout_ms, summary, latency_ms);
}

int32_t piv_server_cancel(PivServer* sv, uint64_t id) {
    if (!sv) return fail(PIV_ERR_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->by_id.find(id);
    if (it == sv->by_id.end()) return fail(PIV_ERR_ARGUMENT, "unknown request %llu", (unsigned long long)id);
    Request* r = it->second;
    if (r->done) return PIV_OK;  // finished already: its result stands
    auto q = std::find(sv->queue.begin(), sv->queue.end(), r);
    if (q != sv->queue.end()) {
        // not admitted: nothing of it is on the device
        sv->queue.erase(q);
        sv->stats.queued--;
        sv->stats.cancelled++;
        r->status = PIV_ERR_CANCELLED;
        r->error = "cancelled before admission";
        r->done = true;
        r->t_done = Clock::now();
        sv->cv_done.notify_all();
        return PIV_OK;
    }
    r->cancel.store(true);  // admitted: stops at the next step boundary
    return PIV_OK;
}

int32_t piv_server_fail_next_allocations(PivServer* sv, int32_t count) {
    if (!sv || count < 0) return fail(PIV_ERR_ARGUMENT, "bad argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->fail_allocs = count;
    return PIV_OK;
}

int32_t piv_server_set_fused(PivServer* sv, int32_t fused) {
    if (!sv) return fail(PIV_ERR_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->fused = fused != 0;
    return PIV_OK;
}

int32_t piv_server_set_manual(PivServer* sv, int32_t manual) {
    if (!sv) return fail(PIV_ERR_ARGUMENT, "null server");
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->manual = manual != 0;
        sv->granted = 0;
    }
    sv->cv_submit.notify_all();
    sv->cv_step.notify_all();  // an advance still waiting returns
    return PIV_OK;
}

int32_t piv_server_advance(PivServer* sv, int32_t steps, double timeout_ms) {
    if (!sv || steps < 0) return fail(PIV_ERR_ARGUMENT, "bad argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    if (!sv->manual) return fail(PIV_ERR_ARGUMENT, "the server is not in manual mode");
    const int64_t target = sv->stepped + steps;
    sv->granted += steps;
    sv->cv_submit.notify_all();
    const bool ok = sv->cv_step.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms < 0 ? 1e12 : timeout_ms),
                                         [sv, target] { return sv->stepped >= target || !sv->manual || sv->stop; });
    if (!ok) return fail(PIV_ERR_TIMEOUT, "%d steps not taken within %g ms", steps, timeout_ms);
    if (sv->stepped < target)
        return fail(PIV_ERR_ARGUMENT, "manual stepping ended (piv_server_set_manual(0) or destroy) before the steps were taken");
    return PIV_OK;
}

int32_t piv_server_stats(PivServer* sv, PivServerStatsC* out) {
    if (!sv || !out) return fail(PIV_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    *out = sv->stats;
    return PIV_OK;
}

}  // extern "C"
