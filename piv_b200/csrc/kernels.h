// Host-side launchers of the B200 PIV kernels (internal to libpivb200.so).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace pivb200 {

// Sets the message piv_last_error returns on this host thread.
void set_last_error(const char* msg);

// ----------------------------------------------------------------------------- correlation
struct CorrParams {
    const float* img_a;
    const float* img_b;
    int H, W;
    const float4* origins;   // [ax, ay, bx, by] per cell
    const uint8_t* status;   // 1 = window pair has signal, 0 = masked (NO_SIGNAL)
    int ncells;
    float* raw_dx;
    float* raw_dy;
    float* raw_ppr;
    uint8_t* raw_flags;      // 0 or NO_SIGNAL
    // Deformed windows (null = the reference's uniform shift): 2 float4 per cell holding the
    // predictor at the window's four corner pixels (dx00, dy00, dx10, dy10 | dx01, dy01, dx11,
    // dy11), and the pass grid that gives each cell's undeformed position.
    const float4* corners;
    int gx0, gy0, gstep, gnx;
};

// Kernels take a batch of independent work items (pairs, passes or requests, of any sizes) by
// value, so that one launch covers many items and the launch can be captured in a CUDA graph
// without any device-side descriptor table. Launchers split longer lists into batches.
constexpr int kMaxBatch = 64;

// Item index that owns global unit `u` (block or cell) given exclusive prefix starts.
__host__ __device__ __forceinline__ int batch_item(const int* start, int n, int u) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
}

struct CorrBatch {
    int n;
    int block_start[kMaxBatch + 1];
    CorrParams item[kMaxBatch];
};

bool corr_supported(int n);
cudaError_t corr_init_device();  // uploads the root-of-unity table to the current device
cudaError_t launch_correlate(int n, const CorrParams& p, cudaStream_t s);
// Launch variants of one window size (identical results; different geometry), for the autotuner.
int corr_num_variants(int n, bool deform = false);
const char* corr_variant_name(int n, int v, bool deform = false);
cudaError_t launch_correlate_variant(int n, int v, const CorrParams& p, cudaStream_t s);
// All items share window size n and either all have corners (deformed windows) or none; v
// indexes the variants of that kind. Returns the number of launches issued in *launches.
cudaError_t launch_correlate_items(int n, int v, const CorrParams* items, int count, cudaStream_t s, int* launches);
// One launch over FP32 items of different window sizes and kinds: kinds[i] = fused_kind(window,
// deformed) of item i (window 8, 16, 32 or 64). Results equal the per-size launches bit for bit.
int fused_kind(int n, bool deform);
cudaError_t launch_correlate_fused(const CorrParams* items, const int* kinds, int count, cudaStream_t s,
                                   int* launches);
// Split-precision (BF16 or FP16 hi/lo, three products) tensor-core correlation, window sizes 16
// and 32; all items of a call are uniform windows or all deformed (corners set).
// corr_tc_init_device uploads its DFT matrices and deformation ramps to the current device;
// corr_tc_error reads the device's error word (non-zero after a tensor-core wait ran out).
bool corr_tc_supported(int n);
cudaError_t corr_tc_init_device();
unsigned int corr_tc_error(int device);
cudaError_t launch_correlate_tc_items(int n, bool f16, const CorrParams* items, int count, cudaStream_t s,
                                      int* launches);
// D (128 x n) = A (128 x k) * B (n x k)^T on the tensor cores, BF16 operands (device pointers).
cudaError_t tc_selftest(int a_mn, int n, int k, const float* a, const float* b, float* d);
// The correlation kernel's bounded mbarrier wait on a barrier that nothing completes; reports
// whether the wait recorded a timeout and how long the probe kernel took.
cudaError_t tc_wait_probe(int log2_iters, unsigned int* timed_out, float* ms);
// Number of kernel launches launch_correlate issues (for launch accounting).
constexpr int kCorrLaunches = 1;

// ----------------------------------------------------------------------------- field stages
// Exact window statistics of a frame's background-subtracted intensity (preprocess.rs:76-125):
// int64 fixed-point integral tables plus the fixed-point scales.
struct StatsView {
    const long long* sum;    // (H+1) x (W+1)
    const long long* sumsq;  // (H+1) x (W+1)
    const int* scales;       // [s1, s2]
    int H, W;
};

struct PlaceParams {
    GridP grid;
    int H, W;
    GridP pgrid;
    int has_pred;
    const float* pdx;  // predictor = previous pass's validated field
    const float* pdy;
    float4* origins;
    uint8_t* status;
    float4* corners;  // nullable: predictor at the four corner pixels of each window (deformation)
    // signal mask (multipass.rs:233-241); use_stats = 0 means every window has signal
    int use_stats;
    StatsView sa, sb;
    float min_mean, min_std;
};

cudaError_t launch_place(const PlaceParams& p, cudaStream_t s);
cudaError_t launch_place_items(const PlaceParams* items, int count, cudaStream_t s, int* launches);
// Mask only (origins given): fills status from origins.
cudaError_t launch_mask(const PlaceParams& p, const float4* origins, int ncells, cudaStream_t s);

struct ValidateParams {
    int nx, ny;
    const float* dx;      // raw field
    const float* dy;
    const float* ppr;
    const uint8_t* flags0;  // raw flags (0 / NO_SIGNAL)
    uint8_t* flags1;        // scratch: after per-vector tests
    uint8_t* flags2;        // scratch: after the median test
    float* out_dx;
    float* out_dy;
    uint8_t* out_flags;
    float max_displacement, ppr_threshold, median_threshold, median_eps;
    int replace;
};

cudaError_t launch_validate(const ValidateParams& p, cudaStream_t s);
cudaError_t launch_validate_items(const ValidateParams* items, int count, cudaStream_t s, int* launches);
constexpr int kValidateLaunches = 3;

// Summary counts from a validated flag field (validate.rs:40-46): no_signal, low_ppr,
// median_outliers, out_of_range, replaced.
cudaError_t launch_summary(const uint8_t* flags, int n, unsigned long long* counts5, cudaStream_t s);
constexpr int kSummaryLaunches = 2;
struct SummaryItem {
    const uint8_t* flags;
    int n;
    unsigned long long* counts5;
};
cudaError_t launch_summary_items(const SummaryItem* items, int count, cudaStream_t s, int* launches);

// ----------------------------------------------------------------------------- post-processing
// Flow statistics of one validated field (flowstats.rs:67-101 via flow.rs:20-36); blocking.
struct FlowStatsHost {
    float vorticity_mean, vorticity_abs_mean, ke_mean, ke_sum, coverage;
    long long n_usable, n_vorticity;
};
cudaError_t flow_stats_device(int ny, int nx, float step, double dt_s, const float* dx, const float* dy,
                              const uint8_t* flags, float* vort, FlowStatsHost* stats, cudaStream_t s);
// Temporal filter (smooth.rs:44-128) with the offsets already resolved (leave-out applied).
cudaError_t temporal_smooth_device(int nt, int ny, int nx, const float* dx, const float* dy, const uint8_t* usable,
                                   const uint8_t* gate, int median, const int* offsets, int n_off, int min_support,
                                   float* out_dx, float* out_dy, uint16_t* support, cudaStream_t s);
// Spatial filter (smooth.rs:130-207); leave_out < 0 means none. sigma up to 12 grid cells.
cudaError_t spatial_smooth_device(int nt, int ny, int nx, const float* dx, const float* dy, const uint8_t* gate,
                                  float sigma, float min_weight, int leave_out, float* out_dx, float* out_dy,
                                  uint16_t* support, cudaStream_t s);

// ----------------------------------------------------------------------------- preprocessing
enum RawType { RAW_U8 = 0, RAW_U16 = 1, RAW_F32 = 2 };

struct PrepParams {
    int H, W;
    const void* raw;
    int raw_type;
    const float* background;  // nullable
    int clip_percentile_on;
    double clip_percentile;
    unsigned int* hist;       // scratch: 256 + 256 + 4 words when clipping
    float* base;              // background-subtracted intensity (output, H x W)
    float* image;             // prepared image (output, H x W)
    float* tmp;               // scratch H x W (blur intermediate)
    float smooth_sigma;
    int normalize_radius;
    float normalize_eps;
    // integral tables of `base` (built when build_stats)
    int build_stats;
    long long* sum;
    long long* sumsq;
    int* scales;
    unsigned int* maxbits;    // scratch word
};

// Runs the whole PreparedFrame::new chain; returns the number of kernels launched in *launches.
cudaError_t launch_prepare(const PrepParams& p, cudaStream_t s, int* launches);
// Integral tables only (used when the prepared image is supplied directly).
// The reference's f64 IntegralImage tables, already copied into `sum` / `sumsq` (8 bytes per
// entry, (H+1) x (W+1)), converted in place to the fixed-point tables launch_stats builds;
// *nonfinite becomes nonzero if an entry is not finite. maxbits2: 2 device words of scratch.
cudaError_t launch_tables_to_fixed(long long* sum, long long* sumsq, int H, int W, int* scales,
                                   unsigned long long* maxbits2, unsigned int* nonfinite, cudaStream_t s, int* launches);
cudaError_t launch_stats(const float* base, int H, int W, long long* sum, long long* sumsq, int* scales,
                         unsigned int* maxbits, cudaStream_t s, int* launches);

}  // namespace pivb200
