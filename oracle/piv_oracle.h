/*
 * CPU oracle for the PIV multipass analysis path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference's `piv-core` algorithms (Rust):
 *   grid.rs:20-66, field.rs:56-81, preprocess.rs:41-216, correlate.rs:99-303,
 *   multipass.rs:152-259, validate.rs:51-170.
 * Parity is pinned against the seven golden cases the Rust reference itself wrote
 * (swift/Tests/PIVKitTests/Fixtures/cases, generator rust/crates/piv-core/examples/fixtures.rs),
 * committed here as tests/golden/*.npz.
 *
 * Only tests, the smoke check and the CPU-baseline leg of the benchmark may load this library;
 * the product path (libpivb200.so) never calls it.
 *
 * Two arithmetic modes for the correlation:
 *   ORC_REF  (0): f32 where the reference uses f32, f64 where it uses f64 (window mean/energy,
 *                 integral images, correlation scale), no FMA contraction.
 *   ORC_FP64 (1): every correlation step in f64 (the accuracy oracle).
 */
#ifndef PIV_ORACLE_H
#define PIV_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_REF = 0, ORC_FP64 = 1 };

/* Status codes mirror PivError (error.rs:4-19). */
enum { ORC_OK = 0, ORC_ERR_CONFIG = 1, ORC_ERR_SHAPE = 2, ORC_ERR_TOO_SMALL = 3 };

typedef struct {
    int64_t window, step, nx, ny, x0, y0;
} OrcGrid;

typedef struct {
    int64_t no_signal, low_ppr, median_outliers, out_of_range, replaced;
} OrcSummary;

typedef struct {
    /* PivConfig (multipass.rs:39-51) */
    const int32_t* windows;
    int32_t n_windows;
    float overlap;
    int32_t final_iterations;
    float min_mean, min_std;             /* MaskConfig */
    float ppr_threshold, median_threshold, median_eps; /* ValidationConfig */
    int32_t replace;
    int32_t deform; /* 0: the reference's uniform window shift; 1: deformed windows */
} OrcConfig;

int orc_grid(int64_t height, int64_t width, int64_t window, float overlap, OrcGrid* out);

/* u8/u16 samples -> f32 intensities (decode.rs:227-234). */
void orc_u8_to_f32(const uint8_t* src, int64_t n, float* dst);
void orc_u16_to_f32(const uint16_t* src, int64_t n, float* dst);

/* Percentile clip of integer codes (not in the reference): codes above the p-th percentile
 * code (smallest c with count(code <= c) >= ceil(p/100 * n)) are set to it. Returns the code. */
int64_t orc_percentile_clip_u16(uint16_t* codes, int64_t n, double percentile);

/* BackgroundEstimator (preprocess.rs:41-72): mode 0 = min, 1 = mean over `count` frames. */
void orc_background(const float* frames, int64_t count, int64_t npix, int mode, float* out);

/* PreparedFrame::new (preprocess.rs:138-158). base_out (nullable) receives the
 * background-subtracted raw intensity whose integral image drives the signal mask. */
void orc_prepare(const float* raw, const float* background, int64_t h, int64_t w, float smooth_sigma,
                 int64_t normalize_radius, float normalize_eps, float* image_out, float* base_out);
void orc_gaussian_blur(const float* src, int64_t h, int64_t w, float sigma, float* out);
void orc_local_normalize(const float* src, int64_t h, int64_t w, int64_t radius, float eps, float* out);
/* IntegralImage::stats (preprocess.rs:76-125) of `frame` over the w x h box at (x, y). */
void orc_box_stats(const float* frame, int64_t h, int64_t w, int64_t bx, int64_t by, int64_t bw,
                   int64_t bh, float* mean, float* std);

/* Window placement for one pass (multipass.rs:204-231 with field.rs:56-81 as predictor).
 * pgrid/pdx/pdy may be NULL (first pass). origins: [ax, ay, bx, by] per cell. */
void orc_place(const OrcGrid* grid, int64_t h, int64_t w, const OrcGrid* pgrid, const float* pdx,
               const float* pdy, float* origins);

/* Correlate every cell of one pass (multipass.rs:232-259): signal mask on base_a/base_b,
 * correlation of image_a/image_b at the origins, assembly d = (b - a) + peak.
 * flags_out: 0 or NO_SIGNAL. nthreads <= 0 means all. */
void orc_correlate_pass(const float* image_a, const float* image_b, const float* base_a,
                        const float* base_b, int64_t h, int64_t w, int64_t n, int64_t ncells,
                        const float* origins, float min_mean, float min_std, int mode, int nthreads,
                        float* dx, float* dy, float* ppr, uint8_t* flags);

/* CorrelationPlan::correlate for one window pair (correlate.rs:99-139).
 * Returns 1 and fills peak[4] = {dx, dy, height, ppr}, or 0 for a flat window. */
int orc_correlate_window(const float* a, int64_t ha, int64_t wa, float ax, float ay, const float* b,
                         int64_t hb, int64_t wb, float bx, float by, int64_t n, int mode, float* peak);
/* load_window (correlate.rs:182-210): returns the energy. */
double orc_load_window(const float* img, int64_t h, int64_t w, float x, float y, int64_t n, float* dst);
/* find_peak (correlate.rs:215-303) on an n x n f32 plane. */
void orc_find_peak(const float* corr, int64_t n, float* peak);
/* Full correlation plane (scaled) for one window pair; returns 0 for a flat window. */
int orc_correlation_plane(const float* a, int64_t ha, int64_t wa, float ax, float ay, const float* b,
                          int64_t hb, int64_t wb, float bx, float by, int64_t n, int mode, float* plane);

/* Window deformation (not in the reference, whose windows only shift: multipass.rs:224-231;
 * deformation is deferred in docs/phase1-plan.md:104,248). Parity of these is unpinned against the
 * reference and pinned against this restatement only.
 *
 * A deformed window's base position (x0, y0) is its zero-shift origin under the placement clamp
 * (multipass.rs:207-208): the grid origin clamped to [0, w - n - 1] x [0, h - n - 1].
 *
 * orc_place_deform: as orc_place, plus the predictor (field.rs:56-81 sampling) at the four corner
 * pixels of each window's base position (x0, y0), (x0+n-1, y0), (x0, y0+n-1), (x0+n-1, y0+n-1):
 * corners[8k..8k+7] = dx00, dy00, dx10, dy10, dx01, dy01, dx11, dy11. Without a predictor all zero.
 *
 * orc_correlate_pass_deform: every pixel (r, c) of the window at base position (x0, y0) is
 * displaced by the bilinear blend of the corners, D = (1-u)(1-v) D00 + u(1-v) D10 + (1-u)v D01
 * + uv D11 with u = c/(n-1), v = r/(n-1) (f32, left to right); window A samples frame A at
 * (x0+c, y0+r) - D/2 and window B frame B at + D/2, bilinearly with coordinates clamped to the
 * image; the vector is D(center) + peak, D(center) the blend at u = v = 1/2. The signal mask
 * uses the undeformed origins (`origins`, from orc_place). */
void orc_place_deform(const OrcGrid* grid, int64_t h, int64_t w, const OrcGrid* pgrid, const float* pdx,
                      const float* pdy, float* origins, float* corners);
void orc_correlate_pass_deform(const float* image_a, const float* image_b, const float* base_a,
                               const float* base_b, int64_t h, int64_t w, const OrcGrid* grid,
                               const float* origins, const float* corners, float min_mean, float min_std,
                               int mode, int nthreads, float* dx, float* dy, float* ppr, uint8_t* flags);

/* validate (validate.rs:51-130) in place. */
void orc_validate(float* dx, float* dy, const float* ppr, uint8_t* flags, int64_t ny, int64_t nx,
                  float ppr_threshold, float median_threshold, float median_eps, int replace,
                  float max_displacement, OrcSummary* summary);

/* PivAnalyzer::{new, analyze_traced} (multipass.rs:91-192).
 * If trace_* are non-NULL they receive every pass concatenated (cells of pass 0, then pass 1, ...).
 * final_* receive the last pass's validated field. Returns a status code. */
int orc_check_config(const OrcConfig* cfg);
int orc_num_passes(const OrcConfig* cfg);
int orc_analyze(const OrcConfig* cfg, const float* image_a, const float* image_b, const float* base_a,
                const float* base_b, int64_t h, int64_t w, int mode, int nthreads, float* final_dx,
                float* final_dy, float* final_ppr, uint8_t* final_flags, OrcSummary* summary,
                float* trace_origins, float* trace_raw_dx, float* trace_raw_dy, float* trace_raw_ppr,
                uint8_t* trace_raw_flags, float* trace_dx, float* trace_dy, float* trace_ppr,
                uint8_t* trace_flags);

/* Post-processing of validated fields (the next components after the pair analysis).
 * orc_usable: flow.rs:13-17. orc_vorticity / orc_flow_stats: flowstats.rs:28-101. orc_pair_stats:
 * flow.rs:20-36 (displacement px -> px/s with k = f32(1/dt)). orc_temporal: smooth.rs:44-128
 * (median != 0: median kernel). orc_spatial: smooth.rs:130-207 (leave_out < 0: none). */
typedef struct {
    float vorticity_mean, vorticity_abs_mean, ke_mean, ke_sum, coverage;
    int64_t n_usable, n_vorticity;
} OrcFlowStats;
void orc_usable(const float* dx, const uint8_t* flags, int64_t n, uint8_t* usable);
void orc_vorticity(const float* u, const float* v, const uint8_t* usable, int64_t ny, int64_t nx, float step,
                   float* w);
void orc_flow_stats(const float* u, const float* v, const uint8_t* usable, int64_t ny, int64_t nx, float step,
                    OrcFlowStats* out);
void orc_pair_stats(const float* dx, const float* dy, const uint8_t* flags, int64_t ny, int64_t nx, int64_t step,
                    double dt_s, OrcFlowStats* out);
int orc_temporal_offsets(int32_t window, const int32_t* leave_out, int32_t n_leave, int32_t* offsets);
void orc_temporal(const float* dx, const float* dy, const uint8_t* usable, const uint8_t* gate, int64_t nt,
                  int64_t ny, int64_t nx, int32_t median, int32_t window, int32_t min_support, const int32_t* leave_out,
                  int32_t n_leave, float* out_dx, float* out_dy, uint16_t* support);
int orc_spatial_kernel(float sigma, int32_t leave_out, float* weights, float* full, float* total);
void orc_spatial(const float* dx, const float* dy, const uint8_t* gate, int64_t nt, int64_t ny, int64_t nx,
                 float sigma, float min_weight, int32_t leave_out, float* out_dx, float* out_dy, uint16_t* support);

/* SplitMix64 (synthetic.rs:10-36), exposed so tests can pin the Python restatement. */
uint64_t orc_splitmix_next(uint64_t* state);

#ifdef __cplusplus
}
#endif
#endif
