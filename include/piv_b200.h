/*
 * piv_b200 — C ABI of the B200 PIV analysis path (libpivb200.so).
 *
 * Drop-in boundary for the reference's per-pair analysis (agoodman/piv, crate piv-core):
 * plain pointers, sizes and status codes; no CUDA or torch types in any signature. Device
 * pointers are plain `void*`/`float*` addresses in the current CUDA context; a stream is passed
 * as `void*` (a cudaStream_t, NULL = the analyzer's own stream).
 *
 * Reference interfaces replaced (paths within the reference project):
 *   PivAnalyzer::new(PivConfig)            rust/crates/piv-core/src/multipass.rs:91-119
 *   PivAnalyzer::output_grid               rust/crates/piv-core/src/multipass.rs:126-133
 *   PivAnalyzer::analyze                   rust/crates/piv-core/src/multipass.rs:136-138
 *   PivAnalyzer::analyze_traced            rust/crates/piv-core/src/multipass.rs:142-150
 *   PreparedFrame::new                     rust/crates/piv-core/src/preprocess.rs:138-158
 *   BackgroundEstimator::{add,finish}      rust/crates/piv-core/src/preprocess.rs:47-72
 *   Grid::new                              rust/crates/piv-core/src/grid.rs:20-44
 *   validate                               rust/crates/piv-core/src/validate.rs:51-130
 *   PivError                               rust/crates/piv-core/src/error.rs:4-19
 *
 * Output layout: fields are [ny * nx] row-major (ndarray standard layout of VectorField,
 * field.rs:26-45); flags use the reference's bits (field.rs:6-20).
 *
 * Threading: an analyzer (and the frames created from it) is used by one host thread at a
 * time, as PIVKit pools one analyzer per in-flight pair (swift/Sources/PIVKit/Run.swift:160).
 */
#ifndef PIV_B200_H
#define PIV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIV_B200_ABI_VERSION 1

/* Status codes. 1-4 mirror PivError's variants (error.rs:4-19). */
typedef enum {
    PIV_OK = 0,
    PIV_ERR_CONFIG = 1,          /* PivError::Config */
    PIV_ERR_SHAPE_MISMATCH = 2,  /* PivError::ShapeMismatch */
    PIV_ERR_IMAGE_TOO_SMALL = 3, /* PivError::ImageTooSmall */
    PIV_ERR_FRAME_RATE = 4,      /* PivError::FrameRate (not produced by this library) */
    PIV_ERR_CUDA = 5,            /* a CUDA runtime call failed; see piv_last_error */
    PIV_ERR_UNSUPPORTED = 6,     /* valid for the reference, not supported by this GPU path */
    PIV_ERR_ARGUMENT = 7,        /* NULL handle or malformed argument */
    PIV_ERR_CANCELLED = 8,       /* serving form: the request was cancelled (piv_server_cancel) */
    PIV_ERR_TIMEOUT = 9          /* serving form: a bounded wait ran out; nothing was lost */
} PivStatus;

/* Flag bits (field.rs:6-20). */
#define PIV_FLAG_NO_SIGNAL 0x01u
#define PIV_FLAG_LOW_PPR 0x02u
#define PIV_FLAG_MEDIAN_OUTLIER 0x04u
#define PIV_FLAG_REPLACED 0x08u
#define PIV_FLAG_OUT_OF_RANGE 0x10u
#define PIV_FLAG_INVALID 0x17u

typedef enum { PIV_DTYPE_U8 = 0, PIV_DTYPE_U16 = 1, PIV_DTYPE_F32 = 2 } PivDtype;

/* Arithmetic of the window correlation (no counterpart in the reference, which has FP32 only):
 * PIV_PRECISION_FP32 runs the FFTs on the FP32 cores in the reference's precision;
 * PIV_PRECISION_BF16X3 runs the 2-D DFTs as DFT-matrix products on the tensor cores with every
 * operand split into two BF16 halves and three products summed in FP32 (about 16 significant
 * bits) for window sizes 16, 32 and 64, uniform or deformed; other sizes keep the FP32 kernel.
 * piv_analyzer_autotune also times the tensor-core kernel and keeps the FP32 kernel (higher
 * precision) for a size where it is faster. */
#define PIV_PRECISION_FP32 0
#define PIV_PRECISION_BF16X3 1
#define PIV_PRECISION_FP16X3 2  /* as BF16X3 with FP16 halves: about 22 significant bits */

/* PivConfig + MaskConfig + ValidationConfig (multipass.rs:22-63, validate.rs:7-37).
 * Defaults of the reference: windows {96, 64}, overlap 0.5, final_iterations 2, mask 0/0,
 * ppr 1.3, median threshold 2, median eps 0.1, replace 1. */
typedef struct {
    const int32_t* windows; /* window size per pass, largest first; each even and >= 8 */
    int32_t n_windows;
    float overlap;          /* in [0, 1) */
    int32_t final_iterations; /* >= 1 */
    float min_mean;         /* MaskConfig */
    float min_std;
    float ppr_threshold;    /* ValidationConfig */
    float median_threshold;
    float median_eps;
    int32_t replace;
    int32_t device;         /* CUDA device ordinal; -1 = current device */
    int32_t deform;         /* 0: windows shift uniformly (the reference, multipass.rs:224-231);
                             * 1: from the second pass on, windows deform with the predictor
                             * (see piv_correlate_deform) */
    int32_t precision;      /* PIV_PRECISION_FP32 (the reference), _BF16X3 or _FP16X3 */
} PivConfigC;

/* PreprocessConfig (preprocess.rs:5-29) plus the percentile clip of integer codes
 * (clip_percentile in (0, 100]; 0 = off; not in the reference). Reference defaults:
 * smooth_sigma 1, normalize_radius 4, normalize_eps 0.02. */
typedef struct {
    float smooth_sigma;
    int32_t normalize_radius;
    float normalize_eps;
    double clip_percentile;
} PivPreprocessC;

/* Grid (grid.rs:8-16). */
typedef struct {
    int64_t window, step, nx, ny, x0, y0;
} PivGridC;

/* ValidationSummary (validate.rs:39-46). */
typedef struct {
    int64_t no_signal, low_ppr, median_outliers, out_of_range, replaced;
} PivSummaryC;

typedef struct PivAnalyzer PivAnalyzer;
typedef struct PivFrame PivFrame;

/* ----------------------------------------------------------------------------- library */
int32_t piv_abi_version(void);
/* Message of the last failure on this host thread (also set by creation failures). */
const char* piv_last_error(void);
/* Grid::new (grid.rs:20-44) — host arithmetic, no GPU needed. */
int32_t piv_grid(int64_t height, int64_t width, int64_t window, float overlap, PivGridC* out);
/* Validates a config exactly as PivAnalyzer::new does (multipass.rs:91-119), then the GPU
 * restriction (window sizes 8, 12, 16, 24, 32, 48, 64, 96, 128). No GPU needed. */
int32_t piv_check_config(const PivConfigC* cfg);

/* ----------------------------------------------------------------------------- analyzer */
/* PivAnalyzer::new (multipass.rs:91-119). */
int32_t piv_analyzer_create(const PivConfigC* cfg, PivAnalyzer** out);
void piv_analyzer_destroy(PivAnalyzer* an);
/* Passes run per pair: windows + (final_iterations - 1) repeats of the last (multipass.rs:166-171). */
int32_t piv_num_passes(const PivAnalyzer* an);
/* PivAnalyzer::output_grid (multipass.rs:126-133). */
int32_t piv_output_grid(const PivAnalyzer* an, int64_t height, int64_t width, PivGridC* out);
/* Grid of pass `pass` for an image of the given size. */
int32_t piv_pass_grid(const PivAnalyzer* an, int64_t height, int64_t width, int32_t pass, PivGridC* out);
/* Use the caller's CUDA stream for all later work of this analyzer (NULL restores its own). */
int32_t piv_analyzer_set_stream(PivAnalyzer* an, void* stream);
/* Waits for the analyzer's stream. */
int32_t piv_analyzer_sync(PivAnalyzer* an);
/* Kernel launches issued by this analyzer since creation (launch accounting). */
int64_t piv_analyzer_launches(const PivAnalyzer* an);
/* Launch-geometry autotuning (no counterpart in the reference; the batching form of this
 * project): analyses the pair once while timing, for every pass, each launch variant of the
 * correlation kernel of that window size on the live data, and keeps the fastest per window
 * size for this analyzer. Variants of one size differ only in threads per block, register cap
 * and sampler, never in arithmetic: results are bit-identical whichever is chosen. Blocking. */
int32_t piv_analyzer_autotune(PivAnalyzer* an, const PivFrame* a, const PivFrame* b);
/* Launch variants of the FP32 kernel for `window` (uniform windows), and pinning one of them for
 * this analyzer (for tests and external tuning; results are identical whichever is used). */
int32_t piv_num_variants(int32_t window);
int32_t piv_analyzer_set_variant(PivAnalyzer* an, int32_t window, int32_t variant);
/* Name of the variant in use for `window` ("<n>/T<lanes per line>/G<groups>/B<min blocks>/<sampler>"). */
int32_t piv_analyzer_variant(const PivAnalyzer* an, int32_t window, char* name, int32_t capacity);
/* Stage timing (no counterpart in the reference, which has only wall-clock splits,
 * swift/Sources/PIVKit/Run.swift:189-196): when enabled, CUDA events bracket every correlation
 * kernel; piv_analyzer_profile waits for the stream and returns, for pass `pass`, the summed
 * kernel milliseconds and the number of launches timed since the last read (then resets). */
int32_t piv_analyzer_set_profiling(PivAnalyzer* an, int32_t enable);
int32_t piv_analyzer_profile(PivAnalyzer* an, int32_t pass, double* correlate_ms, int64_t* launches);

/* ----------------------------------------------------------------------------- frames */
/* Device-resident prepared frame of a fixed size (PreparedFrame, preprocess.rs:127-135). */
int32_t piv_frame_create(PivAnalyzer* an, int64_t height, int64_t width, PivFrame** out);
void piv_frame_destroy(PivFrame* f);
/* PreparedFrame::new (preprocess.rs:138-158) from HOST samples: raw is height*width samples of
 * `dtype` (u8 -> v/255, u16 -> v/65535 as decode.rs:227-234; f32 as is); background (nullable)
 * is a host f32 image. Copies to the device and prepares asynchronously on the analyzer stream
 * (raw and background must stay valid until piv_analyzer_sync or the next blocking call). */
int32_t piv_frame_prepare(PivAnalyzer* an, PivFrame* f, const void* raw, int32_t dtype, const PivPreprocessC* pre,
                          const float* background);
/* Same with DEVICE pointers (raw, background). */
int32_t piv_frame_prepare_device(PivAnalyzer* an, PivFrame* f, const void* raw_dev, int32_t dtype,
                                 const PivPreprocessC* pre, const float* background_dev);
/* Installs an already prepared image (host) and the background-subtracted intensity used by the
 * signal mask (host; NULL = the image itself), as PIVKit's makeFrame(image:stats:) does. */
int32_t piv_frame_set_prepared(PivAnalyzer* an, PivFrame* f, const float* image, const float* base);
/* Installs a frame prepared on the host by the reference itself: PreparedFrame's `image` (HOST,
 * height*width f32) and its `stats: IntegralImage` tables `sum` and `sumsq` (HOST, (height+1) x
 * (width+1) f64 each, row-major with stride width+1, as IntegralImage::new builds them,
 * preprocess.rs:76-103, 127-135). The tables are converted on the device to this library's exact
 * fixed-point form with integer operations only: entries finer than the table's quantum
 * (2^-(61 - e) for entries below 2^e) round to it, and window statistics are exact differences
 * of the entries where IntegralImage::rect rounds each f64 subtraction, so a signal-mask
 * decision can differ only for a window whose mean or standard deviation lies on the f32
 * rounding boundary of its threshold. PIV_ERR_ARGUMENT for a non-finite entry. Blocking. This
 * is the compatibility path for an unchanged PivAnalyzer::analyze(&PreparedFrame,
 * &PreparedFrame); piv_frame_prepare from raw samples is the fast path. */
int32_t piv_frame_set_prepared_tables(PivAnalyzer* an, PivFrame* f, const float* image, const double* sum,
                                      const double* sumsq);
/* Copies the prepared image back to the host. */
int32_t piv_frame_download(PivAnalyzer* an, const PivFrame* f, float* image);
/* Device address of the prepared image (height*width f32, row-major). */
const float* piv_frame_image_device(const PivFrame* f);

/* BackgroundEstimator (preprocess.rs:41-72) on DEVICE data: `count` frames of height*width
 * samples of `dtype`, mode 0 = per-pixel min, 1 = mean; output f32 image (device). */
int32_t piv_background_device(PivAnalyzer* an, const void* frames_dev, int32_t dtype, int64_t count,
                              int64_t height, int64_t width, int32_t mode, float* out_dev);

/* ----------------------------------------------------------------------------- analysis */
/* PivAnalyzer::analyze (multipass.rs:136-138): final field into HOST arrays of
 * output_grid().nx*ny elements, summary of the final pass. Blocking. */
int32_t piv_analyze(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, float* dx, float* dy, float* peak_ratio,
                    uint8_t* flags, PivSummaryC* summary);
/* Same into DEVICE arrays, asynchronous on the analyzer's stream. summary_dev (nullable) is a
 * device array of 5 uint64 counts (no_signal, low_ppr, median_outliers, out_of_range, replaced). */
int32_t piv_analyze_device(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, float* dx, float* dy,
                           float* peak_ratio, uint8_t* flags, uint64_t* summary_dev);

/* ----------------------------------------------------------------------------- batching form
 * No counterpart in the reference, which analyses one pair per call (multipass.rs:136) and
 * parallelises only inside it. PivAnalyzer::analyze for `count` pairs of equal-size frames in
 * one go: every stage of every pass is one kernel launch covering all pairs. Outputs are DEVICE
 * arrays, pair k's final field at offset k * nx*ny (output_grid); summaries_dev (nullable) gets
 * 8 uint64 per pair (the first 5 as in piv_analyze_device). Asynchronous. */
int32_t piv_analyze_batch_device(PivAnalyzer* an, const PivFrame* const* a, const PivFrame* const* b, int32_t count,
                                 float* dx, float* dy, float* peak_ratio, uint8_t* flags, uint64_t* summaries_dev);

/* A fixed batch for streams of frames, replayed from a CUDA graph. It owns a private copy of the
 * analyzer (configuration and tuned launch variants), a device slab for the raw samples of its
 * frames (sequential: pairs+1 frames, pair k = (frame k, frame k+1); otherwise 2*pairs frames,
 * pair k = (frame 2k, frame 2k+1)), the prepared frames, the workspace and an output slab. The
 * first run executes eagerly (allocating everything), then captures preparation of every frame
 * and every pass of every pair into one graph; later runs launch that graph. */
typedef struct PivBatch PivBatch;
int32_t piv_batch_create(const PivAnalyzer* an, int64_t height, int64_t width, int32_t pairs, int32_t sequential,
                         int32_t dtype, const PivPreprocessC* pre, PivBatch** out);
void piv_batch_destroy(PivBatch* batch);
/* Device slab of raw samples (frames back to back) and its size in bytes. */
void* piv_batch_input_device(PivBatch* batch);
int64_t piv_batch_input_bytes(const PivBatch* batch);
/* Runs the batch on its stream (asynchronous). */
int32_t piv_batch_run(PivBatch* batch);
/* The batch's CUDA stream (a cudaStream_t), for callers that order their own work after it. */
void* piv_batch_stream(PivBatch* batch);
/* Runs the batch's kernels on `stream` from now on (NULL: its own stream again). Batches that
 * share one stream replay their graphs one after another while their host copies (which go on
 * private copy streams, see piv_batch_submit_host) overlap. Not while a submission is pending.
 * The stream must stay valid while the batch runs on it; piv_batch_destroy itself needs no
 * stream (it waits for the device). */
int32_t piv_batch_set_stream(PivBatch* batch, void* stream);
/* Background image (DEVICE, height*width f32) subtracted from every frame of the batch, as
 * piv_frame_prepare's `background` (preprocess.rs:138-145); NULL = none. The next run records
 * the batch's graph again. The image must stay valid while the batch uses it. */
int32_t piv_batch_set_background(PivBatch* batch, const float* background_dev);
int32_t piv_batch_sync(PivBatch* batch);
/* Device output slabs: dx, dy, peak ratio (f32) and flags (u8), pairs*nx*ny each; 8 uint64
 * summary counters per pair; nx*ny is piv_output_grid's. */
int32_t piv_batch_outputs_device(PivBatch* batch, float** dx, float** dy, float** peak_ratio, uint8_t** flags,
                                 uint64_t** summaries);
/* Host convenience: copies `raw` (all frames, pinned memory recommended) into the slab, runs,
 * copies the results back; any output may be NULL. Blocking. */
int32_t piv_batch_run_host(PivBatch* batch, const void* raw, float* dx, float* dy, float* peak_ratio, uint8_t* flags,
                           PivSummaryC* summaries);
/* As piv_batch_run_host without waiting: the upload (on a private upload stream), the run (on the
 * batch's stream, after the upload) and the downloads (on a private download stream, after the
 * run) are queued and the call returns; piv_batch_wait_host waits and fills the summaries. Two
 * batches used in turn overlap one's copies with the other's kernels; sharing one stream
 * (piv_batch_set_stream) keeps their kernels from running at the same time.
 * `raw` and the outputs should be pinned and must stay valid until the wait returns; a batch
 * takes a new submission only after the previous one was waited for. */
int32_t piv_batch_submit_host(PivBatch* batch, const void* raw, float* dx, float* dy, float* peak_ratio, uint8_t* flags);
int32_t piv_batch_wait_host(PivBatch* batch, PivSummaryC* summaries);
/* Kernels executed per run (counted on the eager first run; the graph replays the same set). */
int64_t piv_batch_kernels(const PivBatch* batch);

/* Pipelined pairs (no counterpart in the reference, which analyses pairs one after another,
 * analyze.rs:441): pairs of HOST frames are submitted without waiting; `depth` slots, each with
 * its own prepared frames and workspace, let the uploads and downloads of one pair overlap the
 * kernels of the others. Uploads, frame preparation, analysis and downloads go on four streams
 * shared by the slots: the preparation of a pair overlaps the analysis of the one before it, and
 * the analyses of successive pairs run in submission order. Each result equals piv_analyze of
 * that pair. Host buffers should be
 * pinned (cudaHostAlloc) for the copies to be asynchronous, and must stay valid (outputs
 * untouched) until piv_pipeline_wait returns for that ticket. Submitting blocks only when the
 * next slot still holds an unfinished pair. */
typedef struct PivPipeline PivPipeline;
int32_t piv_pipeline_create(const PivAnalyzer* an, int64_t height, int64_t width, int32_t dtype,
                            const PivPreprocessC* pre, int32_t depth, PivPipeline** out);
void piv_pipeline_destroy(PivPipeline* pipeline);
/* Outputs as piv_analyze (any may be NULL); returns a ticket for piv_pipeline_wait. */
int32_t piv_pipeline_submit(PivPipeline* pipeline, const void* frame_a, const void* frame_b, float* dx, float* dy,
                            float* peak_ratio, uint8_t* flags, uint64_t* ticket);
/* Waits for the pair of `ticket`; every ticket is waited for exactly once. */
int32_t piv_pipeline_wait(PivPipeline* pipeline, uint64_t ticket, PivSummaryC* summary);
/* Background image (DEVICE, height*width f32, e.g. from piv_background_device) subtracted from
 * every frame submitted from now on, as piv_frame_prepare's `background` (preprocess.rs:138-145:
 * base = max(raw - background, 0)); NULL = none. The reference estimates one background per run
 * and uses it for every frame. Not while pairs are in flight; the image must outlive them. */
int32_t piv_pipeline_set_background(PivPipeline* pipeline, const float* background_dev);

/* ----------------------------------------------------------------------------- serving form
 * No counterpart in the reference. A request loop on one GPU with continuous batching: frame
 * pairs of any size with their own PivConfig are submitted at any time; a scheduler thread
 * admits them (FIFO) while the in-flight count and a device-memory budget allow, keeps each
 * request's state (prepared frames, per-pass origins and predictor fields) on the device, and
 * advances ALL admitted requests by one pass per step: one placement launch for all of them,
 * one fused correlation launch for all FP32 windows of 8 to 64 px (piv_server_set_fused), one
 * validation chain. A request joins at the next
 * step boundary and leaves when its last pass is done, so requests that arrive while others run
 * share kernel launches with them. Window pairs are independent inside a launch, so each
 * result is bit-identical to PivAnalyzer::analyze of that pair alone. */
typedef struct PivServer PivServer;
typedef struct {
    int32_t device;              /* CUDA device ordinal (-1: current) */
    int64_t memory_budget_bytes; /* device memory admitted requests may hold together */
    int32_t max_in_flight;       /* admitted requests at most */
} PivServerConfigC;
typedef struct {
    PivConfigC config;           /* window schedule, overlap, mask, validation of this request */
    PivPreprocessC preprocess;
    int32_t dtype;               /* PIV_DTYPE_* of the samples */
    int64_t height, width;
    const void* frame_a;         /* HOST samples (pinned memory recommended); valid until done */
    const void* frame_b;
    float* dx;                   /* HOST outputs of output_grid's nx*ny elements; valid until done
                                  * (pageable memory is staged through the server's pinned blocks) */
    float* dy;
    float* peak_ratio;
    uint8_t* flags;
} PivRequestC;
typedef struct {
    int64_t submitted, admitted, completed, failed, queued, in_flight;
    int64_t memory_in_use_bytes, steps, kernel_launches;
    int64_t cancelled;          /* requests that ended cancelled */
    int64_t deferred;           /* admissions put back after a failed allocation */
    int64_t last_step_requests; /* requests advanced by the most recent step */
    int64_t max_step_requests;  /* most requests advanced by one step */
} PivServerStatsC;
int32_t piv_server_create(const PivServerConfigC* cfg, PivServer** out);
/* Finishes the admitted and queued requests, then stops the scheduler and frees the server. */
void piv_server_destroy(PivServer* server);
/* Queues a request; fails at once, queuing nothing, for a malformed request: an invalid config
 * (odd or too small window, overlap outside [0, 1): PIV_ERR_CONFIG, as multipass.rs:91-119), a
 * window larger than the image (PIV_ERR_IMAGE_TOO_SMALL, as grid.rs:27-33), an unknown dtype or
 * NULL frames (PIV_ERR_ARGUMENT), or a request larger than the budget (PIV_ERR_UNSUPPORTED). */
int32_t piv_server_submit(PivServer* server, const PivRequestC* request, uint64_t* id);
/* Blocks until request `id` is done; fills its summary and its latency (submit to results in
 * host memory, milliseconds). Returns the request's own status: PIV_OK, PIV_ERR_CANCELLED, or
 * the error that ended it (e.g. PIV_ERR_CUDA when its device memory could not be allocated
 * while nothing else was in flight). Each id may be waited once. */
int32_t piv_server_wait(PivServer* server, uint64_t id, PivSummaryC* summary, double* latency_ms);
/* piv_server_wait with a bound: PIV_ERR_TIMEOUT when the request is not done within timeout_ms
 * (it stays pending and may be waited again). */
int32_t piv_server_wait_timeout(PivServer* server, uint64_t id, double timeout_ms, PivSummaryC* summary,
                                double* latency_ms);
/* Cancels request `id`. A queued request is dropped at once; an admitted one stops at the next
 * step boundary, its memory given back once the passes already queued for it have run. Either
 * way its wait returns PIV_ERR_CANCELLED and its outputs are not written. A request whose last
 * pass was already launched finishes normally. PIV_ERR_ARGUMENT for an unknown id. */
int32_t piv_server_cancel(PivServer* server, uint64_t id);
/* Host-side fault injection: the next `count` admissions fail as an out-of-memory allocation
 * would, without calling the allocator. With other requests in flight the admission is put back
 * and retried after one of them finishes (stats.deferred); with none, the request fails. */
int32_t piv_server_fail_next_allocations(PivServer* server, int32_t count);
/* Correlation launches per step: with fused != 0 (the default) the FP32 windows of 8, 16, 32 and
 * 64 px of all requests, uniform or deformed, run in ONE fused launch (each CTA runs the
 * per-size kernel body of its window size, so results are bit-identical); other sizes and the
 * tensor-core kinds take one launch per (size, kind). fused == 0: one launch per (size, kind). */
int32_t piv_server_set_fused(PivServer* server, int32_t fused);
/* Manual stepping (testing and external pacing): with manual != 0 the scheduler admits requests
 * and launches steps only when piv_server_advance grants them; 0 returns to free running. */
int32_t piv_server_set_manual(PivServer* server, int32_t manual);
/* Grants `steps` steps (admission, then one pass of every admitted request) and blocks until the
 * scheduler has taken them (a step with nothing to launch counts), or PIV_ERR_TIMEOUT after
 * timeout_ms (< 0: no bound); PIV_ERR_ARGUMENT if manual stepping ends meanwhile (set_manual(0)
 * from another thread, or destroy). */
int32_t piv_server_advance(PivServer* server, int32_t steps, double timeout_ms);
int32_t piv_server_stats(PivServer* server, PivServerStatsC* stats);
/* No counterpart in the reference (the serving form's memory). Each server allocates its
 * requests from a memory pool of its own, which keeps freed memory for later requests. The
 * first admissions that reach a new peak of memory in flight make the pool map more device
 * memory, and the driver call that does so can block the scheduler for hundreds of milliseconds
 * (measured: one 54 MB admission, 585 ms), stalling every request in flight. This call grows the
 * pool ahead of time by `bytes` (allocated and freed again in chunks of at most 1 GiB, blocking),
 * so later admissions up to that much memory in flight are served from memory the pool already
 * holds. With bytes > 0 it also pins the server's first host staging blocks for result downloads
 * (8 MiB for each download size up to 1 MiB). The memory stays reserved to the server until
 * piv_server_destroy; it does not count against memory_budget_bytes. bytes == 0 only reports. *reserved_bytes (may be NULL): the
 * memory the pool holds after the call. PIV_ERR_CUDA if the device runs out of memory part way
 * (what was reserved stays reserved). */
int32_t piv_server_reserve(PivServer* server, int64_t bytes, int64_t* reserved_bytes);

/* PivAnalyzer::analyze_traced (multipass.rs:142-150, PassTrace :72-81): HOST arrays holding
 * every pass back to back (pass 0 cells, then pass 1 ...; piv_pass_grid gives each count):
 * origins 4 floats per cell [ax, ay, bx, by]; raw_* before validation; the rest after.
 * Any pointer may be NULL. Blocking. */
typedef struct {
    float* origins;
    float* raw_dx;
    float* raw_dy;
    float* raw_peak_ratio;
    uint8_t* raw_flags;
    float* dx;
    float* dy;
    float* peak_ratio;
    uint8_t* flags;
} PivTraceC;
int32_t piv_analyze_traced(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, PivTraceC* trace,
                           PivSummaryC* summary);

/* ----------------------------------------------------------------------------- stage hooks
 * Single stages on HOST arrays, for stage-by-stage parity (the reference's own split:
 * multipass.rs:194-259 pass, validate.rs:51 validate; PIVKit's placeOnGPU/validateOnGPU,
 * PIVAnalyzer.swift:318-348). Blocking. */
/* Window origins of one pass from an optional predictor field (NULL = first pass). */
int32_t piv_place_windows(PivAnalyzer* an, int64_t height, int64_t width, const PivGridC* grid,
                          const PivGridC* pred_grid, const float* pred_dx, const float* pred_dy, float* origins);
/* Correlates given origins (4 floats per cell) of frames a, b with window `window`, applying
 * the analyzer's signal mask: raw dx, dy, peak ratio and flags (0 or NO_SIGNAL). */
int32_t piv_correlate_origins(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, int64_t window,
                              const float* origins, int64_t ncells, float* dx, float* dy, float* peak_ratio,
                              uint8_t* flags);
/* Window deformation (no counterpart in the reference, whose windows only shift,
 * multipass.rs:224-231; deformation is listed as deferred in docs/phase1-plan.md:104,248).
 * A deformed window's base position (x0, y0) is its zero-shift origin under the placement clamp
 * (multipass.rs:207-208): the grid origin clamped to [0, W - n - 1] x [0, H - n - 1].
 * piv_place_windows_deform: as piv_place_windows, plus the predictor (field.rs:56-81 sampling) at
 * the four corner pixels of each window's base position (x0, y0), (x0+n-1, y0), (x0, y0+n-1),
 * (x0+n-1, y0+n-1): corners[8k..8k+7] = dx00, dy00, dx10, dy10, dx01, dy01, dx11, dy11 (zero
 * without a predictor).
 * piv_correlate_deform: correlates the deformed windows of `grid`: pixel (r, c) of the window at
 * base position (x0, y0) is displaced by D, the bilinear blend of the corners at u = c/(n-1),
 * v = r/(n-1); window A samples frame A at (x0+c, y0+r) - D/2 and window B frame B at + D/2
 * (bilinear, clamped to the image). The signal mask uses `origins` (4 floats per cell, as
 * piv_place_windows returns them); the vector is D(centre) + peak. */
int32_t piv_place_windows_deform(PivAnalyzer* an, int64_t height, int64_t width, const PivGridC* grid,
                                 const PivGridC* pred_grid, const float* pred_dx, const float* pred_dy, float* origins,
                                 float* corners);
int32_t piv_correlate_deform(PivAnalyzer* an, const PivFrame* a, const PivFrame* b, const PivGridC* grid,
                             const float* origins, const float* corners, float* dx, float* dy, float* peak_ratio,
                             uint8_t* flags);
/* validate (validate.rs:51-130) of a raw field with the analyzer's thresholds and
 * max_displacement = windows[0] / 2. Outputs validated dx, dy, flags. */
int32_t piv_validate_field(PivAnalyzer* an, int64_t ny, int64_t nx, const float* dx, const float* dy,
                           const float* peak_ratio, const uint8_t* flags, float* out_dx, float* out_dy,
                           uint8_t* out_flags, PivSummaryC* summary);

/* ----------------------------------------------------------------------------- post-processing
 * The path's next components, on DEVICE arrays of validated fields (row-major [ny, nx] per pair,
 * pairs stacked [nt, ny, nx]); work is queued on `stream` (NULL = default stream).
 *
 * piv_flow_stats_device: FlowStats of one pair (flowstats.rs:67-101) in px/s units from
 * displacements in px (flow.rs:20-36: u = dx * f32(1/dt_s)), over the usable vectors (finite,
 * accepted or REPLACED: flow.rs:13-17); `step` is the grid spacing in px. `vorticity` (nullable,
 * device, [ny, nx]) receives the vorticity field (flowstats.rs:44-64). Blocking. */
typedef struct {
    float vorticity_mean, vorticity_abs_mean, ke_mean, ke_sum, coverage;
    int64_t n_usable, n_vorticity;
} PivFlowStatsC;
int32_t piv_flow_stats_device(int64_t ny, int64_t nx, int64_t step, double dt_s, const float* dx, const float* dy,
                              const uint8_t* flags, float* vorticity, PivFlowStatsC* stats, void* stream);
/* temporal (smooth.rs:44-128): moving mean (median = 0) or median over `window` (odd, <= 63)
 * consecutive pairs; `usable` marks contributing raw vectors, `gate` where outputs are wanted;
 * outputs with fewer than min_support contributions are NaN; `leave_out` lists time offsets to
 * skip (each non-zero one replaced by the next further out). Asynchronous. */
int32_t piv_temporal_smooth_device(int64_t nt, int64_t ny, int64_t nx, const float* dx, const float* dy,
                                   const uint8_t* usable, const uint8_t* gate, int32_t median, int32_t window,
                                   int32_t min_support, const int32_t* leave_out, int32_t n_leave_out, float* out_dx,
                                   float* out_dy, uint16_t* support, void* stream);
/* spatial (smooth.rs:130-207): Gaussian normalized convolution of each pair's field, sigma in
 * grid cells (<= 12), outputs need min_weight of the kernel's weight; leave_out < 0: none, else
 * the Chebyshev radius left out. Asynchronous. */
int32_t piv_spatial_smooth_device(int64_t nt, int64_t ny, int64_t nx, const float* dx, const float* dy,
                                  const uint8_t* gate, float sigma, float min_weight, int32_t leave_out, float* out_dx,
                                  float* out_dy, uint16_t* support, void* stream);

/* Diagnostics (no counterpart in the reference): D (128 x n) = A (128 x k) * B (n x k)^T on the
 * tensor cores of `device` with BF16 operands (inputs rounded to BF16) and FP32 accumulation, A
 * stored K-major (a_mn = 0) or MN-major (a_mn = 1) as the tensor-core correlation stores its
 * operands. a, b, d are row-major DEVICE arrays; n, k multiples of 16 in [16, 256]. Blocking. */
int32_t piv_tc_selftest(int32_t device, int32_t a_mn, int32_t n, int32_t k, const float* a, const float* b, float* d);
/* Diagnostics (no counterpart in the reference): runs the tensor-core kernel's bounded mbarrier
 * wait on a barrier that nothing completes, with 2^log2_iters try_wait rounds (18 is the kernel's
 * own bound, about a second; at most 18). The wait gives up, and *timed_out is set to 1; *ms is the probe
 * kernel's duration. Uses a private status word: the device's tensor-core error status read by
 * piv_analyze is not touched. Blocking. */
int32_t piv_tc_wait_probe(int32_t device, int32_t log2_iters, int32_t* timed_out, float* ms);

/* ----------------------------------------------------------------------------- no allocation
 * No counterpart in the reference. Validation of a raw field (the same rules as
 * piv_validate_field, with the thresholds and max_displacement passed in) that allocates no
 * device memory, for callers that cannot call cudaMalloc once running: deadline-bound
 * acquisition loops (cudaFree waits for the whole device) and processes whose device memory is
 * already reserved by another allocator. All pointers are DEVICE pointers owned by the caller;
 * work is queued on `stream` (NULL = the default stream) and the call returns without waiting.
 * Scratch lives in a fixed device array inside the library of 2 x 2,097,152 bytes, held by every
 * GPU that loads the library until exit; fields above 2,097,152 cells are rejected
 * (PIV_ERR_UNSUPPORTED). The first call on a device looks up that array's address, so make it
 * before any stream capture; the address is kept until exit, so do not call this on a device
 * after cudaDeviceReset. All calls share the array: calls whose work overlaps on the GPU race.
 * Outputs must not overlap any input or each other (the median test reads neighbours while
 * others are written): such calls are rejected (PIV_ERR_ARGUMENT). */
int32_t piv_validate_field_noalloc(int64_t ny, int64_t nx, const float* dx, const float* dy, const float* peak_ratio,
                                   const uint8_t* flags, float max_displacement, float ppr_threshold,
                                   float median_threshold, float median_eps, int32_t replace, float* out_dx,
                                   float* out_dy, uint8_t* out_flags, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PIV_B200_H */
