/* A plain C99 program that drives libpivb200.so through include/piv_b200.h, as a Rust or C
 * host would bind it (no Python, no ctypes). Two modes:
 *
 *   piv_c_driver host
 *       Calls that need no GPU: ABI version, Grid::new (grid.rs:20-44) on the reference's own
 *       test cases (grid.rs:81-108), PivAnalyzer::new's config errors (multipass.rs:91-119), status codes and
 *       messages. Prints "host ok" and exits 0, or names the failed check and exits 1.
 *
 *   piv_c_driver analyze <request.bin> <result.bin>
 *       One PivAnalyzer::analyze (multipass.rs:136-138) of a pair of frames prepared on the host.
 *       request.bin (little-endian): int64 H, W; int32 n_windows; int32 windows[n_windows];
 *       float overlap; int32 final_iterations; float min_mean, min_std; int32 has_tables;
 *       float image_a[H*W], image_b[H*W]; then, if has_tables, the IntegralImage tables of both
 *       frames (preprocess.rs:84-103): double sum_a[(H+1)*(W+1)], sumsq_a[...], sum_b[...],
 *       sumsq_b[...]; else float base_a[H*W], base_b[H*W] (the mask's intensity).
 *       result.bin: int64 ny, nx; float dx[ny*nx], dy[...], peak_ratio[...]; uint8 flags[...];
 *       int64 summary[5] (ValidationSummary, validate.rs:39-46).
 *       Exits with the library's status code (0 on success) after printing piv_last_error().
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "piv_b200.h"

static int failures = 0;

#define CHECK(cond, ...)                           \
    do {                                           \
        if (!(cond)) {                             \
            fprintf(stderr, "check failed: ");     \
            fprintf(stderr, __VA_ARGS__);          \
            fprintf(stderr, "\n");                 \
            ++failures;                            \
        }                                          \
    } while (0)

static PivConfigC default_config(const int32_t* windows, int32_t n) {
    PivConfigC c;
    memset(&c, 0, sizeof(c));
    c.windows = windows;
    c.n_windows = n;
    c.overlap = 0.5f;
    c.final_iterations = 2;
    c.min_mean = 0.0f;
    c.min_std = 0.0f;
    c.ppr_threshold = 1.3f;
    c.median_threshold = 2.0f;
    c.median_eps = 0.1f;
    c.replace = 1;
    c.device = -1;
    c.deform = 0;
    c.precision = PIV_PRECISION_FP32;
    return c;
}

static int run_host(void) {
    CHECK(piv_abi_version() == PIV_B200_ABI_VERSION, "abi version %d", piv_abi_version());
    /* grid.rs:81-108: the reference's own grid tests */
    PivGridC g;
    CHECK(piv_grid(1080, 1920, 32, 0.5f, &g) == PIV_OK, "grid 1080x1920/32/0.5");
    CHECK(g.step == 16 && g.nx == 119 && g.ny == 66 && g.x0 == 0 && g.y0 == 4, "full-HD grid values");
    CHECK(piv_grid(64, 64, 32, 0.0f, &g) == PIV_OK, "grid 64x64/32/0");
    CHECK(g.nx == 2 && g.ny == 2 && g.step == 32 && g.x0 == 0, "exact-fit grid values");
    CHECK(piv_grid(16, 64, 32, 0.5f, &g) == PIV_ERR_IMAGE_TOO_SMALL, "window taller than the image");
    CHECK(strlen(piv_last_error()) > 0, "message after a failure");
    CHECK(piv_grid(64, 64, 32, 1.0f, &g) == PIV_ERR_CONFIG, "overlap 1");
    CHECK(piv_grid(64, 64, 32, -0.1f, &g) == PIV_ERR_CONFIG, "overlap -0.1");
    /* the benchmark's final pass: 4096 x 4096, 16 px at 75 % */
    CHECK(piv_grid(4096, 4096, 16, 0.75f, &g) == PIV_OK && g.nx == 1021 && g.ny == 1021, "grid 4096/16/0.75");
    /* multipass.rs:91-119 */
    int32_t ok_w[2] = {64, 32}, odd_w[1] = {33}, small_w[1] = {6}, big_w[1] = {256};
    PivConfigC c = default_config(ok_w, 2);
    CHECK(piv_check_config(&c) == PIV_OK, "default config");
    c = default_config(odd_w, 1);
    CHECK(piv_check_config(&c) == PIV_ERR_CONFIG, "odd window");
    c = default_config(small_w, 1);
    CHECK(piv_check_config(&c) == PIV_ERR_CONFIG, "window below 8");
    c = default_config(ok_w, 0);
    CHECK(piv_check_config(&c) == PIV_ERR_CONFIG, "no windows");
    c = default_config(ok_w, 2);
    c.overlap = -0.1f;
    CHECK(piv_check_config(&c) == PIV_ERR_CONFIG, "negative overlap");
    c = default_config(ok_w, 2);
    c.final_iterations = 0;
    CHECK(piv_check_config(&c) == PIV_ERR_CONFIG, "final_iterations 0");
    c = default_config(big_w, 1);
    CHECK(piv_check_config(&c) == PIV_ERR_UNSUPPORTED, "window 256 is valid for the reference, not on the GPU");
    CHECK(piv_check_config(NULL) == PIV_ERR_ARGUMENT, "null config");
    if (failures) return 1;
    printf("host ok\n");
    return 0;
}

static void* read_exact(FILE* f, size_t bytes) {
    void* p = malloc(bytes ? bytes : 1);
    if (!p || fread(p, 1, bytes, f) != bytes) {
        free(p);
        return NULL;
    }
    return p;
}

static int run_analyze(const char* in_path, const char* out_path) {
    FILE* f = fopen(in_path, "rb");
    if (!f) {
        fprintf(stderr, "cannot open %s\n", in_path);
        return PIV_ERR_ARGUMENT;
    }
    int64_t hw[2];
    int32_t nwin = 0;
    if (fread(hw, sizeof(int64_t), 2, f) != 2 || fread(&nwin, sizeof(int32_t), 1, f) != 1 || nwin <= 0 || nwin > 16) {
        fclose(f);
        return PIV_ERR_ARGUMENT;
    }
    const int64_t H = hw[0], W = hw[1];
    int32_t windows[16];
    float overlap = 0.0f, min_mean = 0.0f, min_std = 0.0f;
    int32_t final_iterations = 0, has_tables = 0;
    if (fread(windows, sizeof(int32_t), (size_t)nwin, f) != (size_t)nwin || fread(&overlap, 4, 1, f) != 1 ||
        fread(&final_iterations, 4, 1, f) != 1 || fread(&min_mean, 4, 1, f) != 1 || fread(&min_std, 4, 1, f) != 1 ||
        fread(&has_tables, 4, 1, f) != 1) {
        fclose(f);
        return PIV_ERR_ARGUMENT;
    }
    const size_t n = (size_t)H * (size_t)W, nt = (size_t)(H + 1) * (size_t)(W + 1);
    float* img[2] = {read_exact(f, 4 * n), read_exact(f, 4 * n)};
    void* extra[4] = {NULL, NULL, NULL, NULL};
    if (has_tables)
        for (int k = 0; k < 4; ++k) extra[k] = read_exact(f, 8 * nt);
    else
        for (int k = 0; k < 2; ++k) extra[k] = read_exact(f, 4 * n);
    fclose(f);
    if (!img[0] || !img[1] || !extra[0] || !extra[1] || (has_tables && (!extra[2] || !extra[3]))) return PIV_ERR_ARGUMENT;

    PivConfigC cfg = default_config(windows, nwin);
    cfg.overlap = overlap;
    cfg.final_iterations = final_iterations;
    cfg.min_mean = min_mean;
    cfg.min_std = min_std;
    PivAnalyzer* an = NULL;
    PivFrame* fr[2] = {NULL, NULL};
    int32_t st = piv_analyzer_create(&cfg, &an);
    for (int k = 0; st == PIV_OK && k < 2; ++k) st = piv_frame_create(an, H, W, &fr[k]);
    for (int k = 0; st == PIV_OK && k < 2; ++k)
        st = has_tables ? piv_frame_set_prepared_tables(an, fr[k], img[k], (const double*)extra[2 * k],
                                                        (const double*)extra[2 * k + 1])
                        : piv_frame_set_prepared(an, fr[k], img[k], (const float*)extra[k]);
    PivGridC g;
    memset(&g, 0, sizeof(g));
    if (st == PIV_OK) st = piv_output_grid(an, H, W, &g);
    const size_t cells = (size_t)(g.nx * g.ny);
    float* dx = malloc(4 * (cells ? cells : 1));
    float* dy = malloc(4 * (cells ? cells : 1));
    float* ppr = malloc(4 * (cells ? cells : 1));
    uint8_t* flags = malloc(cells ? cells : 1);
    PivSummaryC sum;
    memset(&sum, 0, sizeof(sum));
    if (st == PIV_OK) st = piv_analyze(an, fr[0], fr[1], dx, dy, ppr, flags, &sum);
    if (st == PIV_OK) {
        FILE* o = fopen(out_path, "wb");
        int64_t shape[2] = {g.ny, g.nx};
        int64_t s5[5] = {sum.no_signal, sum.low_ppr, sum.median_outliers, sum.out_of_range, sum.replaced};
        if (!o || fwrite(shape, 8, 2, o) != 2 || fwrite(dx, 4, cells, o) != cells || fwrite(dy, 4, cells, o) != cells ||
            fwrite(ppr, 4, cells, o) != cells || fwrite(flags, 1, cells, o) != cells || fwrite(s5, 8, 5, o) != 5)
            st = PIV_ERR_ARGUMENT;
        if (o) fclose(o);
    } else {
        fprintf(stderr, "status %d: %s\n", (int)st, piv_last_error());
    }
    for (int k = 0; k < 2; ++k) piv_frame_destroy(fr[k]);
    piv_analyzer_destroy(an);
    free(dx);
    free(dy);
    free(ppr);
    free(flags);
    for (int k = 0; k < 2; ++k) free(img[k]);
    for (int k = 0; k < 4; ++k) free(extra[k]);
    if (st == PIV_OK) printf("analyze ok: %lld x %lld vectors\n", (long long)g.ny, (long long)g.nx);
    return st;
}

int main(int argc, char** argv) {
    if (argc >= 2 && strcmp(argv[1], "host") == 0) return run_host();
    if (argc >= 4 && strcmp(argv[1], "analyze") == 0) return run_analyze(argv[2], argv[3]);
    fprintf(stderr, "usage: %s host | analyze <request.bin> <result.bin>\n", argv[0]);
    return 2;
}
