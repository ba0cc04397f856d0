// Window placement, signal mask, validation and summary kernels.
//
// These stages are bit-exact against the reference: every f32 operation is written with the
// round-to-nearest intrinsics in the reference's order (Rust never contracts into FMA), and the
// translation unit is additionally compiled with --fmad=false.
//   placement:  PivAnalyzer::pass (multipass.rs:204-231) with VectorField::sample (field.rs:56-81)
//   mask:       has_signal (multipass.rs:233-241) over IntegralImage::stats (preprocess.rs:114-125)
//   validation: validate (validate.rs:51-130), collect_neighbours / residual / median (:133-170)
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace pivb200 {

__device__ __forceinline__ float grid_center(int origin0, int i, int step, int window) {
    // grid.rs:60-66: (origin0 + i*step) as f32 + (window as f32 - 1) / 2
    return __fadd_rn((float)(origin0 + i * step), __fdiv_rn(__fsub_rn((float)window, 1.0f), 2.0f));
}

// VectorField::sample (field.rs:56-81).
__device__ float2 sample_predictor(const float* __restrict__ dx, const float* __restrict__ dy, const GridP& g, float x,
                                   float y) {
    const float fx = rclamp(__fdiv_rn(__fsub_rn(x, grid_center(g.x0, 0, g.step, g.window)), (float)g.step), 0.0f,
                            (float)(g.nx - 1));
    const float fy = rclamp(__fdiv_rn(__fsub_rn(y, grid_center(g.y0, 0, g.step, g.window)), (float)g.step), 0.0f,
                            (float)(g.ny - 1));
    const int ix = (int)floorf(fx), iy = (int)floorf(fy);
    const float tx = __fsub_rn(fx, (float)ix), ty = __fsub_rn(fy, (float)iy);
    const int ix1 = min(ix + 1, g.nx - 1), iy1 = min(iy + 1, g.ny - 1);
    const int rr[4] = {iy, iy, iy1, iy1};
    const int cc[4] = {ix, ix1, ix, ix1};
    const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty);
    const float ww[4] = {__fmul_rn(ux, uy), __fmul_rn(tx, uy), __fmul_rn(ux, ty), __fmul_rn(tx, ty)};
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float u = dx[rr[j] * g.nx + cc[j]], v = dy[rr[j] * g.nx + cc[j]];
        if (ww[j] > 0.0f && isfinite(u) && isfinite(v)) {
            a0 = __fadd_rn(a0, __fmul_rn(ww[j], u));
            a1 = __fadd_rn(a1, __fmul_rn(ww[j], v));
            a2 = __fadd_rn(a2, ww[j]);
        }
    }
    if (a2 > 0.0f) return make_float2(__fdiv_rn(a0, a2), __fdiv_rn(a1, a2));
    return make_float2(0.0f, 0.0f);
}

// The `place` closure (multipass.rs:224-231): returns (a0, a0 + shift).
__device__ __forceinline__ float2 place1(int origin, float shift, float mx) {
    const float s = rclamp(shift, -mx, mx);
    const float a0 = rclamp(__fsub_rn((float)origin, __fdiv_rn(s, 2.0f)), fmaxf(-s, 0.0f), fminf(__fsub_rn(mx, s), mx));
    return make_float2(a0, __fadd_rn(a0, s));
}

__device__ __forceinline__ long long rect(const long long* t, int stride, int x0, int y0, int x1, int y1) {
    return t[(size_t)y1 * stride + x1] - t[(size_t)y0 * stride + x1] - t[(size_t)y1 * stride + x0] + t[(size_t)y0 * stride + x0];
}

// has_signal (multipass.rs:233-241): stats of the n x n box at the rounded origin.
__device__ bool has_signal(const StatsView& s, float x, float y, int n, float min_mean, float min_std) {
    int bx = (int)roundf(x), by = (int)roundf(y);  // f32::round: half away from zero
    bx = min(max(bx, 0), s.W - n);
    by = min(max(by, 0), s.H - n);
    const int stride = s.W + 1;
    const FixScale fs{s.scales[0], s.scales[1]};
    float mean, sd;
    fix_stats(rect(s.sum, stride, bx, by, bx + n, by + n), rect(s.sumsq, stride, bx, by, bx + n, by + n), fs,
              (float)(n * n), &mean, &sd);
    return mean >= min_mean && sd >= min_std;
}

__global__ void place_kernel(const PlaceParams p) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = p.grid.nx * p.grid.ny;
    if (k >= cells) return;
    const int ix = k % p.grid.nx, iy = k / p.grid.nx;
    const int n = p.grid.window;
    // max = (w - n).saturating_sub(1) (multipass.rs:207-208)
    const float max_x = (float)max(p.W - n - 1, 0), max_y = (float)max(p.H - n - 1, 0);
    float2 shift = make_float2(0.0f, 0.0f);
    if (p.has_pred)
        shift = sample_predictor(p.pdx, p.pdy, p.pgrid, grid_center(p.grid.x0, ix, p.grid.step, n),
                                 grid_center(p.grid.y0, iy, p.grid.step, n));
    const float2 xs = place1(p.grid.x0 + ix * p.grid.step, shift.x, max_x);
    const float2 ys = place1(p.grid.y0 + iy * p.grid.step, shift.y, max_y);
    const float4 o = make_float4(xs.x, ys.x, xs.y, ys.y);
    p.origins[k] = o;
    uint8_t st = 1;
    if (p.use_stats)
        st = has_signal(p.sa, o.x, o.y, n, p.min_mean, p.min_std) && has_signal(p.sb, o.z, o.w, n, p.min_mean, p.min_std);
    p.status[k] = st;
}

__global__ void mask_kernel(const PlaceParams p, const float4* origins, int ncells) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ncells) return;
    const float4 o = origins[k];
    const int n = p.grid.window;
    uint8_t st = 1;
    if (p.use_stats)
        st = has_signal(p.sa, o.x, o.y, n, p.min_mean, p.min_std) && has_signal(p.sb, o.z, o.w, n, p.min_mean, p.min_std);
    p.status[k] = st;
}

cudaError_t launch_place(const PlaceParams& p, cudaStream_t s) {
    const int cells = p.grid.nx * p.grid.ny;
    if (cells <= 0) return cudaSuccess;
    place_kernel<<<(cells + 255) / 256, 256, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_mask(const PlaceParams& p, const float4* origins, int ncells, cudaStream_t s) {
    if (ncells <= 0) return cudaSuccess;
    mask_kernel<<<(ncells + 255) / 256, 256, 0, s>>>(p, origins, ncells);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Validation
// ---------------------------------------------------------------------------------------------
// Sorts v[0..n) ascending (insertion sort; usable neighbours are never NaN, so this orders them
// as f32::total_cmp does) and returns the median, the mean of the middle two when n is even.
__device__ float median_sorted(float* v, int n) {
    for (int i = 1; i < n; ++i) {
        const float x = v[i];
        int j = i;
        while (j > 0 && v[j - 1] > x) {
            v[j] = v[j - 1];
            --j;
        }
        v[j] = x;
    }
    if (n % 2 == 1) return v[n / 2];
    return __fmul_rn(0.5f, __fadd_rn(v[n / 2 - 1], v[n / 2]));
}

__device__ int collect_neighbours(const float* dx, const float* dy, const uint8_t* snap, int nx, int ny, int ix, int iy,
                                  int radius, float* nu, float* nv) {
    int c = 0;
    const int y0 = max(iy - radius, 0), y1 = min(iy + radius, ny - 1);
    const int x0 = max(ix - radius, 0), x1 = min(ix + radius, nx - 1);
    for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x)
            if (!(x == ix && y == iy) && (snap[y * nx + x] & F_INVALID) == 0) {
                nu[c] = dx[y * nx + x];
                nv[c] = dy[y * nx + x];
                ++c;
            }
    return c;
}

__device__ float residual(float value, float* nb, int n, float eps) {
    const float med = median_sorted(nb, n);
    float dev[8];
    for (int i = 0; i < n; ++i) dev[i] = fabsf(__fsub_rn(nb[i], med));
    return __fdiv_rn(fabsf(__fsub_rn(value, med)), __fadd_rn(median_sorted(dev, n), eps));
}

// Per-vector tests (validate.rs:59-78).
__global__ void validate_vector_kernel(const ValidateParams p) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.nx * p.ny) return;
    uint8_t f = p.flags0[k];
    if (!(f & F_NO_SIGNAL)) {
        if (hypotf(p.dx[k], p.dy[k]) > p.max_displacement) f |= F_OUT_OF_RANGE;
        if (p.ppr[k] < p.ppr_threshold) f |= F_LOW_PPR;
    }
    p.flags1[k] = f;
}

// Normalized median test on a snapshot of the flags (validate.rs:80-100).
__global__ void validate_median_kernel(const ValidateParams p) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.nx * p.ny) return;
    const int ix = k % p.nx, iy = k / p.nx;
    uint8_t f = p.flags1[k];
    if ((f & F_INVALID) == 0) {
        float nu[8], nv[8];
        const int c = collect_neighbours(p.dx, p.dy, p.flags1, p.nx, p.ny, ix, iy, 1, nu, nv);
        if (c >= 2) {
            const float ru = residual(p.dx[k], nu, c, p.median_eps);
            const float rv = residual(p.dy[k], nv, c, p.median_eps);
            if (__fsqrt_rn(__fadd_rn(__fmul_rn(ru, ru), __fmul_rn(rv, rv))) > p.median_threshold) f |= F_MEDIAN_OUTLIER;
        }
    }
    p.flags2[k] = f;
}

// Replacement by the median of usable neighbours at radius 1, then 2 (validate.rs:102-128).
__global__ void validate_replace_kernel(const ValidateParams p) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.nx * p.ny) return;
    const int ix = k % p.nx, iy = k / p.nx;
    uint8_t f = p.flags2[k];
    float u = p.dx[k], v = p.dy[k];
    if (p.replace && (f & F_NO_SIGNAL) == 0 && (f & F_INVALID) != 0) {
        float nu[24], nv[24];
        bool done = false;
        for (int radius = 1; radius <= 2 && !done; ++radius) {
            const int c = collect_neighbours(p.dx, p.dy, p.flags2, p.nx, p.ny, ix, iy, radius, nu, nv);
            if (c > 0) {
                u = median_sorted(nu, c);
                v = median_sorted(nv, c);
                f |= F_REPLACED;
                done = true;
            }
        }
        if (!done) {
            u = NAN;
            v = NAN;
        }
    }
    p.out_dx[k] = u;
    p.out_dy[k] = v;
    p.out_flags[k] = f;
}

cudaError_t launch_validate(const ValidateParams& p, cudaStream_t s) {
    const int cells = p.nx * p.ny;
    if (cells <= 0) return cudaSuccess;
    const int blocks = (cells + 255) / 256;
    validate_vector_kernel<<<blocks, 256, 0, s>>>(p);
    validate_median_kernel<<<blocks, 256, 0, s>>>(p);
    validate_replace_kernel<<<blocks, 256, 0, s>>>(p);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Summary counts (validate.rs:40-46), from the final flags as `validate` counts them.
// ---------------------------------------------------------------------------------------------
__global__ void summary_zero_kernel(unsigned long long* c) {
    if (threadIdx.x < 5) c[threadIdx.x] = 0;
}

__global__ void summary_kernel(const uint8_t* flags, int n, unsigned long long* c) {
    unsigned int loc[5] = {0, 0, 0, 0, 0};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint8_t f = flags[k];
        if (f & F_NO_SIGNAL) {
            loc[0]++;
            continue;
        }
        if (f & F_LOW_PPR) loc[1]++;
        if (f & F_MEDIAN_OUTLIER) loc[2]++;
        if (f & F_OUT_OF_RANGE) loc[3]++;
        if (f & F_REPLACED) loc[4]++;
    }
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        unsigned int v = loc[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&c[i], (unsigned long long)v);
    }
}

cudaError_t launch_summary(const uint8_t* flags, int n, unsigned long long* counts5, cudaStream_t s) {
    summary_zero_kernel<<<1, 32, 0, s>>>(counts5);
    const int blocks = n > 0 ? min((n + 255) / 256, 592) : 1;
    summary_kernel<<<blocks, 256, 0, s>>>(flags, n, counts5);
    return cudaGetLastError();
}

}  // namespace pivb200
