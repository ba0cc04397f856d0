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

// Batches of items of any grid size: item i owns cells [cell_start[i], cell_start[i+1]).
struct PlaceBatch {
    int n;
    int cell_start[kMaxBatch + 1];
    PlaceParams item[kMaxBatch];
};

struct ValidateBatch {
    int n;
    int cell_start[kMaxBatch + 1];
    ValidateParams item[kMaxBatch];
};

struct SummaryBatch {
    int n;
    int cell_start[kMaxBatch + 1];
    SummaryItem item[kMaxBatch];
};

__global__ void place_kernel(const __grid_constant__ PlaceBatch b) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= b.cell_start[b.n]) return;
    const int it = batch_item(b.cell_start, b.n, u);
    const PlaceParams& p = b.item[it];
    const int k = u - b.cell_start[it];
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
    if (p.corners) {
        // Predictor at the corner pixels (x0, y0), (x0+n-1, y0), (x0, y0+n-1), (x0+n-1, y0+n-1) of
        // the deformed window's base position: the zero-shift origin under the placement clamp.
        const float xa = (float)min(p.grid.x0 + ix * p.grid.step, max(p.W - n - 1, 0));
        const float ya = (float)min(p.grid.y0 + iy * p.grid.step, max(p.H - n - 1, 0));
        const float xb = __fadd_rn(xa, (float)(n - 1)), yb = __fadd_rn(ya, (float)(n - 1));
        float2 c00 = make_float2(0.0f, 0.0f), c10 = c00, c01 = c00, c11 = c00;
        if (p.has_pred) {
            c00 = sample_predictor(p.pdx, p.pdy, p.pgrid, xa, ya);
            c10 = sample_predictor(p.pdx, p.pdy, p.pgrid, xb, ya);
            c01 = sample_predictor(p.pdx, p.pdy, p.pgrid, xa, yb);
            c11 = sample_predictor(p.pdx, p.pdy, p.pgrid, xb, yb);
        }
        p.corners[2 * (size_t)k] = make_float4(c00.x, c00.y, c10.x, c10.y);
        p.corners[2 * (size_t)k + 1] = make_float4(c01.x, c01.y, c11.x, c11.y);
    }
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

cudaError_t launch_place_items(const PlaceParams* items, int count, cudaStream_t s, int* launches) {
    for (int off = 0; off < count; off += kMaxBatch) {
        PlaceBatch b;
        b.n = min(count - off, kMaxBatch);
        long long total = 0;
        for (int i = 0; i < b.n; ++i) {
            b.item[i] = items[off + i];
            b.cell_start[i] = (int)total;
            total += (long long)b.item[i].grid.nx * b.item[i].grid.ny;
        }
        b.cell_start[b.n] = (int)total;
        if (total <= 0) continue;
        if (total > 0x7fffffffll) return cudaErrorInvalidValue;
        place_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(b);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (launches) ++*launches;
    }
    return cudaSuccess;
}

cudaError_t launch_place(const PlaceParams& p, cudaStream_t s) { return launch_place_items(&p, 1, s, nullptr); }

cudaError_t launch_mask(const PlaceParams& p, const float4* origins, int ncells, cudaStream_t s) {
    if (ncells <= 0) return cudaSuccess;
    mask_kernel<<<(ncells + 255) / 256, 256, 0, s>>>(p, origins, ncells);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Validation
// ---------------------------------------------------------------------------------------------
// Total-order key of a non-NaN float: signed integer order of the keys is f32::total_cmp order
// (-0.0 before +0.0), which validate.rs:164 sorts by. The map is its own inverse.
__device__ __forceinline__ int tkey(float f) {
    const int b = __float_as_int(f);
    return b ^ ((b >> 31) & 0x7fffffff);
}
__device__ __forceinline__ float tval(int k) { return __int_as_float(k ^ ((k >> 31) & 0x7fffffff)); }

// Sorts v[0..n) ascending by total order (insertion sort) and returns the median, the mean of
// the middle two when n is even (validate.rs:163-170).
__device__ float median_sorted(float* v, int n) {
    for (int i = 1; i < n; ++i) {
        const float x = v[i];
        const int kx = tkey(x);
        int j = i;
        while (j > 0 && tkey(v[j - 1]) > kx) {
            v[j] = v[j - 1];
            --j;
        }
        v[j] = x;
    }
    if (n % 2 == 1) return v[n / 2];
    return __fmul_rn(0.5f, __fadd_rn(v[n / 2 - 1], v[n / 2]));
}

// Radius-1 neighbourhoods in registers: eight key slots, absent or unusable neighbours padded with
// INT_MAX (above every finite key), sorted by Batcher's odd-even merge network (19 exchanges), so
// the c usable keys come first in order.
__device__ __forceinline__ void kx_swap(int& a, int& b) {
    const int lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}
__device__ __forceinline__ void sort8(int (&k)[8]) {
    kx_swap(k[0], k[1]); kx_swap(k[2], k[3]); kx_swap(k[4], k[5]); kx_swap(k[6], k[7]);
    kx_swap(k[0], k[2]); kx_swap(k[1], k[3]); kx_swap(k[4], k[6]); kx_swap(k[5], k[7]);
    kx_swap(k[1], k[2]); kx_swap(k[5], k[6]);
    kx_swap(k[0], k[4]); kx_swap(k[1], k[5]); kx_swap(k[2], k[6]); kx_swap(k[3], k[7]);
    kx_swap(k[2], k[4]); kx_swap(k[3], k[5]);
    kx_swap(k[1], k[2]); kx_swap(k[3], k[4]); kx_swap(k[5], k[6]);
}
// Median of the first c (1..8) of eight sorted keys, as median_sorted computes it.
__device__ __forceinline__ float median8(const int (&k)[8], int c) {
    int lo = k[0], hi = k[0];
#pragma unroll
    for (int i = 1; i < 8; ++i) {
        if (i == (c - 1) / 2) lo = k[i];
        if (i == c / 2) hi = k[i];
    }
    if (c % 2 == 1) return tval(hi);
    return __fmul_rn(0.5f, __fadd_rn(tval(lo), tval(hi)));
}
// Normalised residual |value - med| / (median |nb - med| + eps) over the first c sorted keys
// (validate.rs:157-161).
__device__ __forceinline__ float residual8(float value, const int (&k)[8], int c, float eps) {
    const float med = median8(k, c);
    int dev[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) dev[i] = i < c ? tkey(fabsf(__fsub_rn(tval(k[i]), med))) : 0x7fffffff;
    sort8(dev);
    return __fdiv_rn(fabsf(__fsub_rn(value, med)), __fadd_rn(median8(dev, c), eps));
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

// Per-vector tests (validate.rs:59-78).
__device__ __forceinline__ void validate_vector(const ValidateParams& p, int k) {
    uint8_t f = p.flags0[k];
    if (!(f & F_NO_SIGNAL)) {
        if (hypotf(p.dx[k], p.dy[k]) > p.max_displacement) f |= F_OUT_OF_RANGE;
        if (p.ppr[k] < p.ppr_threshold) f |= F_LOW_PPR;
    }
    p.flags1[k] = f;
}

// Normalized median test on a snapshot of the flags (validate.rs:80-100).
__device__ __forceinline__ void validate_median(const ValidateParams& p, int k) {
    const int ix = k % p.nx, iy = k / p.nx;
    uint8_t f = p.flags1[k];
    if ((f & F_INVALID) == 0) {
        // usable 3x3 neighbours (validate.rs:133-155), padded slots for the others
        int ku[8], kv[8];
        int c = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int dxo = (j < 3) ? j - 1 : (j < 5 ? (j == 3 ? -1 : 1) : j - 6);
            const int dyo = (j < 3) ? -1 : (j < 5 ? 0 : 1);
            const int x = ix + dxo, y = iy + dyo;
            ku[j] = kv[j] = 0x7fffffff;
            if (x >= 0 && x < p.nx && y >= 0 && y < p.ny) {
                const int o = y * p.nx + x;
                if ((p.flags1[o] & F_INVALID) == 0) {
                    ku[j] = tkey(p.dx[o]);
                    kv[j] = tkey(p.dy[o]);
                    ++c;
                }
            }
        }
        if (c >= 2) {
            sort8(ku);
            sort8(kv);
            const float ru = residual8(p.dx[k], ku, c, p.median_eps);
            const float rv = residual8(p.dy[k], kv, c, p.median_eps);
            if (__fsqrt_rn(__fadd_rn(__fmul_rn(ru, ru), __fmul_rn(rv, rv))) > p.median_threshold) f |= F_MEDIAN_OUTLIER;
        }
    }
    p.flags2[k] = f;
}

// Replacement by the median of usable neighbours at radius 1, then 2 (validate.rs:102-128).
__device__ __forceinline__ void validate_replace(const ValidateParams& p, int k) {
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

template <int STAGE>
__global__ void validate_kernel(const __grid_constant__ ValidateBatch b) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= b.cell_start[b.n]) return;
    const int it = batch_item(b.cell_start, b.n, u);
    const int k = u - b.cell_start[it];
    if (STAGE == 0) validate_vector(b.item[it], k);
    if (STAGE == 1) validate_median(b.item[it], k);
    if (STAGE == 2) validate_replace(b.item[it], k);
}

cudaError_t launch_validate_items(const ValidateParams* items, int count, cudaStream_t s, int* launches) {
    for (int off = 0; off < count; off += kMaxBatch) {
        ValidateBatch b;
        b.n = min(count - off, kMaxBatch);
        long long total = 0;
        for (int i = 0; i < b.n; ++i) {
            b.item[i] = items[off + i];
            b.cell_start[i] = (int)total;
            total += (long long)b.item[i].nx * b.item[i].ny;
        }
        b.cell_start[b.n] = (int)total;
        if (total <= 0) continue;
        if (total > 0x7fffffffll) return cudaErrorInvalidValue;
        const unsigned blocks = (unsigned)((total + 255) / 256);
        validate_kernel<0><<<blocks, 256, 0, s>>>(b);
        validate_kernel<1><<<blocks, 256, 0, s>>>(b);
        validate_kernel<2><<<blocks, 256, 0, s>>>(b);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (launches) *launches += 3;
    }
    return cudaSuccess;
}

cudaError_t launch_validate(const ValidateParams& p, cudaStream_t s) { return launch_validate_items(&p, 1, s, nullptr); }

// ---------------------------------------------------------------------------------------------
// Summary counts (validate.rs:40-46), from the final flags as `validate` counts them.
// ---------------------------------------------------------------------------------------------
__global__ void summary_zero_kernel(const __grid_constant__ SummaryBatch b) {
    const int i = threadIdx.x / 5, j = threadIdx.x % 5;
    if (i < b.n) b.item[i].counts5[j] = 0;
}

__global__ void summary_kernel(const __grid_constant__ SummaryBatch b) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = u < b.cell_start[b.n];
    const int it = in ? batch_item(b.cell_start, b.n, u) : 0;
    unsigned int loc[5] = {0, 0, 0, 0, 0};
    if (in) {
        const uint8_t f = b.item[it].flags[u - b.cell_start[it]];
        if (f & F_NO_SIGNAL) {
            loc[0] = 1;
        } else {
            loc[1] = (f & F_LOW_PPR) ? 1 : 0;
            loc[2] = (f & F_MEDIAN_OUTLIER) ? 1 : 0;
            loc[3] = (f & F_OUT_OF_RANGE) ? 1 : 0;
            loc[4] = (f & F_REPLACED) ? 1 : 0;
        }
    }
    // Lanes of one item reduce together; the leader of each item's lanes adds the totals.
    const unsigned same = __match_any_sync(0xffffffffu, in ? it : -1);
    const int leader = __ffs(same) - 1;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const unsigned int v = __reduce_add_sync(same, loc[i]);
        if (in && (int)(threadIdx.x & 31) == leader && v) atomicAdd(&b.item[it].counts5[i], (unsigned long long)v);
    }
}

cudaError_t launch_summary_items(const SummaryItem* items, int count, cudaStream_t s, int* launches) {
    for (int off = 0; off < count; off += kMaxBatch) {
        SummaryBatch b;
        b.n = min(count - off, kMaxBatch);
        long long total = 0;
        for (int i = 0; i < b.n; ++i) {
            b.item[i] = items[off + i];
            b.cell_start[i] = (int)total;
            total += b.item[i].n;
        }
        b.cell_start[b.n] = (int)total;
        summary_zero_kernel<<<1, 5 * kMaxBatch, 0, s>>>(b);
        if (total > 0) summary_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(b);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (launches) *launches += total > 0 ? 2 : 1;
    }
    return cudaSuccess;
}

cudaError_t launch_summary(const uint8_t* flags, int n, unsigned long long* counts5, cudaStream_t s) {
    SummaryItem it{flags, n, counts5};
    return launch_summary_items(&it, 1, s, nullptr);
}

}  // namespace pivb200
