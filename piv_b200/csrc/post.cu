// Post-processing of validated fields on the device: flow statistics (vorticity, kinetic energy,
// coverage) of one pair and the temporal / spatial smoothing filters of a pair series.
//
// Reference semantics: usable (flow.rs:13-17), pair_stats (flow.rs:20-36), vorticity and
// flow_stats (flowstats.rs:28-101), temporal (smooth.rs:44-128), spatial (smooth.rs:130-207).
// Compiled with --fmad=false: every f32 expression rounds as the reference's, so vorticity,
// smoothed fields and supports are bit-identical to a sequential evaluation; the f64 sums of the
// statistics use a fixed-order tree and agree to f32 rounding.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace pivb200 {

constexpr int kMaxTemporalOffsets = 64;
constexpr int kMaxSpatialDiameter = 61;  // sigma <= 12

struct FlowPartial {
    double ws, wa, e;
    long long nw, n;
};

__device__ __forceinline__ bool usable_cell(float dx, uint8_t f) {
    return isfinite(dx) && ((f & F_INVALID) == 0 || (f & F_REPLACED) != 0);
}

// Velocity component at a cell (px/s) when the cell is usable and the value finite.
__device__ __forceinline__ bool comp_at(const float* d, const float* dxf, const uint8_t* fl, int i, float k, float* o) {
    if (!usable_cell(dxf[i], fl[i])) return false;
    const float x = __fmul_rn(d[i], k);
    if (!isfinite(x)) return false;
    *o = x;
    return true;
}

// flowstats.rs:28-39 on a line through cell i with neighbours i - s and i + s.
__device__ __forceinline__ bool deriv(const float* d, const float* dxf, const uint8_t* fl, int pos, int n, int i, int s,
                                      float k, float h, float* out) {
    float c, l, r;
    if (!comp_at(d, dxf, fl, i, k, &c)) return false;
    const bool hl = pos >= 1 && comp_at(d, dxf, fl, i - s, k, &l);
    const bool hr = pos + 1 < n && comp_at(d, dxf, fl, i + s, k, &r);
    if (hl && hr) *out = __fdiv_rn(__fsub_rn(r, l), __fmul_rn(2.0f, h));
    else if (hl) *out = __fdiv_rn(__fsub_rn(c, l), h);
    else if (hr) *out = __fdiv_rn(__fsub_rn(r, c), h);
    else return false;
    return true;
}

__global__ void flow_kernel(int ny, int nx, float k, float h, const float* __restrict__ dx, const float* __restrict__ dy,
                            const uint8_t* __restrict__ fl, float* vort, FlowPartial* part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ws = 0.0, wa = 0.0, e = 0.0;
    long long nw = 0, n = 0;
    if (i < ny * nx) {
        const int iy = i / nx, ix = i % nx;
        float a, b;
        const bool ha = deriv(dx, dx, fl, iy, ny, i, nx, k, h, &a);  // du/dy
        const bool hb = deriv(dy, dx, fl, ix, nx, i, 1, k, h, &b);   // dv/dx
        const float w = (ha && hb) ? __fsub_rn(a, b) : NAN;
        if (vort) vort[i] = w;
        if (isfinite(w)) {
            ws = (double)w;
            wa = (double)fabsf(w);
            nw = 1;
        }
        const float u = __fmul_rn(dx[i], k), v = __fmul_rn(dy[i], k);
        if (usable_cell(dx[i], fl[i]) && isfinite(u) && isfinite(v)) {
            e = 0.5 * __dadd_rn(__dmul_rn((double)u, (double)u), __dmul_rn((double)v, (double)v));
            n = 1;
        }
    }
    // fixed-order block reduction
    __shared__ FlowPartial sh[256];
    sh[threadIdx.x] = FlowPartial{ws, wa, e, nw, n};
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            FlowPartial& p = sh[threadIdx.x];
            const FlowPartial& q = sh[threadIdx.x + s];
            p.ws += q.ws;
            p.wa += q.wa;
            p.e += q.e;
            p.nw += q.nw;
            p.n += q.n;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void flow_final_kernel(const FlowPartial* part, int nparts, FlowPartial* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    FlowPartial t{0.0, 0.0, 0.0, 0, 0};
    for (int j = 0; j < nparts; ++j) {
        t.ws += part[j].ws;
        t.wa += part[j].wa;
        t.e += part[j].e;
        t.nw += part[j].nw;
        t.n += part[j].n;
    }
    *out = t;
}

cudaError_t flow_stats_device(int ny, int nx, float step, double dt_s, const float* dx, const float* dy,
                              const uint8_t* flags, float* vort, FlowStatsHost* stats, cudaStream_t s) {
    const int cells = ny * nx;
    const int blocks = (cells + 255) / 256;
    void* buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, sizeof(FlowPartial) * (size_t)(blocks + 1), s);
    if (e != cudaSuccess) return e;
    FlowPartial* part = static_cast<FlowPartial*>(buf);
    const float k = (float)(1.0 / dt_s);
    flow_kernel<<<blocks, 256, 0, s>>>(ny, nx, k, step, dx, dy, flags, vort, part);
    flow_final_kernel<<<1, 32, 0, s>>>(part, blocks, part + blocks);
    FlowPartial t{};
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&t, part + blocks, sizeof(t), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(buf, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    auto mean = [](double v, long long c) { return c > 0 ? (float)(v / (double)c) : NAN; };
    stats->vorticity_mean = mean(t.ws, t.nw);
    stats->vorticity_abs_mean = mean(t.wa, t.nw);
    stats->ke_mean = mean(t.e, t.n);
    stats->ke_sum = (float)(t.e * ((double)step * (double)step));
    stats->coverage = (float)t.n / (float)(cells > 0 ? cells : 1);
    stats->n_usable = t.n;
    stats->n_vorticity = t.nw;
    return cudaSuccess;
}

// ---------------------------------------------------------------------------------------------
// Temporal filter (smooth.rs:44-128): one thread per (pair, cell).
// ---------------------------------------------------------------------------------------------
struct TemporalParams {
    int nt, plane, n_off, median, min_support;
    int off[kMaxTemporalOffsets];
};

__device__ __forceinline__ float seq_mean(const float* v, int n) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s = __fadd_rn(s, v[i]);
    return __fdiv_rn(s, (float)n);
}
__device__ __forceinline__ float sorted_median(float* v, int n) {
    for (int i = 1; i < n; ++i) {
        const float x = v[i];
        int j = i;
        while (j > 0 && v[j - 1] > x) {
            v[j] = v[j - 1];
            --j;
        }
        v[j] = x;
    }
    return (n & 1) ? v[n / 2] : __fmul_rn(0.5f, __fadd_rn(v[n / 2 - 1], v[n / 2]));
}

__global__ void temporal_kernel(const __grid_constant__ TemporalParams p, const float* __restrict__ dx,
                                const float* __restrict__ dy, const uint8_t* __restrict__ usable,
                                const uint8_t* __restrict__ gate, float* out_dx, float* out_dy, uint16_t* support) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= (long long)p.nt * p.plane) return;
    const int t = (int)(o / p.plane), k = (int)(o % p.plane);
    out_dx[o] = NAN;
    out_dy[o] = NAN;
    support[o] = 0;
    if (!gate[o]) return;
    float bu[kMaxTemporalOffsets], bv[kMaxTemporalOffsets];
    int c = 0;
    for (int j = 0; j < p.n_off; ++j) {
        const int s = t + p.off[j];
        if (s < 0 || s >= p.nt) continue;
        const long long q = (long long)s * p.plane + k;
        if (!usable[q]) continue;
        bu[c] = dx[q];
        bv[c] = dy[q];
        ++c;
    }
    support[o] = (uint16_t)c;
    if (c >= max(p.min_support, 1)) {
        out_dx[o] = p.median ? sorted_median(bu, c) : seq_mean(bu, c);
        out_dy[o] = p.median ? sorted_median(bv, c) : seq_mean(bv, c);
    }
}

cudaError_t temporal_smooth_device(int nt, int ny, int nx, const float* dx, const float* dy, const uint8_t* usable,
                                   const uint8_t* gate, int median, const int* offsets, int n_off, int min_support,
                                   float* out_dx, float* out_dy, uint16_t* support, cudaStream_t s) {
    if (n_off < 0 || n_off > kMaxTemporalOffsets) return cudaErrorInvalidValue;
    TemporalParams p{};
    p.nt = nt;
    p.plane = ny * nx;
    p.n_off = n_off;
    p.median = median;
    p.min_support = min_support;
    for (int i = 0; i < n_off; ++i) p.off[i] = offsets[i];
    const long long total = (long long)nt * ny * nx;
    if (total <= 0) return cudaSuccess;
    temporal_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(p, dx, dy, usable, gate, out_dx, out_dy, support);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Spatial filter (smooth.rs:130-207): normalized Gaussian convolution, one thread per output.
// ---------------------------------------------------------------------------------------------
struct SpatialParams {
    int nt, ny, nx, r, leave_out;
    int none;         // most of the kernel's weight left out: no prediction anywhere (smooth.rs:164-166)
    float threshold;  // min_weight * full
    float w[kMaxSpatialDiameter * kMaxSpatialDiameter];
};

__global__ void spatial_kernel(const __grid_constant__ SpatialParams p, const float* __restrict__ dx,
                               const float* __restrict__ dy, const uint8_t* __restrict__ gate, float* out_dx,
                               float* out_dy, uint16_t* support) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long plane = (long long)p.ny * p.nx;
    if (o >= (long long)p.nt * plane) return;
    const int t = (int)(o / plane), y = (int)((o % plane) / p.nx), x = (int)(o % p.nx);
    out_dx[o] = NAN;
    out_dy[o] = NAN;
    support[o] = 0;
    if (p.none || !gate[o]) return;
    const int d = 2 * p.r + 1;
    float su = 0.0f, sv = 0.0f, sw = 0.0f;
    int n = 0;
    for (int j = -p.r; j <= p.r; ++j) {
        const int yy = y + j;
        if (yy < 0 || yy >= p.ny) continue;
        for (int i = -p.r; i <= p.r; ++i) {
            const int xx = x + i;
            if (xx < 0 || xx >= p.nx) continue;
            if (p.leave_out >= 0 && max(abs(i), abs(j)) <= p.leave_out) continue;
            const long long q = (long long)t * plane + (long long)yy * p.nx + xx;
            const float a = dx[q], b = dy[q];
            if (isfinite(a) && isfinite(b)) {
                const float w = p.w[(j + p.r) * d + (i + p.r)];
                su = __fadd_rn(su, __fmul_rn(w, a));
                sv = __fadd_rn(sv, __fmul_rn(w, b));
                sw = __fadd_rn(sw, w);
                ++n;
            }
        }
    }
    support[o] = (uint16_t)n;
    if (sw >= p.threshold && sw > 0.0f) {
        out_dx[o] = __fdiv_rn(su, sw);
        out_dy[o] = __fdiv_rn(sv, sw);
    }
}

cudaError_t spatial_smooth_device(int nt, int ny, int nx, const float* dx, const float* dy, const uint8_t* gate,
                                  float sigma, float min_weight, int leave_out, float* out_dx, float* out_dy,
                                  uint16_t* support, cudaStream_t s) {
    SpatialParams p{};
    // smooth.rs:143-166, on the host in f32 (the same exp as the reference's platform libm)
    const int r = std::max((int)std::ceil(2.5f * sigma), 1);
    const int d = 2 * r + 1;
    if (d > kMaxSpatialDiameter) return cudaErrorInvalidValue;
    float full = 0.0f, total = 0.0f;
    for (int j = -r; j <= r; ++j)
        for (int i = -r; i <= r; ++i) {
            const float w = std::exp(-((float)(i * i + j * j)) / (2.0f * sigma * sigma));
            p.w[(j + r) * d + (i + r)] = w;
        }
    for (int j = -r; j <= r; ++j)
        for (int i = -r; i <= r; ++i) {
            const float w = p.w[(j + r) * d + (i + r)];
            if (!(leave_out >= 0 && std::max(std::abs(i), std::abs(j)) <= leave_out)) full += w;
            total += w;
        }
    p.nt = nt;
    p.ny = ny;
    p.nx = nx;
    p.r = r;
    p.leave_out = leave_out;
    p.threshold = min_weight * full;
    const long long cells = (long long)nt * ny * nx;
    if (cells <= 0) return cudaSuccess;
    p.none = full < 0.5f * total;
    spatial_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(p, dx, dy, gate, out_dx, out_dy, support);
    return cudaGetLastError();
}

}  // namespace pivb200
