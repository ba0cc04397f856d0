// Window sampling and peak-fit helpers shared by the FP32 and tensor-core correlation kernels.
#pragma once

#include <cmath>

#include "common.cuh"

namespace pivb200 {

// (value, row-major index): larger value wins, then the lower index (correlate.rs:233-238).
__device__ __forceinline__ void amax_combine(float& v, int& i, float ov, int oi) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

// ---------------------------------------------------------------------------------------------
// Window sampling (correlate.rs:182-202): integer copy when both fractional parts are < 1e-4,
// otherwise bilinear with weights (1-tx)(1-ty), tx(1-ty), (1-tx)ty, tx*ty summed left to right.
// Indices are clamped into the image so that no access can leave it whatever the origin.
// ---------------------------------------------------------------------------------------------
//
// Where a sampler reads the image: the image in global memory through the read-only path. The
// samplers address pixels by their clamped image coordinates through at(row, col) and step rows
// by stride().
struct GlobalSrc {
    const float* img;
    int W;
    __device__ __forceinline__ const float* at(int row, int col) const { return img + (size_t)row * W + col; }
    __device__ __forceinline__ int stride() const { return W; }
    __device__ __forceinline__ static float ld(const float* p) { return __ldg(p); }
};

// Two samplers with identical results. sample_column_direct loads the four bilinear taps of
// every pixel itself (fewest live registers). sample_column loads each pixel of the patch once
// and trades the other taps through shuffles (fewest load instructions); it suits the window
// sizes whose register budget allows it.
template <int N, int T, bool IMAG, class Src>
__device__ __forceinline__ void sample_column_direct(const Src& src, int H, int W, float ox, float oy, int x, int t,
                                                     float2 (&z)[N / T]) {
    constexpr int P = N / T;
    const float fx0 = floorf(ox), fy0 = floorf(oy);
    const int x0 = min(max((int)fx0, 0), W - 1), y0 = min(max((int)fy0, 0), H - 1);
    const float tx = __fsub_rn(ox, fx0), ty = __fsub_rn(oy, fy0);
    const int c0 = min(x0 + x, W - 1);
    const int dc = min(x0 + x + 1, W - 1) - c0;  // right-hand tap: next float, or the same at the border
    const int last = H - 1 - y0;                  // rows below y0 that exist (row clamp)
    const int stride = src.stride();
    const float* base = src.at(y0, c0);
    if (tx < 1e-4f && ty < 1e-4f) {
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const float v = Src::ld(base + min(t + T * p, last) * stride);
            if (IMAG) z[p].y = v; else z[p].x = v;
        }
    } else {
        const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty);
        const float w00 = __fmul_rn(ux, uy), w01 = __fmul_rn(tx, uy), w10 = __fmul_rn(ux, ty), w11 = __fmul_rn(tx, ty);
        if constexpr (T == 1) {
            // One lane holds the whole column: stream down the rows, carrying the row below. The
            // right-hand tap is the next float (an immediate offset), or the same value at the
            // right border (dc == 0), where that load is skipped.
            auto blend = [&](int p, float tl, float tr, float bl, float br) {
                float s = __fmul_rn(w00, tl);
                s = __fadd_rn(s, __fmul_rn(w01, tr));
                s = __fadd_rn(s, __fmul_rn(w10, bl));
                s = __fadd_rn(s, __fmul_rn(w11, br));
                if (IMAG) z[p].y = s; else z[p].x = s;
            };
            float top = Src::ld(base);
            float topr = dc ? Src::ld(base + 1) : top;
            if (last >= P) {  // rows y0 .. y0 + P all exist: no row clamp, the row pointer steps by the pitch
                const float* bot = base;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    bot += stride;
                    const float b0 = Src::ld(bot);
                    const float b1 = dc ? Src::ld(bot + 1) : b0;
                    blend(p, top, topr, b0, b1);
                    top = b0;
                    topr = b1;
                }
            } else {
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const float* bot = base + min(p + 1, last) * stride;
                    const float b0 = Src::ld(bot);
                    const float b1 = dc ? Src::ld(bot + 1) : b0;
                    blend(p, top, topr, b0, b1);
                    top = b0;
                    topr = b1;
                }
            }
        } else {
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const float* top = base + min(t + T * p, last) * stride;
                const float* bot = base + min(t + T * p + 1, last) * stride;
                float s = __fmul_rn(w00, Src::ld(top));
                s = __fadd_rn(s, __fmul_rn(w01, Src::ld(top + dc)));
                s = __fadd_rn(s, __fmul_rn(w10, Src::ld(bot)));
                s = __fadd_rn(s, __fmul_rn(w11, Src::ld(bot + dc)));
                if (IMAG) z[p].y = s; else z[p].x = s;
            }
        }
    }
}

// Each pixel of the (N+1) x (N+1) source patch is loaded once: a lane loads its own column at
// its own rows; the right-hand column comes from the lane of the next line (T lanes further) by
// a shuffle, and the row below from the lane holding that row (the next register for T = 1, the
// next lane of the line otherwise). Lanes whose neighbour is outside their warp or beyond the
// window load the missing value themselves.
template <int N, int T, bool IMAG, class Src>
__device__ __forceinline__ void sample_column(const Src& src, int H, int W, float ox, float oy, int x, int t,
                                              float2 (&z)[N / T]) {
    constexpr int P = N / T;
    const int lane = threadIdx.x & 31;
    const float fx0 = floorf(ox), fy0 = floorf(oy);
    const int x0 = min(max((int)fx0, 0), W - 1), y0 = min(max((int)fy0, 0), H - 1);
    const float tx = __fsub_rn(ox, fx0), ty = __fsub_rn(oy, fy0);
    const int c0 = min(x0 + x, W - 1);
    const int dc = min(x0 + x + 1, W - 1) - c0;  // right-hand tap: next float, or the same at the border
    const int last = H - 1 - y0;                  // rows below y0 that exist (row clamp)
    const int stride = src.stride();
    const float* base = src.at(y0, c0);
    const bool integer = tx < 1e-4f && ty < 1e-4f;
    float top[P];
#pragma unroll
    for (int p = 0; p < P; ++p) top[p] = Src::ld(base + min(t + T * p, last) * stride);
    // Every lane runs the shuffles below (a warp may hold windows of both kinds); an integer
    // window then keeps its copied values.
    // Row N of the patch (below the window), held by the last lane of each line.
    const float* rowN = base + min(N, last) * stride;
    const float extra = Src::ld(rowN);
    const bool edge = lane + T >= 32 || x == N - 1;  // right neighbour not reachable by a shuffle
    float right[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        right[p] = __shfl_down_sync(0xffffffffu, top[p], T);
        if (edge) right[p] = Src::ld(base + min(t + T * p, last) * stride + dc);
    }
    float extra_r = __shfl_down_sync(0xffffffffu, extra, T);
    if (edge) extra_r = Src::ld(rowN + dc);
    const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty);
    const float w00 = __fmul_rn(ux, uy), w01 = __fmul_rn(tx, uy), w10 = __fmul_rn(ux, ty), w11 = __fmul_rn(tx, ty);
#pragma unroll
    for (int p = 0; p < P; ++p) {
        float b0, b1;  // row y + 1 at columns x and x + 1
        if constexpr (T == 1) {
            b0 = p + 1 < P ? top[p + 1] : extra;
            b1 = p + 1 < P ? right[p + 1] : extra_r;
        } else {
            // Row y + 1 of lane t < T-1 is the next lane's element p; of lane T-1 it is lane 0's
            // element p + 1. The source lane chooses what it sends: lane 0 sends element p + 1,
            // every other lane element p.
            const int q = p + 1 < P ? p + 1 : p;
            const int src = t < T - 1 ? lane + 1 : lane - (T - 1);
            const float n0 = __shfl_sync(0xffffffffu, t == 0 ? top[q] : top[p], src);
            const float n1 = __shfl_sync(0xffffffffu, t == 0 ? right[q] : right[p], src);
            const bool last = (t == T - 1) && (p == P - 1);
            b0 = last ? extra : n0;
            b1 = last ? extra_r : n1;
        }
        float s = __fmul_rn(w00, top[p]);
        s = __fadd_rn(s, __fmul_rn(w01, right[p]));
        s = __fadd_rn(s, __fmul_rn(w10, b0));
        s = __fadd_rn(s, __fmul_rn(w11, b1));
        if (integer) s = top[p];
        if (IMAG) z[p].y = s; else z[p].x = s;
    }
}

// Block layout for T > 1 lanes per column: lane (x, rt) holds column x at the P consecutive rows
// P*rt .. P*rt + P - 1 (rt = the lane's block). The lane streams down its rows carrying the row
// below, as the one-lane-per-column sampler does, so each sample needs one new row: two loads
// (DIRECT), or one load and the right-hand tap from the lane of the next column (lane + T, same
// block) by a shuffle (SHFL), where lanes whose neighbour is beyond their warp or the window load
// it themselves. The taps, weights and summation order are those of the other samplers, so the
// samples are the same bit for bit; only their place in the lanes differs.
template <int N, int T, bool IMAG, bool SHFL, class Src>
__device__ __forceinline__ void sample_block(const Src& src, int H, int W, float ox, float oy, int x, int rt,
                                             float2 (&z)[N / T]) {
    constexpr int P = N / T;
    const float fx0 = floorf(ox), fy0 = floorf(oy);
    const int x0 = min(max((int)fx0, 0), W - 1), y0 = min(max((int)fy0, 0), H - 1);
    const float tx = __fsub_rn(ox, fx0), ty = __fsub_rn(oy, fy0);
    const int c0 = min(x0 + x, W - 1);
    const int dc = min(x0 + x + 1, W - 1) - c0;  // right-hand tap: next float, or the same at the border
    const int last = H - 1 - y0;                  // rows below y0 that exist (row clamp)
    const int stride = src.stride();
    const int r0 = P * rt;
    const float* base = src.at(y0, c0);
    const bool integer = tx < 1e-4f && ty < 1e-4f;
    const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty);
    const float w00 = __fmul_rn(ux, uy), w01 = __fmul_rn(tx, uy), w10 = __fmul_rn(ux, ty), w11 = __fmul_rn(tx, ty);
    auto blend = [&](float tl, float tr, float bl, float br) {
        float s = __fmul_rn(w00, tl);
        s = __fadd_rn(s, __fmul_rn(w01, tr));
        s = __fadd_rn(s, __fmul_rn(w10, bl));
        return __fadd_rn(s, __fmul_rn(w11, br));
    };
    if constexpr (!SHFL) {
        if (integer) {
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const float v = Src::ld(base + min(r0 + p, last) * stride);
                if (IMAG) z[p].y = v; else z[p].x = v;
            }
            return;
        }
        const float* row = base + min(r0, last) * stride;
        float top = Src::ld(row);
        float topr = dc ? Src::ld(row + 1) : top;
        if (last >= r0 + P) {  // rows r0 .. r0 + P all exist: the row pointer steps by the pitch
#pragma unroll
            for (int p = 0; p < P; ++p) {
                row += stride;
                const float b0 = Src::ld(row);
                const float b1 = dc ? Src::ld(row + 1) : b0;
                const float s = blend(top, topr, b0, b1);
                if (IMAG) z[p].y = s; else z[p].x = s;
                top = b0;
                topr = b1;
            }
        } else {
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const float* bot = base + min(r0 + p + 1, last) * stride;
                const float b0 = Src::ld(bot);
                const float b1 = dc ? Src::ld(bot + 1) : b0;
                const float s = blend(top, topr, b0, b1);
                if (IMAG) z[p].y = s; else z[p].x = s;
                top = b0;
                topr = b1;
            }
        }
    } else {
        // Every lane runs the shuffles (an integer window then keeps its copied values).
        const int lane = threadIdx.x & 31;
        const bool edge = lane + T >= 32 || x == N - 1;  // right neighbour not reachable by a shuffle
        const float* row = base + min(r0, last) * stride;
        float top = Src::ld(row);
        float topr = __shfl_down_sync(0xffffffffu, top, T);
        if (edge) topr = Src::ld(row + dc);
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const float* bot = base + min(r0 + p + 1, last) * stride;
            const float b0 = Src::ld(bot);
            float b1 = __shfl_down_sync(0xffffffffu, b0, T);
            if (edge) b1 = Src::ld(bot + dc);
            const float s = integer ? top : blend(top, topr, b0, b1);
            if (IMAG) z[p].y = s; else z[p].x = s;
            top = b0;
            topr = b1;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Deformed windows (no counterpart in the reference, whose windows only shift): pixel (r, c) of
// the window at base position (x0, y0) (the grid origin under the placement clamp to W - n - 1,
// as a zero shift is placed by multipass.rs:207-231) is displaced by the bilinear blend D of the predictor at
// the window's four corner pixels, with u = c/(n-1), v = r/(n-1):
//   D = (1-u)(1-v) D00 + u(1-v) D10 + (1-u)v D01 + uv D11      (f32, summed left to right)
// frame A is sampled at (x0+c, y0+r) - D/2 and frame B at + D/2, bilinearly, coordinates
// clamped into the image and the tap clamped to the last full cell. Every operation is a
// round-to-nearest intrinsic in that order, so the samples are bit-identical to a sequential f32
// evaluation. Both frames' samples of one pixel share D: lane (x, t) fills z[p] = (A, B) at
// column x, row t + T*p.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float corner_blend(float c00, float c10, float c01, float c11, float u, float v) {
    const float ou = __fsub_rn(1.0f, u), ov = __fsub_rn(1.0f, v);
    float d = __fmul_rn(__fmul_rn(ou, ov), c00);
    d = __fadd_rn(d, __fmul_rn(__fmul_rn(u, ov), c10));
    d = __fadd_rn(d, __fmul_rn(__fmul_rn(ou, v), c01));
    return __fadd_rn(d, __fmul_rn(__fmul_rn(u, v), c11));
}

__device__ __forceinline__ float bilinear_clamped(const float* __restrict__ img, int H, int W, float px, float py) {
    px = px < 0.0f ? 0.0f : px;
    px = (float)(W - 1) < px ? (float)(W - 1) : px;
    py = py < 0.0f ? 0.0f : py;
    py = (float)(H - 1) < py ? (float)(H - 1) : py;
    const int ix = min((int)floorf(px), max(W - 2, 0)), iy = min((int)floorf(py), max(H - 2, 0));
    const float tx = __fsub_rn(px, (float)ix), ty = __fsub_rn(py, (float)iy);
    const int ix1 = min(ix + 1, W - 1), iy1 = min(iy + 1, H - 1);
    const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty);
    const float* top = img + (size_t)iy * W;
    const float* bot = img + (size_t)iy1 * W;
    float s = __fmul_rn(__fmul_rn(ux, uy), __ldg(top + ix));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(tx, uy), __ldg(top + ix1)));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(ux, ty), __ldg(bot + ix)));
    return __fadd_rn(s, __fmul_rn(__fmul_rn(tx, ty), __ldg(bot + ix1)));
}

// BLOCKROWS: lane (x, t) fills rows P*t + p (t then names the lane's row block) instead of t + T*p.
template <int N, int T, bool BLOCKROWS = false>
__device__ __forceinline__ void sample_deformed(const float* __restrict__ img_a, const float* __restrict__ img_b, int H,
                                                int W, int x0, int y0, float4 k0, float4 k1, int x, int t,
                                                const float* s_ramp, float2 (&z)[N / T]) {
    constexpr int P = N / T;
    const float u = s_ramp[x];
    const float xf = (float)(x0 + x);
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int r = BLOCKROWS ? P * t + p : t + T * p;
        const float v = s_ramp[r];
        const float hx = __fmul_rn(0.5f, corner_blend(k0.x, k0.z, k1.x, k1.z, u, v));
        const float hy = __fmul_rn(0.5f, corner_blend(k0.y, k0.w, k1.y, k1.w, u, v));
        const float yf = (float)(y0 + r);
        z[p].x = bilinear_clamped(img_a, H, W, __fsub_rn(xf, hx), __fsub_rn(yf, hy));
        z[p].y = bilinear_clamped(img_b, H, W, __fadd_rn(xf, hx), __fadd_rn(yf, hy));
    }
}

// 3-point Gaussian sub-pixel offset, parabolic when a value is not positive (correlate.rs:269-281).
__device__ __forceinline__ float subpixel(float m, float c, float p) {
    float d;
    if (m > 0.0f && c > 0.0f && p > 0.0f) {
        const float lm = logf(m), lc = logf(c), lp = logf(p);
        d = __fdiv_rn(__fsub_rn(lm, lp), __fmul_rn(2.0f, __fadd_rn(__fsub_rn(lm, __fmul_rn(2.0f, lc)), lp)));
    } else {
        d = __fdiv_rn(__fsub_rn(m, p), __fmul_rn(2.0f, __fadd_rn(__fsub_rn(m, __fmul_rn(2.0f, c)), p)));
    }
    if (isfinite(d)) return fminf(fmaxf(d, -0.5f), 0.5f);
    return 0.0f;
}

}  // namespace pivb200
