// Fused per-window FFT cross-correlation and peak fit (FP32 plain path).
//
// Reference semantics: CorrelationPlan::correlate (correlate.rs:99-139), load_window
// (correlate.rs:182-210), find_peak (correlate.rs:215-303) and the pair assembly of
// PivAnalyzer::pass (multipass.rs:242-259).
//
// Work decomposition (one thread group = N*T threads, one window PAIR per group):
//   1. window A and window B of a pair are sampled (bilinear, same f32 operation order as the
//      reference, no FMA) straight into registers as one complex plane z = a + i*b; lane (x, t)
//      holds column x at rows t + T*p, so every load instruction reads contiguous image rows;
//   2. mean removal and energy (group reductions), 2-D FFT of z (columns in registers, transpose
//      through shared memory, rows in registers);
//   3. the two real spectra are separated with the Hermitian partner Z[-k] (one shared-memory
//      exchange) and the cross spectrum conj(FA)*FB formed in registers;
//   4. the second window of the pair repeats 1-3; both cross spectra are Hermitian, so their
//      inverse transforms are packed into ONE complex inverse 2-D FFT (real part = first
//      correlation plane, imaginary part = second);
//   5. the scaled planes go to shared memory; argmax (lowest row-major index on ties), the
//      half-width footprint, the second local maximum and the 3-point Gaussian fit run on them.
// The 128 px window has no room for the pair stash in registers and runs one window per group
// with a full complex inverse.
#include <cfloat>
#include <cmath>
#include <cstdio>

#include "common.cuh"
#include "fft.cuh"
#include "kernels.h"

namespace pivb200 {

template <int N, int T, bool PAIR, int G>
struct CorrCfg {
    static constexpr int P = N / T;
    static constexpr int NT = N * T;
    static constexpr int THREADS = G * NT;
    static constexpr int LD = N + 1;
    static constexpr int WPG = PAIR ? 2 : 1;
    // Shuffle segment: largest power of two dividing NT, at most a warp.
    static constexpr int SW = (NT % 32 == 0) ? 32 : (NT % 16 == 0) ? 16 : (NT % 8 == 0) ? 8 : (NT % 4 == 0) ? 4 : (NT % 2 == 0) ? 2 : 1;
    static constexpr int NSEG = NT / SW;
    static constexpr size_t SMEM = sizeof(float2) * (size_t)(G * N * LD + N) + sizeof(float) * (size_t)(G * NSEG * 4) + 64;
};

// ---------------------------------------------------------------------------------------------
// Group reductions (segments of SW lanes by shuffles, then NSEG partials through shared memory).
// Every thread of the group returns the same value; the combination order is fixed.
// ---------------------------------------------------------------------------------------------
template <class C>
__device__ __forceinline__ float2 group_sum2(float2 v, float* s_red, int g, int gt) {
    constexpr int SW = C::SW, NSEG = C::NSEG;
#pragma unroll
    for (int o = SW / 2; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if constexpr (NSEG == 1) {
        return v;
    } else {
        float* r = s_red + g * NSEG * 4;
        if (gt % SW == 0) {
            r[(gt / SW) * 2 + 0] = v.x;
            r[(gt / SW) * 2 + 1] = v.y;
        }
        __syncthreads();
        float2 s = make_float2(0.f, 0.f);
#pragma unroll
        for (int i = 0; i < NSEG; ++i) {
            s.x += r[i * 2 + 0];
            s.y += r[i * 2 + 1];
        }
        __syncthreads();
        return s;
    }
}

template <class C>
__device__ __forceinline__ float group_max(float v, float* s_red, int g, int gt) {
    constexpr int SW = C::SW, NSEG = C::NSEG;
#pragma unroll
    for (int o = SW / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if constexpr (NSEG == 1) {
        return v;
    } else {
        float* r = s_red + g * NSEG * 4;
        if (gt % SW == 0) r[gt / SW] = v;
        __syncthreads();
        float s = -INFINITY;
#pragma unroll
        for (int i = 0; i < NSEG; ++i) s = fmaxf(s, r[i]);
        __syncthreads();
        return s;
    }
}

// (value, row-major index): larger value wins, then the lower index (correlate.rs:233-238).
__device__ __forceinline__ void amax_combine(float& v, int& i, float ov, int oi) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

template <class C>
__device__ __forceinline__ void group_argmax(float& v, int& idx, float* s_red, int g, int gt) {
    constexpr int SW = C::SW, NSEG = C::NSEG;
#pragma unroll
    for (int o = SW / 2; o > 0; o >>= 1) {
        float ov = __shfl_xor_sync(0xffffffffu, v, o);
        int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        amax_combine(v, idx, ov, oi);
    }
    if constexpr (NSEG > 1) {
        float* r = s_red + g * NSEG * 4;
        if (gt % SW == 0) {
            r[(gt / SW) * 2 + 0] = v;
            r[(gt / SW) * 2 + 1] = __int_as_float(idx);
        }
        __syncthreads();
        float bv = -INFINITY;
        int bi = 0x7fffffff;
#pragma unroll
        for (int i = 0; i < NSEG; ++i) amax_combine(bv, bi, r[i * 2 + 0], __float_as_int(r[i * 2 + 1]));
        __syncthreads();
        v = bv;
        idx = bi;
    }
}

// ---------------------------------------------------------------------------------------------
// Window sampling (correlate.rs:182-202): integer copy when both fractional parts are < 1e-4,
// otherwise bilinear with weights (1-tx)(1-ty), tx(1-ty), (1-tx)ty, tx*ty summed left to right.
// Indices are clamped into the image so that no access can leave it whatever the origin.
// ---------------------------------------------------------------------------------------------
template <int N, int T>
__device__ __forceinline__ void sample_column(const float* __restrict__ img, int H, int W, float ox, float oy,
                                              int x, int t, float (&v)[N / T]) {
    constexpr int P = N / T;
    const float fx0 = floorf(ox), fy0 = floorf(oy);
    const int x0 = min(max((int)fx0, 0), W - 1), y0 = min(max((int)fy0, 0), H - 1);
    const float tx = __fsub_rn(ox, fx0), ty = __fsub_rn(oy, fy0);
    const int c0 = min(x0 + x, W - 1), c1 = min(x0 + x + 1, W - 1);
    if (tx < 1e-4f && ty < 1e-4f) {
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int r = min(y0 + t + T * p, H - 1);
            v[p] = __ldg(img + (size_t)r * W + c0);
        }
    } else {
        const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty);
        const float w00 = __fmul_rn(ux, uy), w01 = __fmul_rn(tx, uy), w10 = __fmul_rn(ux, ty), w11 = __fmul_rn(tx, ty);
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int r0 = min(y0 + t + T * p, H - 1), r1 = min(y0 + t + T * p + 1, H - 1);
            const float* top = img + (size_t)r0 * W;
            const float* bot = img + (size_t)r1 * W;
            float s = __fmul_rn(w00, __ldg(top + c0));
            s = __fadd_rn(s, __fmul_rn(w01, __ldg(top + c1)));
            s = __fadd_rn(s, __fmul_rn(w10, __ldg(bot + c0)));
            s = __fadd_rn(s, __fmul_rn(w11, __ldg(bot + c1)));
            v[p] = s;
        }
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

template <int N, int T, bool PAIR, int G>
__global__ void __launch_bounds__(G * N * T) correlate_kernel(const CorrParams prm) {
    using C = CorrCfg<N, T, PAIR, G>;
    constexpr int P = C::P, NT = C::NT, LD = C::LD, WPG = C::WPG;
    extern __shared__ float4 smem_f4[];
    float2* planes = reinterpret_cast<float2*>(smem_f4);
    float2* s_roots = planes + G * N * LD;
    float* s_red = reinterpret_cast<float*>(s_roots + N);
    __shared__ int s_hw[G][8];

    const int tid = threadIdx.x;
    const int g = tid / NT;
    const int gt = tid - g * NT;
    const int line = gt / T;
    const int t = gt - line * T;
    const int rt = bitrev<T>(t);
    float2* plane = planes + g * N * LD;

    for (int i = tid; i < N; i += C::THREADS) s_roots[i] = c_roots[root_off(N) + i];
    __syncthreads();

    const long long base_cell = ((long long)blockIdx.x * G + g) * WPG;

    float2 stash[PAIR ? P : 1];
    float2 z[P];
    float scale[WPG];
    bool ok[WPG];
    float4 org[WPG];

#pragma unroll
    for (int wi = 0; wi < WPG; ++wi) {
        const long long cell = base_cell + wi;
        const bool active = cell < prm.ncells;
        const float4 o = active ? prm.origins[cell] : make_float4(0.f, 0.f, 0.f, 0.f);
        const bool sig = active && prm.status[cell] != 0;
        org[wi] = o;
        {
            float va[P], vb[P];
            sample_column<N, T>(prm.img_a, prm.H, prm.W, o.x, o.y, line, t, va);
            sample_column<N, T>(prm.img_b, prm.H, prm.W, o.z, o.w, line, t, vb);
            float2 s = make_float2(0.f, 0.f);
#pragma unroll
            for (int p = 0; p < P; ++p) {
                s.x += va[p];
                s.y += vb[p];
            }
            s = group_sum2<C>(s, s_red, g, gt);
            const float inv = 1.0f / (float)(N * N);
            const float ma = s.x * inv, mb = s.y * inv;
            float2 e = make_float2(0.f, 0.f);
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const float a = __fsub_rn(va[p], ma), b = __fsub_rn(vb[p], mb);
                z[p] = make_float2(a, b);
                e.x += a * a;
                e.y += b * b;
            }
            e = group_sum2<C>(e, s_red, g, gt);
            ok[wi] = sig && e.x > 1e-12f && e.y > 1e-12f;
            // correlate.rs:136: 1 / (n^2 * sqrt(Ea*Eb)); the factor 1/4 undoes the 2x folded
            // into each separated spectrum below (exact power-of-two scaling).
            scale[wi] = 0.25f / ((float)(N * N) * (sqrtf(e.x) * sqrtf(e.y)));
        }
        // Forward 2-D FFT: columns (lane = column, interleaved rows) ...
        fft_line_interleaved<N, T, 1>(z, t, s_roots);
#pragma unroll
        for (int k = 0; k < P; ++k) plane[(k + P * rt) * LD + line] = z[k];
        __syncthreads();
        // ... then rows (lane = row ky, interleaved columns).
#pragma unroll
        for (int q = 0; q < P; ++q) z[q] = plane[line * LD + t + T * q];
        __syncthreads();
        fft_line_interleaved<N, T, 1>(z, t, s_roots);
        // Cross spectrum from Z[k] and its Hermitian partner Z[-k]:
        //   2FA = Z + conj(Z[-k]), 2FB = -i (Z - conj(Z[-k])), C = conj(2FA) * 2FB.
#pragma unroll
        for (int k = 0; k < P; ++k) plane[line * LD + k + P * rt] = z[k];
        __syncthreads();
        {
            const int my = (N - line) % N;
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const int kx = k + P * rt;
                const float2 m = plane[my * LD + (N - kx) % N];
                const float far = z[k].x + m.x, fai = z[k].y - m.y;
                const float fbr = z[k].y + m.y, fbi = m.x - z[k].x;
                z[k] = make_float2(far * fbr + fai * fbi, far * fbi - fai * fbr);
            }
        }
        __syncthreads();
        if constexpr (PAIR) {
            if (wi == 0) {
#pragma unroll
                for (int k = 0; k < P; ++k) stash[k] = z[k];
            }
        }
    }

    if constexpr (PAIR) {
        // D = C0 + i*C1: both inverse transforms in one complex transform.
#pragma unroll
        for (int k = 0; k < P; ++k) z[k] = make_float2(stash[k].x - z[k].y, stash[k].y + z[k].x);
    }
    // Inverse 2-D FFT: rows first (block layout from the forward pass) ...
    fft_line_blocked<N, T, -1>(z, t, s_roots);
#pragma unroll
    for (int k = 0; k < P; ++k) plane[line * LD + t + T * k] = z[k];
    __syncthreads();
    // ... then columns.
#pragma unroll
    for (int q = 0; q < P; ++q) z[q] = plane[(t + T * q) * LD + line];
    __syncthreads();
    fft_line_interleaved<N, T, -1>(z, t, s_roots);
    // Lane now holds corr[y = k + P*rt][x = line]; scale as the reference does (c *= scale).
#pragma unroll
    for (int k = 0; k < P; ++k) {
        z[k].x = z[k].x * scale[0];
        z[k].y = PAIR ? z[k].y * scale[WPG - 1] : 0.0f;
        plane[(k + P * rt) * LD + line] = z[k];
    }
    __syncthreads();

    // --------------------------------------------------------------------------- find_peak
#pragma unroll
    for (int wi = 0; wi < WPG; ++wi) {
        auto at = [&](int y, int x) -> float {
            const float2 v = plane[(y % N) * LD + (x % N)];
            return wi == 0 ? v.x : v.y;
        };
        float best = -INFINITY;
        int bidx = 0x7fffffff;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const float v = wi == 0 ? z[k].x : z[k].y;
            const int idx = (k + P * rt) * N + line;
            if (v > -INFINITY) amax_combine(best, bidx, v, idx);
        }
        group_argmax<C>(best, bidx, s_red, g, gt);
        if (!(best > -INFINITY)) bidx = 0;
        const int by = bidx / N, bx = bidx % N;
        // Footprint of the primary peak (correlate.rs:242-254): half-width along +-x, +-y.
        if (gt < 4) {
            const int sy = gt == 0 ? 1 : (gt == 1 ? N - 1 : 0);
            const int sx = gt == 2 ? 1 : (gt == 3 ? N - 1 : 0);
            const float half = 0.5f * best;
            int k = 0;
            while (k < N / 2 && at(by + k * sy, bx + k * sx) > half) ++k;
            s_hw[g][gt] = k;
        }
        __syncthreads();
        const int hw = max(max(s_hw[g][0], s_hw[g][1]), max(s_hw[g][2], s_hw[g][3]));
        const int exclude = max((int)ceilf(1.5f * (float)hw), 2);
        // Highest local maximum outside the footprint (correlate.rs:255-267).
        float second = -INFINITY;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const float v = wi == 0 ? z[k].x : z[k].y;
            const int y = k + P * rt, x = line;
            if (v > second) {
                const int dy = abs(y - by), dx = abs(x - bx);
                const int cy = min(dy, N - dy), cx = min(dx, N - dx);
                if (max(cy, cx) > exclude) {
                    const bool lm = at(y + N - 1, x + N - 1) <= v && at(y + N - 1, x) <= v && at(y + N - 1, x + 1) <= v &&
                                    at(y, x + N - 1) <= v && at(y, x + 1) <= v && at(y + 1, x + N - 1) <= v &&
                                    at(y + 1, x) <= v && at(y + 1, x + 1) <= v;
                    if (lm) second = v;
                }
            }
        }
        second = group_max<C>(second, s_red, g, gt);
        if (gt == 0) {
            const long long cell = base_cell + wi;
            if (cell < prm.ncells) {
                if (ok[wi]) {
                    const float sx = subpixel(at(by, bx + N - 1), best, at(by, bx + 1));
                    const float sy = subpixel(at(by + N - 1, bx), best, at(by + 1, bx));
                    const float wx = bx >= N / 2 ? (float)bx - (float)N : (float)bx;
                    const float wy = by >= N / 2 ? (float)by - (float)N : (float)by;
                    const float pdx = __fadd_rn(wx, sx), pdy = __fadd_rn(wy, sy);
                    const float ppr = second > 0.0f ? fminf(__fdiv_rn(best, second), MAX_PPR) : MAX_PPR;
                    const float4 o = org[wi];
                    prm.raw_dx[cell] = __fadd_rn(__fsub_rn(o.z, o.x), pdx);
                    prm.raw_dy[cell] = __fadd_rn(__fsub_rn(o.w, o.y), pdy);
                    prm.raw_ppr[cell] = ppr;
                    prm.raw_flags[cell] = 0;
                } else {
                    prm.raw_dx[cell] = NAN;
                    prm.raw_dy[cell] = NAN;
                    prm.raw_ppr[cell] = 0.0f;
                    prm.raw_flags[cell] = F_NO_SIGNAL;
                }
            }
        }
        __syncthreads();
    }
}

template <int N, int T, bool PAIR, int G>
static cudaError_t launch_t(const CorrParams& p, cudaStream_t s) {
    using C = CorrCfg<N, T, PAIR, G>;
    static_assert(C::SMEM <= 227 * 1024, "shared memory");
    if (p.ncells <= 0) return cudaSuccess;
    auto kern = correlate_kernel<N, T, PAIR, G>;
    // Attribute setting is idempotent and per device; done on every launch for simplicity.
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (e != cudaSuccess) return e;
    const long long per_block = (long long)G * C::WPG;
    const long long blocks = (p.ncells + per_block - 1) / per_block;
    kern<<<(unsigned)blocks, C::THREADS, C::SMEM, s>>>(p);
    return cudaGetLastError();
}

bool corr_supported(int n) {
    switch (n) {
        case 8: case 12: case 16: case 24: case 32: case 48: case 64: case 96: case 128: return true;
        default: return false;
    }
}

cudaError_t launch_correlate(int n, const CorrParams& p, cudaStream_t s) {
    switch (n) {
        case 8: return launch_t<8, 1, true, 32>(p, s);
        case 12: return launch_t<12, 1, true, 16>(p, s);
        case 16: return launch_t<16, 1, true, 16>(p, s);
        case 24: return launch_t<24, 2, true, 4>(p, s);
        case 32: return launch_t<32, 2, true, 4>(p, s);
        case 48: return launch_t<48, 4, true, 1>(p, s);
        case 64: return launch_t<64, 4, true, 1>(p, s);
        case 96: return launch_t<96, 4, true, 1>(p, s);
        case 128: return launch_t<128, 4, false, 1>(p, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t corr_init_device() {
    float2 h[kRootTableLen];
    int off = 0;
    for (int i = 0; i < kNumRootSizes; ++i) {
        const int n = kRootSizes[i];
        for (int k = 0; k < n; ++k) {
            const double a = 2.0 * M_PI * (double)k / (double)n;
            h[off + k] = make_float2((float)std::cos(a), (float)-std::sin(a));
        }
        off += n;
    }
    return cudaMemcpyToSymbol(c_roots, h, sizeof(h));
}

}  // namespace pivb200
