// Small FFTs for square interrogation windows (N = 2^a * 3^b, N <= 128).
//
// A length-N line is handled by T lanes of one warp (T a power of two); each lane holds P = N/T
// complex values in registers. Two decompositions of the DFT are used (four-step FFT):
//
//  * interleaved input (lane t holds x[t + T*p]):
//      P-point DFT in registers, twiddle w_N^(t*k1), T-point DFT across lanes (radix-2
//      decimation in frequency over shuffles; natural lane order in, bit-reversed out).
//      Lane t ends with X[k1 + P*rev(t)], k1 = 0..P-1 (a contiguous block).
//  * block input with bit-reversed blocks (lane t holds x[P*rev(t) + p]):
//      T-point DFT across lanes (radix-2 decimation in time; bit-reversed in, natural out),
//      twiddle w_N^(p*t), P-point DFT in registers.
//      Lane t ends with X[t + T*k1] (interleaved).
//
// The first is used for the forward transforms and for the last inverse stage, the second for
// the first inverse stage, so the data never has to be re-ordered inside a lane.
//
// Unnormalized DFT, forward kernel exp(-2 pi i j k / N), inverse exp(+2 pi i j k / N) — the
// definition rustfft/realfft implement (the reference's FFT crates, rust/Cargo.lock:1644-1646,
// 1703-1705).
#pragma once

#include <cuda_runtime.h>

namespace pivb200 {

// Table of N-th roots of unity for every supported line length, rounded from f64 on the host:
// c_roots[root_off(N) + k] = (cos(2 pi k / N), -sin(2 pi k / N)).
constexpr int kRootSizes[] = {8, 12, 16, 24, 32, 48, 64, 96, 128};
constexpr int kNumRootSizes = 9;
constexpr int kRootTableLen = 8 + 12 + 16 + 24 + 32 + 48 + 64 + 96 + 128;

__host__ __device__ constexpr int root_off(int n) {
    int off = 0;
    for (int i = 0; i < kNumRootSizes; ++i) {
        if (kRootSizes[i] == n) return off;
        off += kRootSizes[i];
    }
    return -1;
}

// Defined here: the header is included by exactly one translation unit (no relocatable device code).
__constant__ float2 c_roots[kRootTableLen];

template <int N>
__device__ __forceinline__ float2 croot(int k) {
    return c_roots[root_off(N) + k];
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// a * w (DIR = +1) or a * conj(w) (DIR = -1); w is a forward root.
template <int DIR>
__device__ __forceinline__ float2 cmulw(float2 a, float2 w) {
    if constexpr (DIR > 0)
        return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
    else
        return make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}

// Multiply by -i (forward) or +i (inverse).
template <int DIR>
__device__ __forceinline__ float2 mul_mi(float2 a) {
    if constexpr (DIR > 0)
        return make_float2(a.y, -a.x);
    else
        return make_float2(-a.y, a.x);
}

// v * w_N^j (DIR = +1) or v * conj(w_N^j) (DIR = -1). Quarter and half turns are applied as the
// exact swap and sign changes they are; in unrolled loops j is a constant, so the choice costs
// nothing. (The root table holds f64 values rounded to f32, so its quarter turn carries a
// cosine of 6.1e-17 instead of 0; multiplying by it changes a result only when one component
// exceeds the other by about 2^30, so the exact form agrees except in that last bit.)
template <int N, int DIR>
__device__ __forceinline__ float2 twiddle(float2 v, int j, const float2 w) {
    if (j == 0) return v;
    if (4 * j == N) return mul_mi<DIR>(v);
    if (2 * j == N) return make_float2(-v.x, -v.y);
    if (4 * j == 3 * N) return mul_mi<-DIR>(v);
    return cmulw<DIR>(v, w);
}

template <int R, int DIR>
__device__ __forceinline__ void butterfly(float2 (&t)[R]) {
    if constexpr (R == 2) {
        float2 a = t[0], b = t[1];
        t[0] = cadd(a, b);
        t[1] = csub(a, b);
    } else if constexpr (R == 4) {
        float2 a0 = cadd(t[0], t[2]), a1 = csub(t[0], t[2]);
        float2 b0 = cadd(t[1], t[3]), b1 = mul_mi<DIR>(csub(t[1], t[3]));
        t[0] = cadd(a0, b0);
        t[1] = cadd(a1, b1);
        t[2] = csub(a0, b0);
        t[3] = csub(a1, b1);
    } else {
        static_assert(R == 3, "radix");
        constexpr float kS3 = 0.866025403784438646763723f;  // sqrt(3)/2
        float2 s = cadd(t[1], t[2]), d = csub(t[1], t[2]);
        float2 m = make_float2(t[0].x - 0.5f * s.x, t[0].y - 0.5f * s.y);
        float2 r = mul_mi<DIR>(make_float2(kS3 * d.x, kS3 * d.y));
        t[0] = cadd(t[0], s);
        t[1] = cadd(m, r);
        t[2] = csub(m, r);
    }
}

// out[k] = sum_j in[j*IS] * w_LEN^(DIR*j*k), k < LEN (out-of-place, fully unrolled; every index is
// a compile-time constant so the arrays live in registers). Roots come from the N-th root table.
template <int N, int LEN, int IS, int DIR>
__device__ __forceinline__ void dft_rec(const float2* in, float2* out) {
    if constexpr (LEN == 1) {
        out[0] = in[0];
    } else {
        constexpr int R = (LEN % 4 == 0) ? 4 : ((LEN % 2 == 0) ? 2 : 3);
        constexpr int M = LEN / R;
#pragma unroll
        for (int q = 0; q < R; ++q) dft_rec<N, M, IS * R, DIR>(in + q * IS, out + q * M);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            float2 t[R];
#pragma unroll
            for (int q = 0; q < R; ++q) {
                float2 v = out[q * M + k];
                if (q > 0 && k > 0) {
                    const int j = (q * k * (N / LEN)) % N;
                    v = twiddle<N, DIR>(v, j, croot<N>(j));
                }
                t[q] = v;
            }
            butterfly<R, DIR>(t);
#pragma unroll
            for (int q = 0; q < R; ++q) out[k + q * M] = t[q];
        }
    }
}

// In-register P-point DFT, natural order in and out.
template <int N, int P, int DIR>
__device__ __forceinline__ void dft_reg(float2 (&x)[P]) {
    float2 y[P];
    dft_rec<N, P, 1, DIR>(x, y);
#pragma unroll
    for (int i = 0; i < P; ++i) x[i] = y[i];
}

template <int T>
__device__ __forceinline__ int bitrev(int t) {
    int r = 0;
#pragma unroll
    for (int b = 1; b < T; b <<= 1) {
        r <<= 1;
        if (t & b) r |= 1;
    }
    return r;
}

// T-point DFT across the T lanes of a line, natural lane order in, bit-reversed out (DIF).
// Radix-2 step over lane pairs (t, t ^ h): the lower lane keeps x + o, the upper (o - x) * w.
// Both are written as one signed add fma(s, x, o) (s = +1 or -1, an exact single rounding like a
// plain add) and one complex multiply by w, with w = 1 on the lower lane (exact up to the sign of
// a zero), so a lane issues no instructions for the other lane's formula.
// The stage twiddle of the upper lane is w_N^((t mod h) * N/(2h)): 1 for h = 1, 1 or a quarter
// turn for h = 2, applied exactly (twiddle()); other stages multiply.
template <int N, int T, int P, int DIR>
__device__ __forceinline__ void xlane_dif(float2 (&x)[P], int t, const float2* s_roots) {
#pragma unroll
    for (int h = T / 2; h >= 1; h >>= 1) {
        const bool upper = (t & h) != 0;
        const float sg = upper ? -1.0f : 1.0f;
        if (h <= 2) {
            const bool quarter = h == 2 && upper && (t & 1);  // w = w_N^(N/4)
#pragma unroll
            for (int i = 0; i < P; ++i) {
                float2 o;
                o.x = __shfl_xor_sync(0xffffffffu, x[i].x, h);
                o.y = __shfl_xor_sync(0xffffffffu, x[i].y, h);
                const float2 v = make_float2(fmaf(sg, x[i].x, o.x), fmaf(sg, x[i].y, o.y));
                x[i] = quarter ? mul_mi<DIR>(v) : v;
            }
        } else {
            const float2 w = upper ? s_roots[(t & (h - 1)) * (N / (2 * h))] : make_float2(1.0f, 0.0f);
#pragma unroll
            for (int i = 0; i < P; ++i) {
                float2 o;
                o.x = __shfl_xor_sync(0xffffffffu, x[i].x, h);
                o.y = __shfl_xor_sync(0xffffffffu, x[i].y, h);
                x[i] = cmulw<DIR>(make_float2(fmaf(sg, x[i].x, o.x), fmaf(sg, x[i].y, o.y)), w);
            }
        }
    }
}

// T-point DFT across the T lanes of a line, bit-reversed lane order in, natural out (DIT).
// SIGNED: the upper lane of each pair first multiplies by w (w = 1 on the lower lane), then the
// lower keeps v + o and the upper o - v, again as one signed add. Otherwise each lane selects
// between the two formulas. Both give the same values (up to the sign of a zero); which one
// schedules better depends on the window size (measured: the select form for 32 and 64 points,
// the signed form elsewhere).
template <int N, int T, int P, int DIR, bool SIGNED>
__device__ __forceinline__ void xlane_dit(float2 (&x)[P], int t, const float2* s_roots) {
#pragma unroll
    for (int h = 1; h < T; h <<= 1) {
        const bool upper = (t & h) != 0;
        // the upper lane's twiddle: 1 for h = 1, 1 or a quarter turn for h = 2 (exact forms)
        const bool quarter = h == 2 && upper && (t & 1);
        auto tw = [&](float2 v, float2 w) -> float2 {
            if (h == 1) return v;
            if (h == 2) return quarter ? mul_mi<DIR>(v) : v;
            return cmulw<DIR>(v, w);
        };
        if constexpr (SIGNED) {
            const float sg = upper ? -1.0f : 1.0f;
            const float2 w = upper ? s_roots[(t & (h - 1)) * (N / (2 * h))] : make_float2(1.0f, 0.0f);
#pragma unroll
            for (int i = 0; i < P; ++i) {
                const float2 v = tw(x[i], w);
                float2 o;
                o.x = __shfl_xor_sync(0xffffffffu, v.x, h);
                o.y = __shfl_xor_sync(0xffffffffu, v.y, h);
                x[i] = make_float2(fmaf(sg, v.x, o.x), fmaf(sg, v.y, o.y));
            }
        } else {
            const float2 w = s_roots[(t & (h - 1)) * (N / (2 * h))];
#pragma unroll
            for (int i = 0; i < P; ++i) {
                float2 v = upper ? tw(x[i], w) : x[i];
                float2 o;
                o.x = __shfl_xor_sync(0xffffffffu, v.x, h);
                o.y = __shfl_xor_sync(0xffffffffu, v.y, h);
                x[i] = upper ? csub(o, v) : cadd(v, o);
            }
        }
    }
}

// Interleaved input -> lane t holds X[k1 + P*rev(t)].
template <int N, int T, int DIR>
__device__ __forceinline__ void fft_line_interleaved(float2 (&x)[N / T], int t, const float2* s_roots) {
    constexpr int P = N / T;
    dft_reg<N, P, DIR>(x);
    if constexpr (T > 1) {
#pragma unroll
        for (int k = 1; k < P; ++k) x[k] = cmulw<DIR>(x[k], s_roots[t * k]);
        xlane_dif<N, T, P, DIR>(x, t, s_roots);
    }
}

// Bit-reversed block input -> lane t holds X[t + T*k1].
template <int N, int T, int DIR>
__device__ __forceinline__ void fft_line_blocked(float2 (&x)[N / T], int t, const float2* s_roots) {
    constexpr int P = N / T;
    if constexpr (T > 1) {
        xlane_dit<N, T, P, DIR, !(N == 32 || N == 64)>(x, t, s_roots);
#pragma unroll
        for (int p = 1; p < P; ++p) x[p] = cmulw<DIR>(x[p], s_roots[p * t]);
    }
    dft_reg<N, P, DIR>(x);
}

// Two lines at once (the two windows of a pair), stage by stage: the same operations per value as
// two calls of fft_line_interleaved (so the same results), ordered so that one line's shuffles
// overlap the other's arithmetic. Measured per window size, it is used where it is faster: 64
// points on four lanes (2.37 -> 2.20 ms for the c5 64 px pass; 32 points on two lanes 2.00 ->
// 2.05, 96 points 2.247 -> 2.256).
template <int N, int T, int DIR>
__device__ __forceinline__ void fft_line_interleaved2(float2 (&x)[N / T], float2 (&y)[N / T], int t,
                                                      const float2* s_roots) {
    constexpr int P = N / T;
    dft_reg<N, P, DIR>(x);
    dft_reg<N, P, DIR>(y);
    if constexpr (T > 1) {
#pragma unroll
        for (int k = 1; k < P; ++k) {
            const float2 w = s_roots[t * k];
            x[k] = cmulw<DIR>(x[k], w);
            y[k] = cmulw<DIR>(y[k], w);
        }
#pragma unroll
        for (int h = T / 2; h >= 1; h >>= 1) {
            const bool upper = (t & h) != 0;
            const float sg = upper ? -1.0f : 1.0f;
            if (h <= 2) {
                const bool quarter = h == 2 && upper && (t & 1);
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    float2 o, q;
                    o.x = __shfl_xor_sync(0xffffffffu, x[i].x, h);
                    o.y = __shfl_xor_sync(0xffffffffu, x[i].y, h);
                    q.x = __shfl_xor_sync(0xffffffffu, y[i].x, h);
                    q.y = __shfl_xor_sync(0xffffffffu, y[i].y, h);
                    const float2 v = make_float2(fmaf(sg, x[i].x, o.x), fmaf(sg, x[i].y, o.y));
                    const float2 u = make_float2(fmaf(sg, y[i].x, q.x), fmaf(sg, y[i].y, q.y));
                    x[i] = quarter ? mul_mi<DIR>(v) : v;
                    y[i] = quarter ? mul_mi<DIR>(u) : u;
                }
            } else {
                const float2 w = upper ? s_roots[(t & (h - 1)) * (N / (2 * h))] : make_float2(1.0f, 0.0f);
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    float2 o, q;
                    o.x = __shfl_xor_sync(0xffffffffu, x[i].x, h);
                    o.y = __shfl_xor_sync(0xffffffffu, x[i].y, h);
                    q.x = __shfl_xor_sync(0xffffffffu, y[i].x, h);
                    q.y = __shfl_xor_sync(0xffffffffu, y[i].y, h);
                    x[i] = cmulw<DIR>(make_float2(fmaf(sg, x[i].x, o.x), fmaf(sg, x[i].y, o.y)), w);
                    y[i] = cmulw<DIR>(make_float2(fmaf(sg, y[i].x, q.x), fmaf(sg, y[i].y, q.y)), w);
                }
            }
        }
    }
}

// Two bit-reversed block lines at once (the two windows of a pair), stage by stage: the same
// operations per value as two calls of fft_line_blocked (so the same results), ordered so that
// one line's shuffles overlap the other's arithmetic.
template <int N, int T, int DIR>
__device__ __forceinline__ void fft_line_blocked2(float2 (&x)[N / T], float2 (&y)[N / T], int t,
                                                  const float2* s_roots) {
    constexpr int P = N / T;
    constexpr bool SIGNED = !(N == 32 || N == 64);
    if constexpr (T > 1) {
#pragma unroll
        for (int h = 1; h < T; h <<= 1) {
            const bool upper = (t & h) != 0;
            const bool quarter = h == 2 && upper && (t & 1);
            auto tw = [&](float2 v, float2 w) -> float2 {
                if (h == 1) return v;
                if (h == 2) return quarter ? mul_mi<DIR>(v) : v;
                return cmulw<DIR>(v, w);
            };
            if constexpr (SIGNED) {
                const float sg = upper ? -1.0f : 1.0f;
                const float2 w = upper ? s_roots[(t & (h - 1)) * (N / (2 * h))] : make_float2(1.0f, 0.0f);
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    const float2 v = tw(x[i], w), u = tw(y[i], w);
                    float2 o, q;
                    o.x = __shfl_xor_sync(0xffffffffu, v.x, h);
                    o.y = __shfl_xor_sync(0xffffffffu, v.y, h);
                    q.x = __shfl_xor_sync(0xffffffffu, u.x, h);
                    q.y = __shfl_xor_sync(0xffffffffu, u.y, h);
                    x[i] = make_float2(fmaf(sg, v.x, o.x), fmaf(sg, v.y, o.y));
                    y[i] = make_float2(fmaf(sg, u.x, q.x), fmaf(sg, u.y, q.y));
                }
            } else {
                const float2 w = s_roots[(t & (h - 1)) * (N / (2 * h))];
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    const float2 v = upper ? tw(x[i], w) : x[i];
                    const float2 u = upper ? tw(y[i], w) : y[i];
                    float2 o, q;
                    o.x = __shfl_xor_sync(0xffffffffu, v.x, h);
                    o.y = __shfl_xor_sync(0xffffffffu, v.y, h);
                    q.x = __shfl_xor_sync(0xffffffffu, u.x, h);
                    q.y = __shfl_xor_sync(0xffffffffu, u.y, h);
                    x[i] = upper ? csub(o, v) : cadd(v, o);
                    y[i] = upper ? csub(q, u) : cadd(u, q);
                }
            }
        }
#pragma unroll
        for (int p = 1; p < P; ++p) {
            const float2 w = s_roots[p * t];
            x[p] = cmulw<DIR>(x[p], w);
            y[p] = cmulw<DIR>(y[p], w);
        }
    }
    dft_reg<N, P, DIR>(x);
    dft_reg<N, P, DIR>(y);
}

}  // namespace pivb200
