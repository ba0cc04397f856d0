// Shared device helpers for the B200 PIV path.
//
// Where the reference computes in f64 (integral-image window statistics, preprocess.rs:76-125,
// 199-216) the fast path here uses no FP64: box sums are exact int64 fixed-point sums (integer
// addition is associative, so any parallel order gives the same bits), and the few divisions,
// squares and square roots that turn them into a mean and a standard deviation run in
// double-float arithmetic (an unevaluated sum hi + lo of two f32 values, ~48 significant bits).
// The final f32 values then agree with the reference's f64-then-round results except when the
// exact value lies within ~2^-48 (relative) of an f32 rounding boundary.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pivb200 {

// field.rs:6-20
constexpr uint8_t F_NO_SIGNAL = 1u << 0;
constexpr uint8_t F_LOW_PPR = 1u << 1;
constexpr uint8_t F_MEDIAN_OUTLIER = 1u << 2;
constexpr uint8_t F_REPLACED = 1u << 3;
constexpr uint8_t F_OUT_OF_RANGE = 1u << 4;
constexpr uint8_t F_INVALID = F_NO_SIGNAL | F_LOW_PPR | F_MEDIAN_OUTLIER | F_OUT_OF_RANGE;

constexpr float MAX_PPR = 1000.0f;  // correlate.rs:24

// Grid of interrogation windows (grid.rs:8-16).
struct GridP {
    int32_t window, step, nx, ny, x0, y0;
};

// ---------------------------------------------------------------------------------------------
// Double-float arithmetic (error-free transformations; Dekker/Knuth two-sum and FMA two-product).
// The __f*_rn intrinsics are never contracted or reassociated by the compiler.
// ---------------------------------------------------------------------------------------------
struct dfloat {
    float hi, lo;
};

__device__ __forceinline__ dfloat dd_two_sum(float a, float b) {
    float s = __fadd_rn(a, b);
    float bb = __fsub_rn(s, a);
    float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return {s, e};
}

__device__ __forceinline__ dfloat dd_quick(float a, float b) {
    float s = __fadd_rn(a, b);
    return {s, __fsub_rn(b, __fsub_rn(s, a))};
}

__device__ __forceinline__ dfloat dd_two_prod(float a, float b) {
    float p = __fmul_rn(a, b);
    return {p, __fmaf_rn(a, b, -p)};
}

__device__ __forceinline__ dfloat dd_add(dfloat x, dfloat y) {
    dfloat s = dd_two_sum(x.hi, y.hi);
    dfloat t = dd_two_sum(x.lo, y.lo);
    float e = __fadd_rn(s.lo, t.hi);
    dfloat u = dd_quick(s.hi, e);
    return dd_quick(u.hi, __fadd_rn(u.lo, t.lo));
}

__device__ __forceinline__ dfloat dd_neg(dfloat x) { return {-x.hi, -x.lo}; }

__device__ __forceinline__ dfloat dd_mul(dfloat x, dfloat y) {
    dfloat p = dd_two_prod(x.hi, y.hi);
    float e = __fadd_rn(p.lo, __fadd_rn(__fmul_rn(x.hi, y.lo), __fmul_rn(x.lo, y.hi)));
    return dd_quick(p.hi, e);
}

// x / d for a plain float d.
__device__ __forceinline__ dfloat dd_div_f(dfloat x, float d) {
    float q1 = __fdiv_rn(x.hi, d);
    dfloat p = dd_two_prod(q1, d);
    float r = __fdiv_rn(__fadd_rn(__fsub_rn(__fsub_rn(x.hi, p.hi), p.lo), x.lo), d);
    return dd_quick(q1, r);
}

__device__ __forceinline__ dfloat dd_scale2(dfloat x, int k) {
    return {scalbnf(x.hi, k), scalbnf(x.lo, k)};
}

__device__ __forceinline__ dfloat dd_from_i64(long long v) {
    float hi = __ll2float_rn(v);
    long long rem = v - __float2ll_rn(hi);
    return dd_quick(hi, __ll2float_rn(rem));
}

__device__ __forceinline__ dfloat dd_sqrt(dfloat x) {
    if (!(x.hi > 0.0f)) return {0.0f, 0.0f};
    float s = __fsqrt_rn(x.hi);
    dfloat p = dd_two_prod(s, s);
    float r = __fdiv_rn(__fadd_rn(__fsub_rn(__fsub_rn(x.hi, p.hi), p.lo), x.lo), __fmul_rn(2.0f, s));
    return dd_quick(s, r);
}

__device__ __forceinline__ float dd_to_float(dfloat x) { return __fadd_rn(x.hi, x.lo); }

// ---------------------------------------------------------------------------------------------
// Exact fixed-point box statistics.
//
// A value v is quantised to q1 = round(v * 2^s1) and its exact square v*v (a two-product) to
// q2 = round(hi * 2^s2) + round(lo * 2^s2). The scales are chosen from the frame's largest |v|
// so that a sum over `count` values cannot overflow int64.
// ---------------------------------------------------------------------------------------------
struct FixScale {
    int s1, s2;
    // 2^s1 and 2^s2 as floats when 0 <= s <= 127: multiplying a finite float by 2^s with s >= 0
    // is exact up to overflow, where it rounds to +-inf as scalbnf does, so the product equals
    // scalbnf(v, s) bit for bit. Outside that range the quantisers fall back to scalbnf.
    float m1, m2;
    bool fast1, fast2;
};

__device__ __forceinline__ float pow2f(int s) { return __int_as_float((s + 127) << 23); }

// Largest exponent e with 2^e >= maxabs, then scales that keep count * 2^(e+s) <= 2^62.
__device__ __forceinline__ FixScale fix_scale(float maxabs, long long count) {
    FixScale fs{0, 0, 1.0f, 1.0f, true, true};
    if (!(maxabs > 0.0f) || !isfinite(maxabs)) return fs;
    int e;
    float m = frexpf(maxabs, &e);  // maxabs = m * 2^e, m in [0.5, 1)
    (void)m;
    int lc = 0;
    while ((1ll << lc) < count && lc < 62) ++lc;
    fs.s1 = 62 - lc - e;
    fs.s2 = 62 - lc - 2 * e;
    fs.fast1 = fs.s1 >= 0 && fs.s1 <= 127;
    fs.fast2 = fs.s2 >= 0 && fs.s2 <= 127;
    fs.m1 = fs.fast1 ? pow2f(fs.s1) : 1.0f;
    fs.m2 = fs.fast2 ? pow2f(fs.s2) : 1.0f;
    return fs;
}

__device__ __forceinline__ long long fix_q1(float v, const FixScale& fs) {
    return __float2ll_rn(fs.fast1 ? __fmul_rn(v, fs.m1) : scalbnf(v, fs.s1));
}

__device__ __forceinline__ long long fix_q2(float v, const FixScale& fs) {
    dfloat sq = dd_two_prod(v, v);
    if (fs.fast2) return __float2ll_rn(__fmul_rn(sq.hi, fs.m2)) + __float2ll_rn(__fmul_rn(sq.lo, fs.m2));
    return __float2ll_rn(scalbnf(sq.hi, fs.s2)) + __float2ll_rn(scalbnf(sq.lo, fs.s2));
}

// IntegralImage::stats (preprocess.rs:114-125) from exact sums: mean and standard deviation as
// the reference's f64 arithmetic would round them to f32.
__device__ __forceinline__ void fix_stats(long long sum1, long long sum2, const FixScale& fs, float count,
                                          float* mean_out, float* std_out) {
    dfloat mean = dd_div_f(dd_scale2(dd_from_i64(sum1), -fs.s1), count);
    dfloat ex2 = dd_div_f(dd_scale2(dd_from_i64(sum2), -fs.s2), count);
    dfloat var = dd_add(ex2, dd_neg(dd_mul(mean, mean)));
    *mean_out = dd_to_float(mean);
    *std_out = dd_to_float(dd_sqrt(var));
}

// Rust f32::clamp (NaN passes through).
__device__ __forceinline__ float rclamp(float x, float lo, float hi) {
    if (x < lo) return lo;
    if (x > hi) return hi;
    return x;
}

}  // namespace pivb200
