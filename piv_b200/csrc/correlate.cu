// Fused per-window FFT cross-correlation and peak fit (FP32 plain path).
//
// Reference semantics: CorrelationPlan::correlate (correlate.rs:99-139), load_window
// (correlate.rs:182-210), find_peak (correlate.rs:215-303) and the pair assembly of
// PivAnalyzer::pass (multipass.rs:242-259).
//
// Work decomposition (one thread group = N*T threads, one PAIR of windows per group):
//   1. both windows of the pair are sampled (bilinear, the reference's f32 operation order, no
//      FMA) straight into registers, each as one complex plane z = a + i*b (frame A's window in
//      the real part, frame B's in the imaginary part); lane (x, t) holds column x at rows
//      t + T*p (32 and 64 px: the block of rows P*rev(t) + p, sampled one new row at a time), so
//      each load instruction reads contiguous image rows;
//   2. mean removal and energies (one group reduction of 4 sums for both windows), 2-D FFT of
//      both planes at once: columns in registers, transpose through shared memory, rows in
//      registers;
//   3. each plane's two real spectra are separated with the Hermitian partner Z[-k] (one
//      shared-memory exchange) and the cross spectrum conj(FA)*FB formed in registers;
//   4. both cross spectra are Hermitian, so their inverse transforms are packed into ONE complex
//      inverse 2-D FFT (real part = first correlation plane, imaginary part = second);
//   5. the scaled planes go to shared memory; argmax (lowest row-major index on ties), the
//      half-width footprint, the second local maximum (a vectorised 3x3 maximum) and the 3-point
//      Gaussian fit follow.
// The 128 px window runs one window per group; its real inverse runs as half-size stages (rows
// 0..N/2, then pairs of real columns per complex line).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>

#include "common.cuh"
#include "fft.cuh"
#include "kernels.h"
#include "window.cuh"

namespace pivb200 {

// Compile-time shape of one correlation kernel: window N, lanes per line T, window pairs or
// single windows, groups per CTA G, minimum resident CTAs per SM (register cap), sampler.
// G and MINB only change the launch geometry, never the arithmetic; N, T and PAIR fix the FFT
// decomposition and therefore the rounding of the results.
template <int N_, int T_, bool PAIR_, int G_, int MINB_, bool SHFL_ = false, bool DEFORM_ = false>
struct CorrCfg {
    static constexpr int N = N_, T = T_, G = G_, MINB = MINB_;
    static constexpr bool PAIR = PAIR_, SHFL_SAMPLE = SHFL_, DEFORM = DEFORM_;
    // 32 and 64 px window pairs (uniform and deformed) sample in the block layout (lane t holds
    // rows P*rev(t) + p) and run the column pass of the forward FFT from it (bit-reversed blocks
    // in, lane t ends with the frequency rows t + T*k); every other configuration samples
    // interleaved rows (t + T*p).
    static constexpr bool BLOCK = PAIR && (N_ == 32 || N_ == 64);
    static constexpr int P = N / T;
    static constexpr int NT = N * T;
    static constexpr int THREADS = G * NT;
    static constexpr int WPG = PAIR ? 2 : 1;
    // Shared-memory plane layout (in float2 units), chosen so that every access pattern of a
    // half-warp (16 lanes = 16/T lines x T lanes) hits 16 distinct 8-byte bank pairs:
    //   A(row, col) = row*LD + (row/P)*Q + col           transposes, correlation plane
    //   B(ky, kx)   = ky*LD + (ky/P)*Q + kx + (kx/P)      Hermitian-partner exchange (T > 1)
    // with LD = N + 1 for T = 1; otherwise LD >= N + T - 1, LD = T (mod 16) (lines of a
    // half-warp step by T banks, its T lanes fill the gap) and Q making a block of P rows step
    // by 16/T bank pairs.
    static constexpr int LD = (T == 1) ? N + 1 : ((N + T - 1 + 15 - T) / 16) * 16 + T;
    static constexpr int Q = (T == 1) ? 0 : ((16 / T - (P * LD) % 16) % 16 + 16) % 16;
    static constexpr int PLANE_ELEMS = ((N * LD + (T - 1) * Q) + 1) / 2 * 2;
    // Shuffle segment: largest power of two dividing NT, at most a warp.
    static constexpr int SW = (NT % 32 == 0) ? 32 : (NT % 16 == 0) ? 16 : (NT % 8 == 0) ? 8 : (NT % 4 == 0) ? 4 : (NT % 2 == 0) ? 2 : 1;
    static constexpr int NSEG = NT / SW;
    // plane0: float2 N x LD; plane1: float2 (PAIR) or float (single) N x LD.
    static constexpr size_t PLANE0 = sizeof(float2) * (size_t)PLANE_ELEMS;
    static constexpr size_t PLANE1 = ((PAIR ? sizeof(float2) : sizeof(float)) * (size_t)PLANE_ELEMS + 15) / 16 * 16;
    __host__ __device__ static constexpr int A(int row, int col) { return row * LD + (row / P) * Q + col; }
    // The first transpose (column spectra -> rows): A, except for the block layout on T = 2 lanes,
    // whose stores (rows t + 2k of eight columns per half-warp) would meet its loads' layout on
    // shared banks; there rows of N are rotated by 2 g(row), g(row) = (row/2 mod 4) + 4 (row mod 2),
    // so that both the stores and the loads (eight rows by columns t + 2q) of a half-warp hit 16
    // distinct bank pairs.
    __host__ __device__ static constexpr int AF(int row, int col) {
        return (BLOCK && T == 2) ? row * N + ((col + 2 * (((row >> 1) & 3) + 4 * (row & 1))) & (N - 1)) : A(row, col);
    }
    __host__ __device__ static constexpr int B(int ky, int kx) {
        return T == 1 ? ky * LD + kx : ky * LD + (ky / P) * Q + kx + kx / P;
    }
    // Single windows (the N = 128 inverse through half-size stages, T2 = 2T lanes per line):
    //   BS(ky, kx)  the spectrum, rows of N + 1 (= 1 mod 16) with each 16-column chunk rotated by
    //               2 * (chunk index), so that both the forward stores (4 rows x T lanes) and the
    //               half-warp reads of the inverse (2 rows x T2 lanes, and their Hermitian
    //               partners) hit 16 distinct bank pairs;
    //   YO(r, x)    the half-inverse rows 0..N/2, x XOR f(r) with f(r) = 8 (r odd) | (r & 6):
    //               two adjacent rows by T2 lanes, and eight adjacent rows by two columns, each
    //               hit 16 distinct bank pairs;
    //   CP(y, x)    the correlation plane and its vertical 3-maxima (float), rows of N plus 4 per
    //               block of 16 rows: a warp's 8 row blocks x 4 columns hit 32 distinct banks.
    // CP lives in plane0 after the YO rows (CP_OFF floats), the 3-maxima in plane1.
    __host__ __device__ static constexpr int BS(int ky, int kx) {
        return ky * (N + 1) + ((kx & ~15) | ((kx + 2 * (kx >> 4)) & 15));
    }
    __host__ __device__ static constexpr int YO(int r, int x) { return r * N + (x ^ (((r & 1) << 3) | (r & 6))); }
    __host__ __device__ static constexpr int CP(int y, int x) { return y * N + x + 4 * (y >> 4); }
    static constexpr int CP_OFF = 2 * (N / 2 + 1) * N;
    static_assert(!(BLOCK && T == 2) || N * N <= PLANE_ELEMS, "first-transpose plane");
    static_assert(PAIR || (N == 128 && BS(N - 1, N - 1) < PLANE_ELEMS &&
                           CP_OFF + CP(N - 1, N - 1) < 2 * PLANE_ELEMS &&
                           sizeof(float) * (size_t)(CP(N - 1, N - 1) + 1) <= PLANE1),
                  "single-window planes");
    static constexpr size_t SMEM = (size_t)G * (PLANE0 + PLANE1) + sizeof(float2) * N + sizeof(float) * (size_t)G * NSEG * 4 +
                                   (DEFORM ? sizeof(float) * N : 0) + 64;
};

// ---------------------------------------------------------------------------------------------
// Barrier of one group (the N*T threads of a window pair). Groups share nothing in shared memory
// but the read-only twiddles, so they need not wait for each other: a named barrier per group
// when a group is whole warps, a warp barrier when groups tile a warp (a warp's groups then wait
// together), the CTA barrier otherwise.
// ---------------------------------------------------------------------------------------------
template <class C>
__device__ __forceinline__ void group_sync(int g) {
    if constexpr (C::G > 1 && C::G <= 15 && C::NT % 32 == 0) {
        asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(C::NT) : "memory");
    } else if constexpr (C::G > 1 && C::NT <= 32 && 32 % C::NT == 0) {
        __syncwarp();
    } else {
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Group reductions (segments of SW lanes by shuffles, then NSEG partials through shared memory).
// Every thread of the group returns the same value; the combination order is fixed.
// ---------------------------------------------------------------------------------------------
template <class C>
__device__ __forceinline__ float4 group_sum4(float4 v, float* s_red, int g, int gt) {
    constexpr int SW = C::SW, NSEG = C::NSEG;
#pragma unroll
    for (int o = SW / 2; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
        v.w += __shfl_xor_sync(0xffffffffu, v.w, o);
    }
    if constexpr (NSEG == 1) {
        return v;
    } else {
        float4* r = reinterpret_cast<float4*>(s_red) + g * NSEG;
        if (gt % SW == 0) r[gt / SW] = v;
        group_sync<C>(g);
        float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int i = 0; i < NSEG; ++i) {
            const float4 q = r[i];
            s.x += q.x;
            s.y += q.y;
            s.z += q.z;
            s.w += q.w;
        }
        group_sync<C>(g);
        return s;
    }
}

template <class C>
__device__ __forceinline__ float2 group_max2(float2 v, float* s_red, int g, int gt) {
    constexpr int SW = C::SW, NSEG = C::NSEG;
#pragma unroll
    for (int o = SW / 2; o > 0; o >>= 1) {
        v.x = fmaxf(v.x, __shfl_xor_sync(0xffffffffu, v.x, o));
        v.y = fmaxf(v.y, __shfl_xor_sync(0xffffffffu, v.y, o));
    }
    if constexpr (NSEG == 1) {
        return v;
    } else {
        float2* r = reinterpret_cast<float2*>(s_red) + g * NSEG * 2;
        if (gt % SW == 0) r[gt / SW] = v;
        group_sync<C>(g);
        float2 s = make_float2(-INFINITY, -INFINITY);
#pragma unroll
        for (int i = 0; i < NSEG; ++i) {
            s.x = fmaxf(s.x, r[i].x);
            s.y = fmaxf(s.y, r[i].y);
        }
        group_sync<C>(g);
        return s;
    }
}

template <class C>
__device__ __forceinline__ void group_argmax(float& v, int& idx, float* s_red, int g, int gt) {
    constexpr int SW = C::SW, NSEG = C::NSEG;
#pragma unroll
    for (int o = SW / 2; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        amax_combine(v, idx, ov, oi);
    }
    if constexpr (NSEG > 1) {
        float2* r = reinterpret_cast<float2*>(s_red) + g * NSEG * 2;
        if (gt % SW == 0) r[gt / SW] = make_float2(v, __int_as_float(idx));
        group_sync<C>(g);
        float bv = -INFINITY;
        int bi = 0x7fffffff;
#pragma unroll
        for (int i = 0; i < NSEG; ++i) amax_combine(bv, bi, r[i].x, __float_as_int(r[i].y));
        group_sync<C>(g);
        v = bv;
        idx = bi;
    }
}

// Rows of the lane with block rt (rows P*rt .. P*rt + P - 1) that lie outside the primary
// peak's footprint: row y qualifies when its circular distance from `by` exceeds `ex`, or every
// row does when the lane's column distance `cx` exceeds `ex`. Bit k of the result is row
// P*rt + k. The rows within `ex` of `by` form one circular interval, at most two linear ones.
template <int N, int P>
__device__ __forceinline__ unsigned eligible_rows(int by, int ex, int cx, int rt) {
    static_assert(P <= 32, "row mask");
    constexpr unsigned all = (unsigned)((1ull << P) - 1ull);
    if constexpr (N <= 32) {
        // the whole column in one word: rotate a band of 2 ex + 1 bits to start at by - ex
        constexpr unsigned long long full = (1ull << N) - 1ull;
        unsigned long long near = full;
        if (2 * ex + 1 < N) {
            const unsigned long long x = ((1ull << (2 * ex + 1)) - 1ull) << ((by - ex + N) % N);
            near = (x | (x >> N)) & full;
        }
        const unsigned long long el = cx > ex ? full : (~near & full);
        return (unsigned)(el >> (P * rt)) & all;
    }
    if (cx > ex) return all;
    if (2 * ex + 1 >= N) return 0u;  // the footprint covers the whole column
    const int r0 = P * rt;
    auto span = [&](int lo, int hi) -> unsigned {  // lane bits of the rows lo..hi
        const int a = max(lo - r0, 0), b = min(hi - r0, P - 1);
        return a > b ? 0u : (unsigned)(((1ull << (b - a + 1)) - 1ull) << a);
    };
    const int lo = by - ex, hi = by + ex;  // not both outside [0, N): 2 ex + 1 < N
    const unsigned near = lo < 0 ? (span(0, hi) | span(lo + N, N - 1))
                                 : (hi >= N ? (span(0, hi - N) | span(lo, N - 1)) : span(lo, hi));
    return ~near & all;
}

// Separates Z and its Hermitian partner M = Z[-k] into the cross spectrum (times 4):
//   2FA = Z + conj(M), 2FB = -i (Z - conj(M)), C = conj(2FA) * 2FB.
__device__ __forceinline__ float2 cross4(float2 z, float2 m) {
    const float far = z.x + m.x, fai = z.y - m.y;
    const float fbr = z.y + m.y, fbi = m.x - z.x;
    return make_float2(far * fbr + fai * fbi, far * fbi - fai * fbr);
}

// One CTA's work: G window pairs (or single windows) of one item, `block` counting the item's
// CTAs; `sbase` is the CTA's dynamic shared memory (at least C::SMEM bytes).
template <class C>
__device__ __forceinline__ void correlate_body(const CorrParams& prm, int block, char* sbase) {
    constexpr int N = C::N, T = C::T, G = C::G, P = C::P, NT = C::NT, WPG = C::WPG;
    constexpr bool PAIR = C::PAIR;
    const int tid = threadIdx.x;
    const int g = tid / NT;
    const int gt = tid - g * NT;
    const int line = gt / T;
    const int t = gt - line * T;
    const int rt = bitrev<T>(t);
    float2* plane0 = reinterpret_cast<float2*>(sbase + (size_t)g * (C::PLANE0 + C::PLANE1));
    char* plane1_raw = sbase + (size_t)g * (C::PLANE0 + C::PLANE1) + C::PLANE0;
    float2* s_roots = reinterpret_cast<float2*>(sbase + (size_t)G * (C::PLANE0 + C::PLANE1));
    float* s_red = reinterpret_cast<float*>(s_roots + N);
    float* s_ramp = s_red + G * C::NSEG * 4;  // c / (N - 1) for c < N (deformed windows only)
    __shared__ int s_hw[G][8];

    for (int i = tid; i < N; i += C::THREADS) {
        s_roots[i] = c_roots[root_off(N) + i];
        if constexpr (C::DEFORM) s_ramp[i] = __fdiv_rn((float)i, (float)(N - 1));
    }
    __syncthreads();

    const long long base_cell = ((long long)block * G + g) * WPG;
    float4 org[WPG];  // uniform shift: origins; deformed: (D(centre).x, D(centre).y, -, -)
    bool ok[WPG];
    float scale[WPG];
    float2 z0[P];
    float2 z1[PAIR ? P : 1];

    // ------------------------------------------------------------------ sampling and moments
#pragma unroll
    for (int wi = 0; wi < WPG; ++wi) {
        const long long cell = base_cell + wi;
        const bool active = cell < prm.ncells;
        if constexpr (!C::DEFORM) org[wi] = active ? prm.origins[cell] : make_float4(0.f, 0.f, 0.f, 0.f);
        ok[wi] = active && prm.status[cell] != 0;
    }
    if constexpr (C::DEFORM) {
#pragma unroll
        for (int wi = 0; wi < WPG; ++wi) {
            const long long cell = base_cell + wi;
            const bool active = cell < prm.ncells;
            const int ci = active ? (int)cell : 0;
            const float4 k0 = active ? prm.corners[2 * (size_t)ci] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 k1 = active ? prm.corners[2 * (size_t)ci + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
            // base position: the grid origin under the placement clamp (multipass.rs:207-208)
            const int gx = min(prm.gx0 + (ci % prm.gnx) * prm.gstep, max(prm.W - N - 1, 0));
            const int gy = min(prm.gy0 + (ci / prm.gnx) * prm.gstep, max(prm.H - N - 1, 0));
            org[wi] = make_float4(corner_blend(k0.x, k0.z, k1.x, k1.z, 0.5f, 0.5f),
                                  corner_blend(k0.y, k0.w, k1.y, k1.w, 0.5f, 0.5f), 0.f, 0.f);
            if (wi == 0) {
                sample_deformed<N, T, C::BLOCK>(prm.img_a, prm.img_b, prm.H, prm.W, gx, gy, k0, k1, line,
                                                C::BLOCK ? rt : t, s_ramp, z0);
            } else if constexpr (PAIR) {
                sample_deformed<N, T, C::BLOCK>(prm.img_a, prm.img_b, prm.H, prm.W, gx, gy, k0, k1, line,
                                                C::BLOCK ? rt : t, s_ramp, z1);
            }
        }
    } else if constexpr (C::BLOCK) {
        const GlobalSrc ga{prm.img_a, prm.W}, gb{prm.img_b, prm.W};
        sample_block<N, T, false, C::SHFL_SAMPLE>(ga, prm.H, prm.W, org[0].x, org[0].y, line, rt, z0);
        sample_block<N, T, true, C::SHFL_SAMPLE>(gb, prm.H, prm.W, org[0].z, org[0].w, line, rt, z0);
        sample_block<N, T, false, C::SHFL_SAMPLE>(ga, prm.H, prm.W, org[1].x, org[1].y, line, rt, z1);
        sample_block<N, T, true, C::SHFL_SAMPLE>(gb, prm.H, prm.W, org[1].z, org[1].w, line, rt, z1);
    } else if constexpr (C::SHFL_SAMPLE) {
        const GlobalSrc ga{prm.img_a, prm.W}, gb{prm.img_b, prm.W};
        sample_column<N, T, false>(ga, prm.H, prm.W, org[0].x, org[0].y, line, t, z0);
        sample_column<N, T, true>(gb, prm.H, prm.W, org[0].z, org[0].w, line, t, z0);
        if constexpr (PAIR) {
            sample_column<N, T, false>(ga, prm.H, prm.W, org[1].x, org[1].y, line, t, z1);
            sample_column<N, T, true>(gb, prm.H, prm.W, org[1].z, org[1].w, line, t, z1);
        }
    } else {
        const GlobalSrc ga{prm.img_a, prm.W}, gb{prm.img_b, prm.W};
        sample_column_direct<N, T, false>(ga, prm.H, prm.W, org[0].x, org[0].y, line, t, z0);
        sample_column_direct<N, T, true>(gb, prm.H, prm.W, org[0].z, org[0].w, line, t, z0);
        if constexpr (PAIR) {
            sample_column_direct<N, T, false>(ga, prm.H, prm.W, org[1].x, org[1].y, line, t, z1);
            sample_column_direct<N, T, true>(gb, prm.H, prm.W, org[1].z, org[1].w, line, t, z1);
        }
    }
    {
        float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int p = 0; p < P; ++p) {
            s.x += z0[p].x;
            s.y += z0[p].y;
            if constexpr (PAIR) {
                s.z += z1[p].x;
                s.w += z1[p].y;
            }
        }
        s = group_sum4<C>(s, s_red, g, gt);
        constexpr float inv = 1.0f / (float)(N * N);
        const float m0a = s.x * inv, m0b = s.y * inv, m1a = s.z * inv, m1b = s.w * inv;
        float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int p = 0; p < P; ++p) {
            z0[p].x = __fsub_rn(z0[p].x, m0a);
            z0[p].y = __fsub_rn(z0[p].y, m0b);
            e.x += z0[p].x * z0[p].x;
            e.y += z0[p].y * z0[p].y;
            if constexpr (PAIR) {
                z1[p].x = __fsub_rn(z1[p].x, m1a);
                z1[p].y = __fsub_rn(z1[p].y, m1b);
                e.z += z1[p].x * z1[p].x;
                e.w += z1[p].y * z1[p].y;
            }
        }
        e = group_sum4<C>(e, s_red, g, gt);
        // correlate.rs:110 (flat window) and :136 (scale 1 / (n^2 sqrt(Ea Eb))); the factor 1/4
        // undoes the 2x folded into each separated spectrum (exact power-of-two scaling).
        ok[0] = ok[0] && e.x > 1e-12f && e.y > 1e-12f;
        scale[0] = 0.25f / ((float)(N * N) * (sqrtf(e.x) * sqrtf(e.y)));
        if constexpr (PAIR) {
            ok[1] = ok[1] && e.z > 1e-12f && e.w > 1e-12f;
            scale[1] = 0.25f / ((float)(N * N) * (sqrtf(e.z) * sqrtf(e.w)));
        }
    }

    // ------------------------------------------------------------------ forward 2-D FFTs
    float2* plane1 = reinterpret_cast<float2*>(plane1_raw);
    if constexpr (C::BLOCK) {
        // lane t ends with the rows ky = t + T*k; both windows stage by stage
        fft_line_blocked2<N, T, 1>(z0, z1, t, s_roots);
#pragma unroll
        for (int k = 0; k < P; ++k) {
            plane0[C::AF(t + T * k, line)] = z0[k];
            plane1[C::AF(t + T * k, line)] = z1[k];
        }
    } else {
        if constexpr (PAIR && N == 64) {
            fft_line_interleaved2<N, T, 1>(z0, z1, t, s_roots);  // both windows stage by stage
        } else {
            fft_line_interleaved<N, T, 1>(z0, t, s_roots);
            if constexpr (PAIR) fft_line_interleaved<N, T, 1>(z1, t, s_roots);
        }
#pragma unroll
        for (int k = 0; k < P; ++k) {
            plane0[C::A(k + P * rt, line)] = z0[k];
            if constexpr (PAIR) plane1[C::A(k + P * rt, line)] = z1[k];
        }
    }
    group_sync<C>(g);
#pragma unroll
    for (int q = 0; q < P; ++q) {
        z0[q] = plane0[C::AF(line, t + T * q)];
        if constexpr (PAIR) z1[q] = plane1[C::AF(line, t + T * q)];
    }
    group_sync<C>(g);
    if constexpr (PAIR && (N == 64 || N == 32)) {
        fft_line_interleaved2<N, T, 1>(z0, z1, t, s_roots);  // both windows stage by stage
    } else {
        fft_line_interleaved<N, T, 1>(z0, t, s_roots);
        if constexpr (PAIR) fft_line_interleaved<N, T, 1>(z1, t, s_roots);
    }
    if constexpr (!PAIR) {
        // ------------------------------------------------------------------ single window
        float2 best = make_float2(-INFINITY, -INFINITY);
        int bi0 = 0x7fffffff;
        float2 second = make_float2(-INFINITY, -INFINITY);
        float* const cplane = reinterpret_cast<float*>(plane0) + C::CP_OFF;
        float* const vm = reinterpret_cast<float*>(plane1_raw);  // vertical 3-maxima
        auto at = [&](int y, int x) -> float { return cplane[C::CP(y % N, x % N)]; };
        auto circ = [](int a, int b) {
            const int d = abs(a - b);
            return min(d, N - d);
        };
        // One window: z0 is the spectrum of a + i*b and the cross spectrum C is Hermitian
        // (C[-k] = conj C[k], exactly so in floating point: cross4(m, z) = conj cross4(z, m)), so
        // its inverse is real and half of a complex inverse computes it:
        //  1. rows ky = 0..N/2 only: Y[ky][x] = sum_kx C[ky][kx] w^(kx x), where Y[-ky] = conj Y[ky]
        //     and rows 0 and N/2 are real, so those two share one line (C[0] + i*C[N/2]);
        //  2. columns in pairs (x, x + N/2): Z[ky] = Y[ky][x] + i*Y[ky][x + N/2] (rows above N/2
        //     from their conjugate partners); the inverse of Z is corr[.][x] + i*corr[.][x + N/2].
        // Each stage is N/2 lines of T2 = 2T lanes (P2 = N/T2 values each) on the same threads.
        constexpr int T2 = 2 * T, P2 = N / T2;
        static_assert(N == 128 && T == 4 && G == 1, "single-window layout");
        const int line2 = gt / T2, t2 = gt - line2 * T2, rt2 = bitrev<T2>(t2);
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int k = 0; k < P; ++k) plane0[C::BS(line, k + P * rt)] = z0[k];
        group_sync<C>(g);
        float2 y[P2];
        {
            const int ky = line2, my = (N - line2) % N;
#pragma unroll
            for (int p = 0; p < P2; ++p) {
                const int kx = p + P2 * rt2, mkx = (N - kx) % N;
                y[p] = cross4(plane0[C::BS(ky, kx)], plane0[C::BS(my, mkx)]);
            }
            if (line2 == 0) {
#pragma unroll
                for (int p = 0; p < P2; ++p) {
                    const int kx = p + P2 * rt2, mkx = (N - kx) % N;
                    const float2 c = cross4(plane0[C::BS(N / 2, kx)], plane0[C::BS(N / 2, mkx)]);
                    y[p] = make_float2(y[p].x - c.y, y[p].y + c.x);  // C[0] + i*C[N/2]
                }
            }
        }
        fft_line_blocked<N, T2, -1>(y, t2, s_roots);  // lane holds Y[line2][t2 + T2*k]
        group_sync<C>(g);                               // every spectrum read is done
        if (line2 == 0) {
#pragma unroll
            for (int k = 0; k < P2; ++k) {
                plane0[C::YO(0, t2 + T2 * k)] = make_float2(y[k].x, 0.0f);
                plane0[C::YO(N / 2, t2 + T2 * k)] = make_float2(y[k].y, 0.0f);
            }
        } else {
#pragma unroll
            for (int k = 0; k < P2; ++k) plane0[C::YO(line2, t2 + T2 * k)] = y[k];
        }
        group_sync<C>(g);
        const int x1 = line2, x2 = line2 + N / 2;
#pragma unroll
        for (int q = 0; q < P2; ++q) {
            const int ky = t2 + T2 * q;
            if (q < P2 / 2) {  // ky < N/2
                const float2 a = plane0[C::YO(ky, x1)], b = plane0[C::YO(ky, x2)];
                y[q] = make_float2(a.x - b.y, a.y + b.x);
            } else {  // ky >= N/2: Y[ky] = conj Y[N - ky]
                const float2 a = plane0[C::YO(N - ky, x1)], b = plane0[C::YO(N - ky, x2)];
                y[q] = make_float2(a.x + b.y, b.x - a.y);
            }
        }
        fft_line_interleaved<N, T2, -1>(y, t2, s_roots);
        // Lane now holds corr[k + P2*rt2][x1] (real part) and corr[k + P2*rt2][x2] (imaginary
        // part); scale as the reference does (c *= scale).
#pragma unroll
        for (int k = 0; k < P2; ++k) {
            y[k].x = y[k].x * scale[0];
            y[k].y = y[k].y * scale[0];
            cplane[C::CP(k + P2 * rt2, x1)] = y[k].x;
            cplane[C::CP(k + P2 * rt2, x2)] = y[k].y;
        }
#pragma unroll
        for (int k = 0; k < P2; ++k) {
            const int row = (k + P2 * rt2) * N;
            if (y[k].x > best.x) {
                best.x = y[k].x;
                bi0 = row + x1;
            }
            if (y[k].y > best.x) {
                best.x = y[k].y;
                bi0 = row + x2;
            }
        }
        group_argmax<C>(best.x, bi0, s_red, g, gt);
        if (!(best.x > -INFINITY)) bi0 = 0;
        group_sync<C>(g);  // the scaled plane is complete in shared memory
        // Footprint of the primary peak (correlate.rs:242-254): half-width along +-y, +-x.
        if (gt < 4) {
            const int by = bi0 / N, bx = bi0 % N;
            const int sy = gt == 0 ? 1 : (gt == 1 ? N - 1 : 0);
            const int sx = gt == 2 ? 1 : (gt == 3 ? N - 1 : 0);
            const float half = 0.5f * best.x;
            int k = 0;
            while (k < N / 2 && at(by + k * sy, bx + k * sx) > half) ++k;
            s_hw[g][gt] = k;
        }
        {
            const int base = lane - t2;  // first lane of this column pair
            const int src_up = base + bitrev<T2>((rt2 + T2 - 1) % T2);
            const int src_dn = base + bitrev<T2>((rt2 + 1) % T2);
            float2 up, dn;
            up.x = __shfl_sync(0xffffffffu, y[P2 - 1].x, src_up);
            up.y = __shfl_sync(0xffffffffu, y[P2 - 1].y, src_up);
            dn.x = __shfl_sync(0xffffffffu, y[0].x, src_dn);
            dn.y = __shfl_sync(0xffffffffu, y[0].y, src_dn);
#pragma unroll
            for (int k = 0; k < P2; ++k) {
                const float2 a = k == 0 ? up : y[k - 1];
                const float2 b = k == P2 - 1 ? dn : y[k + 1];
                vm[C::CP(k + P2 * rt2, x1)] = fmaxf(fmaxf(a.x, b.x), y[k].x);
                vm[C::CP(k + P2 * rt2, x2)] = fmaxf(fmaxf(a.y, b.y), y[k].y);
            }
        }
        group_sync<C>(g);
        const int hw0 = max(max(s_hw[g][0], s_hw[g][1]), max(s_hw[g][2], s_hw[g][3]));
        const int ex0 = max((int)ceilf(1.5f * (float)hw0), 2);
        // Highest local maximum outside the footprint (correlate.rs:255-267), the direct
        // distance test.
        {
            const int by0 = bi0 / N, bx0 = bi0 % N;
            const int cx1 = circ(x1, bx0), cx2 = circ(x2, bx0);
            const int x1l = (x1 + N - 1) % N, x1r = x1 + 1, x2l = x2 - 1, x2r = (x2 + 1) % N;
#pragma unroll
            for (int k = 0; k < P2; ++k) {
                const int r = k + P2 * rt2;
                const int cy = circ(r, by0);
                const float h1 = fmaxf(fmaxf(vm[C::CP(r, x1l)], vm[C::CP(r, x1r)]), vm[C::CP(r, x1)]);
                const float h2 = fmaxf(fmaxf(vm[C::CP(r, x2l)], vm[C::CP(r, x2r)]), vm[C::CP(r, x2)]);
                if (y[k].x == h1 && max(cy, cx1) > ex0) second.x = fmaxf(second.x, y[k].x);
                if (y[k].y == h2 && max(cy, cx2) > ex0) second.x = fmaxf(second.x, y[k].y);
            }
        }
        second = group_max2<C>(second, s_red, g, gt);

        // ------------------------------------------------------------------ sub-pixel fit, output
        if (gt == 0 && base_cell < prm.ncells) {
            const long long cell = base_cell;
            if (ok[0]) {
                const int by = bi0 / N, bx = bi0 % N;
                const float bv = best.x, sv = second.x;
                const float sx = subpixel(at(by, bx + N - 1), bv, at(by, bx + 1));
                const float sy = subpixel(at(by + N - 1, bx), bv, at(by + 1, bx));
                const float wx = bx >= N / 2 ? (float)bx - (float)N : (float)bx;
                const float wy = by >= N / 2 ? (float)by - (float)N : (float)by;
                const float pdx = __fadd_rn(wx, sx), pdy = __fadd_rn(wy, sy);
                const float ppr = sv > 0.0f ? fminf(__fdiv_rn(bv, sv), MAX_PPR) : MAX_PPR;
                const float4 o = org[0];
                if constexpr (C::DEFORM) {
                    prm.raw_dx[cell] = __fadd_rn(o.x, pdx);  // D(centre) + peak
                    prm.raw_dy[cell] = __fadd_rn(o.y, pdy);
                } else {
                    prm.raw_dx[cell] = __fadd_rn(__fsub_rn(o.z, o.x), pdx);
                    prm.raw_dy[cell] = __fadd_rn(__fsub_rn(o.w, o.y), pdy);
                }
                prm.raw_ppr[cell] = ppr;
                prm.raw_flags[cell] = 0;
            } else {
                prm.raw_dx[cell] = NAN;
                prm.raw_dy[cell] = NAN;
                prm.raw_ppr[cell] = 0.0f;
                prm.raw_flags[cell] = F_NO_SIGNAL;
            }
        }
    } else {
        // ------------------------------------------------------------------ cross spectra
        // Both windows' spectra, then D = C0 + i*C1: one complex inverse gives both (real)
        // correlation planes, window 0 in the real part and window 1 in the imaginary part.
#pragma unroll
        for (int k = 0; k < P; ++k) {
            plane0[C::B(line, k + P * rt)] = z0[k];
            plane1[C::B(line, k + P * rt)] = z1[k];
        }
        group_sync<C>(g);
        {
            const int my = (N - line) % N;
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const int kx = (N - (k + P * rt)) % N;
                const float2 c0 = cross4(z0[k], plane0[C::B(my, kx)]);
                const float2 c1 = cross4(z1[k], plane1[C::B(my, kx)]);
                z0[k] = make_float2(c0.x - c1.y, c0.y + c1.x);  // D = C0 + i*C1
            }
        }
        group_sync<C>(g);

        // ------------------------------------------------------------------ inverse 2-D FFT
        fft_line_blocked<N, T, -1>(z0, t, s_roots);
#pragma unroll
        for (int k = 0; k < P; ++k) plane0[C::A(line, t + T * k)] = z0[k];
        group_sync<C>(g);
#pragma unroll
        for (int q = 0; q < P; ++q) z0[q] = plane0[C::A(t + T * q, line)];
        group_sync<C>(g);
        fft_line_interleaved<N, T, -1>(z0, t, s_roots);
        // Lane now holds corr[y = k + P*rt][x = line]; scale as the reference does (c *= scale).
#pragma unroll
        for (int k = 0; k < P; ++k) {
            z0[k].x = z0[k].x * scale[0];
            z0[k].y = z0[k].y * scale[WPG - 1];
            plane0[C::A(k + P * rt, line)] = z0[k];
        }

        // ------------------------------------------------------------------ find_peak
        // Argmax of both planes (lowest row-major index among equal maxima). A lane's indices grow
        // with k, so inside the lane a strictly larger value is the only one that replaces the best.
        float2 best = make_float2(-INFINITY, -INFINITY);
        int bi0 = 0x7fffffff, bi1 = 0x7fffffff;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const int idx = (k + P * rt) * N + line;
            if (z0[k].x > best.x) {
                best.x = z0[k].x;
                bi0 = idx;
            }
            if (z0[k].y > best.y) {
                best.y = z0[k].y;
                bi1 = idx;
            }
        }
        group_argmax<C>(best.x, bi0, s_red, g, gt);
        group_argmax<C>(best.y, bi1, s_red, g, gt);
        if (!(best.x > -INFINITY)) bi0 = 0;
        if (!(best.y > -INFINITY)) bi1 = 0;
        group_sync<C>(g);  // the scaled planes are complete in shared memory
        auto at = [&](int ch, int y, int x) -> float {
            const float2 v = plane0[C::A(y % N, x % N)];
            return ch == 0 ? v.x : v.y;
        };
        // Footprint of the primary peak (correlate.rs:242-254): half-width along +-y, +-x.
        if (gt < 4 * WPG) {
            const int ch = gt >> 2, dir = gt & 3;
            const int bidx = ch == 0 ? bi0 : bi1;
            const int by = bidx / N, bx = bidx % N;
            const int sy = dir == 0 ? 1 : (dir == 1 ? N - 1 : 0);
            const int sx = dir == 2 ? 1 : (dir == 3 ? N - 1 : 0);
            const float half = 0.5f * (ch == 0 ? best.x : best.y);
            int k = 0;
            while (k < N / 2 && at(ch, by + k * sy, bx + k * sx) > half) ++k;
            s_hw[g][gt] = k;
        }
        // Vertical 3-maximum of each column, for the local-maximum test.
        float2* vm = reinterpret_cast<float2*>(plane1_raw);  // vertical 3-maxima of both planes
        float2 up, dn;  // neighbours across this lane's block boundary (rows k = -1 and P)
        {
            if constexpr (T == 1) {
                up = z0[P - 1];
                dn = z0[0];
            } else {
                const int lane = threadIdx.x & 31;
                const int base = lane - t;  // first lane of this line
                const int src_up = base + bitrev<T>((rt + T - 1) % T);
                const int src_dn = base + bitrev<T>((rt + 1) % T);
                up.x = __shfl_sync(0xffffffffu, z0[P - 1].x, src_up);
                up.y = __shfl_sync(0xffffffffu, z0[P - 1].y, src_up);
                dn.x = __shfl_sync(0xffffffffu, z0[0].x, src_dn);
                dn.y = __shfl_sync(0xffffffffu, z0[0].y, src_dn);
            }
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const float2 a = k == 0 ? up : z0[k - 1];
                const float2 b = k == P - 1 ? dn : z0[k + 1];
                const float m0 = fmaxf(fmaxf(a.x, b.x), z0[k].x);
                vm[C::A(k + P * rt, line)] = make_float2(m0, fmaxf(fmaxf(a.y, b.y), z0[k].y));
            }
        }
        group_sync<C>(g);
        const int hw0 = max(max(s_hw[g][0], s_hw[g][1]), max(s_hw[g][2], s_hw[g][3]));
        const int ex0 = max((int)ceilf(1.5f * (float)hw0), 2);
        const int hw1 = max(max(s_hw[g][4], s_hw[g][5]), max(s_hw[g][6], s_hw[g][7]));
        const int ex1 = max((int)ceilf(1.5f * (float)hw1), 2);
        // Highest local maximum outside the footprint (correlate.rs:255-267): v is a local maximum
        // when it equals the maximum of its circular 3x3 neighbourhood.
        float2 second = make_float2(-INFINITY, -INFINITY);
        {
            const int xl = (line + N - 1) % N, xr = (line + 1) % N;
            const int by0 = bi0 / N, bx0 = bi0 % N, by1 = bi1 / N, bx1 = bi1 % N;
            auto circ = [](int a, int b) {
                const int d = abs(a - b);
                return min(d, N - d);
            };
            const int cx0 = circ(line, bx0), cx1 = circ(line, bx1);
            // A cell is outside the footprint when max(circular row distance, column distance) > ex:
            // one bit of a per-lane mask of eligible rows.
            const unsigned el0 = eligible_rows<N, P>(by0, ex0, cx0, rt);
            const unsigned el1 = eligible_rows<N, P>(by1, ex1, cx1, rt);
#pragma unroll
            for (int k = 0; k < P; ++k) {
                const int y = k + P * rt;
                const float2 l = vm[C::A(y, xl)], r = vm[C::A(y, xr)];
                // the lane's own vertical 3-maximum: recomputed from registers at 16 and 64 px
                // (the same value as the one stored; measured faster there), read back otherwise
                float2 c;
                if constexpr (N == 16 || N == 64) {
                    const float2 va = k == 0 ? up : z0[k - 1], vb = k == P - 1 ? dn : z0[k + 1];
                    c = make_float2(fmaxf(fmaxf(va.x, vb.x), z0[k].x), fmaxf(fmaxf(va.y, vb.y), z0[k].y));
                } else {
                    c = vm[C::A(y, line)];
                }
                const float h0 = fmaxf(fmaxf(l.x, r.x), c.x), h1 = fmaxf(fmaxf(l.y, r.y), c.y);
                if (z0[k].x == h0 && ((el0 >> k) & 1u) != 0u) second.x = fmaxf(second.x, z0[k].x);
                if (z0[k].y == h1 && ((el1 >> k) & 1u) != 0u) second.y = fmaxf(second.y, z0[k].y);
            }
        }
        second = group_max2<C>(second, s_red, g, gt);

        // ------------------------------------------------------------------ sub-pixel fit, output
        if (gt < WPG) {
            const int ch = gt;
            const long long cell = base_cell + ch;
            const bool okc = (ch == 0) ? ok[0] : ok[WPG - 1];
            const float4 o = (ch == 0) ? org[0] : org[WPG - 1];
            if (cell < prm.ncells) {
                if (okc) {
                    const int bidx = ch == 0 ? bi0 : bi1;
                    const int by = bidx / N, bx = bidx % N;
                    const float bv = ch == 0 ? best.x : best.y;
                    const float sv = ch == 0 ? second.x : second.y;
                    const float sx = subpixel(at(ch, by, bx + N - 1), bv, at(ch, by, bx + 1));
                    const float sy = subpixel(at(ch, by + N - 1, bx), bv, at(ch, by + 1, bx));
                    const float wx = bx >= N / 2 ? (float)bx - (float)N : (float)bx;
                    const float wy = by >= N / 2 ? (float)by - (float)N : (float)by;
                    const float pdx = __fadd_rn(wx, sx), pdy = __fadd_rn(wy, sy);
                    const float ppr = sv > 0.0f ? fminf(__fdiv_rn(bv, sv), MAX_PPR) : MAX_PPR;
                    if constexpr (C::DEFORM) {
                        prm.raw_dx[cell] = __fadd_rn(o.x, pdx);  // D(centre) + peak
                        prm.raw_dy[cell] = __fadd_rn(o.y, pdy);
                    } else {
                        prm.raw_dx[cell] = __fadd_rn(__fsub_rn(o.z, o.x), pdx);
                        prm.raw_dy[cell] = __fadd_rn(__fsub_rn(o.w, o.y), pdy);
                    }
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
    }
}

template <class C>
__global__ void __launch_bounds__(C::THREADS, C::MINB) correlate_kernel(const __grid_constant__ CorrBatch batch) {
    const int item = batch_item(batch.block_start, batch.n, (int)blockIdx.x);
    extern __shared__ float4 smem_f4[];
    correlate_body<C>(batch.item[item], (int)blockIdx.x - batch.block_start[item], reinterpret_cast<char*>(smem_f4));
}

// ---------------------------------------------------------------------------------------------
// Fused launch over items of different window sizes and window kinds (the serving form's step):
// every configuration below has 256 threads per CTA and the same register cap, so one kernel
// holds them all and each CTA runs the body of its item's configuration. Each configuration is
// the FFT decomposition (N, T, PAIR) of that size's per-size kernel, so the results are bit
// for bit those of the per-size launches.
// ---------------------------------------------------------------------------------------------
using FusedC0 = CorrCfg<8, 1, true, 32, 2, true>;
using FusedC1 = CorrCfg<16, 1, true, 16, 2, false>;
using FusedC2 = CorrCfg<32, 2, true, 4, 2, false>;
using FusedC3 = CorrCfg<64, 4, true, 1, 2, false>;
using FusedC4 = CorrCfg<8, 1, true, 32, 2, false, true>;
using FusedC5 = CorrCfg<16, 1, true, 16, 2, false, true>;
using FusedC6 = CorrCfg<32, 2, true, 4, 2, false, true>;
using FusedC7 = CorrCfg<64, 4, true, 1, 2, false, true>;
constexpr int kFusedThreads = 256;
constexpr size_t kFusedSmem =
    std::max({FusedC0::SMEM, FusedC1::SMEM, FusedC2::SMEM, FusedC3::SMEM, FusedC4::SMEM, FusedC5::SMEM, FusedC6::SMEM,
              FusedC7::SMEM});
static_assert(FusedC0::THREADS == kFusedThreads && FusedC1::THREADS == kFusedThreads &&
                  FusedC2::THREADS == kFusedThreads && FusedC3::THREADS == kFusedThreads &&
                  FusedC4::THREADS == kFusedThreads && FusedC5::THREADS == kFusedThreads &&
                  FusedC6::THREADS == kFusedThreads && FusedC7::THREADS == kFusedThreads,
              "fused configurations share the block size");
static_assert(kFusedSmem <= 227 * 1024, "shared memory");

// Configuration index of (window, deformed) in the fused kernel, or -1.
int fused_kind(int n, bool deform) {
    const int s = n == 8 ? 0 : n == 16 ? 1 : n == 32 ? 2 : n == 64 ? 3 : -1;
    return s < 0 ? -1 : s + (deform ? 4 : 0);
}

static int fused_cells_per_block(int kind) {
    switch (kind & 3) {
        case 0: return FusedC0::G * FusedC0::WPG;
        case 1: return FusedC1::G * FusedC1::WPG;
        case 2: return FusedC2::G * FusedC2::WPG;
        default: return FusedC3::G * FusedC3::WPG;
    }
}

struct FusedBatch {
    int n;
    int block_start[kMaxBatch + 1];
    int kind[kMaxBatch];
    CorrParams item[kMaxBatch];
};

__global__ void __launch_bounds__(kFusedThreads, 2) correlate_fused_kernel(const __grid_constant__ FusedBatch b) {
    const int item = batch_item(b.block_start, b.n, (int)blockIdx.x);
    const CorrParams& prm = b.item[item];
    const int block = (int)blockIdx.x - b.block_start[item];
    extern __shared__ float4 smem_f4[];
    char* sm = reinterpret_cast<char*>(smem_f4);
    switch (b.kind[item]) {
        case 0: correlate_body<FusedC0>(prm, block, sm); break;
        case 1: correlate_body<FusedC1>(prm, block, sm); break;
        case 2: correlate_body<FusedC2>(prm, block, sm); break;
        case 3: correlate_body<FusedC3>(prm, block, sm); break;
        case 4: correlate_body<FusedC4>(prm, block, sm); break;
        case 5: correlate_body<FusedC5>(prm, block, sm); break;
        case 6: correlate_body<FusedC6>(prm, block, sm); break;
        default: correlate_body<FusedC7>(prm, block, sm); break;
    }
}

cudaError_t launch_correlate_fused(const CorrParams* items, const int* kinds, int count, cudaStream_t s,
                                   int* launches) {
    for (int i = 0; i < count; ++i) {
        if (kinds[i] < 0 || kinds[i] > 7) return cudaErrorInvalidValue;
        if ((kinds[i] >= 4) != (items[i].corners != nullptr)) return cudaErrorInvalidValue;
        if (kinds[i] >= 4 && (items[i].gnx <= 0 || items[i].gstep <= 0)) return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaFuncSetAttribute(correlate_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kFusedSmem);
    if (e != cudaSuccess) return e;
    for (int off = 0; off < count; off += kMaxBatch) {
        FusedBatch b;
        b.n = count - off < kMaxBatch ? count - off : kMaxBatch;
        long long total = 0;
        for (int i = 0; i < b.n; ++i) {
            b.item[i] = items[off + i];
            b.kind[i] = kinds[off + i];
            b.block_start[i] = (int)total;
            const int per = fused_cells_per_block(b.kind[i]);
            total += (b.item[i].ncells + per - 1) / per;
        }
        b.block_start[b.n] = (int)total;
        if (total > 0x7fffffffll) return cudaErrorInvalidValue;
        if (total > 0) {
            correlate_fused_kernel<<<(unsigned)total, kFusedThreads, kFusedSmem, s>>>(b);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            if (launches) ++*launches;
        }
    }
    return cudaSuccess;
}

// One launch over all items of the batch: item i owns blocks [block_start[i], block_start[i+1]).
template <class C>
static cudaError_t launch_t(CorrBatch b, cudaStream_t s) {
    static_assert(C::SMEM <= 227 * 1024, "shared memory");
    const long long per_block = (long long)C::G * C::WPG;
    long long total = 0;
    for (int i = 0; i < b.n; ++i) {
        b.block_start[i] = (int)total;
        total += (b.item[i].ncells + per_block - 1) / per_block;
    }
    b.block_start[b.n] = (int)total;
    if (total <= 0) return cudaSuccess;
    if (total > 0x7fffffffll) return cudaErrorInvalidValue;
    auto kern = correlate_kernel<C>;
    // Attribute setting is idempotent and per device; done on every launch for simplicity.
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)total, C::THREADS, C::SMEM, s>>>(b);
    return cudaGetLastError();
}

bool corr_supported(int n) {
    switch (n) {
        case 8: case 12: case 16: case 24: case 32: case 48: case 64: case 96: case 128: return true;
        default: return false;
    }
}

// ---------------------------------------------------------------------------------------------
// Launch variants per window size. Within one size every variant has the same N, T and PAIR,
// so all of them compute bit-identical results; they differ in groups per CTA, register cap and
// sampler. Variant 0 is the default; the autotuner (api.cu) times the others on live data.
// ---------------------------------------------------------------------------------------------
struct CorrVariant {
    const char* name;
    cudaError_t (*launch)(CorrBatch, cudaStream_t);
};

#define PIV_V(N, T, PR, G, MB, SH) {#N "/T" #T "/G" #G "/B" #MB "/" #SH, &launch_t<CorrCfg<N, T, PR, G, MB, SH>>}
static const CorrVariant kV8[] = {PIV_V(8, 1, true, 32, 1, false), PIV_V(8, 1, true, 16, 2, false),
                                  PIV_V(8, 1, true, 32, 2, true), PIV_V(8, 1, true, 4, 16, false)};
static const CorrVariant kV12[] = {PIV_V(12, 1, true, 16, 1, false), PIV_V(12, 1, true, 8, 3, false),
                                   PIV_V(12, 1, true, 16, 2, true)};
static const CorrVariant kV16[] = {PIV_V(16, 1, true, 16, 2, false), PIV_V(16, 1, true, 8, 4, false),
                                   PIV_V(16, 1, true, 8, 3, false), PIV_V(16, 1, true, 16, 2, true),
                                   PIV_V(16, 1, true, 8, 4, true), PIV_V(16, 1, true, 2, 16, false),
                                   PIV_V(16, 1, true, 4, 8, false), PIV_V(16, 1, true, 2, 16, true)};
static const CorrVariant kV24[] = {PIV_V(24, 2, true, 4, 2, true), PIV_V(24, 2, true, 4, 2, false),
                                   PIV_V(24, 2, true, 2, 4, true)};
static const CorrVariant kV32[] = {PIV_V(32, 2, true, 4, 2, false), PIV_V(32, 2, true, 4, 2, true),
                                   PIV_V(32, 2, true, 2, 4, true), PIV_V(32, 2, true, 2, 3, true),
                                   PIV_V(32, 2, true, 1, 8, true), PIV_V(32, 2, true, 1, 8, false)};
static const CorrVariant kV48[] = {PIV_V(48, 4, true, 1, 2, true), PIV_V(48, 4, true, 1, 2, false),
                                   PIV_V(48, 4, true, 1, 1, true)};
static const CorrVariant kV64[] = {PIV_V(64, 4, true, 1, 2, false), PIV_V(64, 4, true, 1, 2, true),
                                   PIV_V(64, 4, true, 1, 1, true)};
static const CorrVariant kV96[] = {PIV_V(96, 4, true, 1, 1, true), PIV_V(96, 4, true, 1, 1, false)};
static const CorrVariant kV128[] = {PIV_V(128, 4, false, 1, 1, false), PIV_V(128, 4, false, 1, 1, true)};
// Deformed-window variants: the same FFT decomposition per size, the deformed sampler.
#define PIV_D(N, T, PR, G, MB) {#N "/T" #T "/G" #G "/B" #MB "/deform", &launch_t<CorrCfg<N, T, PR, G, MB, false, true>>}
static const CorrVariant kD8[] = {PIV_D(8, 1, true, 32, 1)};
static const CorrVariant kD12[] = {PIV_D(12, 1, true, 16, 1)};
static const CorrVariant kD16[] = {PIV_D(16, 1, true, 16, 2), PIV_D(16, 1, true, 8, 4)};
static const CorrVariant kD24[] = {PIV_D(24, 2, true, 4, 2)};
static const CorrVariant kD32[] = {PIV_D(32, 2, true, 4, 2), PIV_D(32, 2, true, 2, 4)};
static const CorrVariant kD48[] = {PIV_D(48, 4, true, 1, 2)};
static const CorrVariant kD64[] = {PIV_D(64, 4, true, 1, 2), PIV_D(64, 4, true, 1, 1)};
static const CorrVariant kD96[] = {PIV_D(96, 4, true, 1, 1)};
static const CorrVariant kD128[] = {PIV_D(128, 4, false, 1, 1)};
#undef PIV_D
#undef PIV_V

static const CorrVariant* variants(int n, bool deform, int* count) {
#define PIV_CASE(N, A, D)                                                       \
    case N:                                                                     \
        *count = deform ? (int)(sizeof(D) / sizeof(D[0])) : (int)(sizeof(A) / sizeof(A[0])); \
        return deform ? D : A;
    switch (n) {
        PIV_CASE(8, kV8, kD8)
        PIV_CASE(12, kV12, kD12)
        PIV_CASE(16, kV16, kD16)
        PIV_CASE(24, kV24, kD24)
        PIV_CASE(32, kV32, kD32)
        PIV_CASE(48, kV48, kD48)
        PIV_CASE(64, kV64, kD64)
        PIV_CASE(96, kV96, kD96)
        PIV_CASE(128, kV128, kD128)
        default:
            *count = 0;
            return nullptr;
    }
#undef PIV_CASE
}

int corr_num_variants(int n, bool deform) {
    int c = 0;
    variants(n, deform, &c);
    return c;
}

const char* corr_variant_name(int n, int v, bool deform) {
    int c = 0;
    const CorrVariant* vs = variants(n, deform, &c);
    return (vs && v >= 0 && v < c) ? vs[v].name : "";
}

cudaError_t launch_correlate_items(int n, int v, const CorrParams* items, int count, cudaStream_t s, int* launches) {
    if (count <= 0) return cudaSuccess;
    const bool deform = items[0].corners != nullptr;
    for (int i = 1; i < count; ++i)
        if ((items[i].corners != nullptr) != deform) return cudaErrorInvalidValue;
    if (deform)
        for (int i = 0; i < count; ++i)
            if (items[i].gnx <= 0 || items[i].gstep <= 0) return cudaErrorInvalidValue;
    int c = 0;
    const CorrVariant* vs = variants(n, deform, &c);
    if (!vs || v < 0 || v >= c) return cudaErrorInvalidValue;
    for (int off = 0; off < count; off += kMaxBatch) {
        CorrBatch b;
        b.n = count - off < kMaxBatch ? count - off : kMaxBatch;
        for (int i = 0; i < b.n; ++i) b.item[i] = items[off + i];
        const cudaError_t e = vs[v].launch(b, s);
        if (e != cudaSuccess) return e;
        if (launches) ++*launches;
    }
    return cudaSuccess;
}

cudaError_t launch_correlate_variant(int n, int v, const CorrParams& p, cudaStream_t s) {
    return launch_correlate_items(n, v, &p, 1, s, nullptr);
}

cudaError_t launch_correlate(int n, const CorrParams& p, cudaStream_t s) { return launch_correlate_variant(n, 0, p, s); }

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
