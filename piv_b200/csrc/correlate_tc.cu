// Split-precision tensor-core form of the window correlation (no counterpart in the reference,
// whose FFTs run on CPU cores: correlate.rs:99-178 through realfft/rustfft).
//
// The 2-D DFTs of CorrelationPlan::correlate become dense DFT-matrix products on the 5th-
// generation tensor cores (tcgen05.mma kind::f16, BF16 operands in shared memory, FP32
// accumulators in TMEM). Every operand x is split into hi = h(x) and lo = h(x - hi), h the
// rounding to BF16 (about 16 significant bits for the pair) or FP16 (about 22), and a product
// A*B is evaluated as hi*hi + lo*hi + hi*lo with FP32 sums.
//
// Operand ranges: each window is normalised to unit variance before F1 (x * N / sqrt(E)); by
// Parseval every spectrum is then bounded by N^2 and every cross spectrum by N^4, so the fixed
// power-of-two factors 2^(12 - 4 log2 N) on the cross spectrum and 1/N before I2 keep all
// operands inside FP16's range. The correlation plane is rescaled by the exact inverse power of
// two, which with the normalisation equals the reference's 1 / (n^2 sqrt(Ea Eb)).
//
// One warpgroup owns a 128-row tile of 128/N windows; thread i is row i of every operand and
// TMEM lane i. Real input makes the transforms half-size, so every stage is a 128 x N x K GEMM
// with the exchanges between stages either inside a thread or between the two lanes of a pair:
//   F1  r2c along x of both frames (rows (w, r), K = x): packed half spectrum per row,
//       columns [re(kx=0..N/2-1) | im(kx=1..N/2-1) with the Nyquist real value in the im(0) slot]
//   F2  complex DFT along y (rows (w, kx', frame), K = [re(r) | im(r)]): row kx' = 0 carries
//       DC + i*Nyquist and is separated inside the thread (Hermitian partner at -ky);
//   --  cross spectrum conj(FA)*FB between the two frame lanes (lane ^ 1), window mean removed by
//       zeroing the DC bin; the frame-1 lane multiplies by (-1)^ky so that the next stage gives
//       it the upper half of the outputs;
//   I1  inverse complex DFT along ky, each lane half of the y outputs;
//   I2  c2r along kx (rows (w, y), K = packed kx): the correlation plane, row y per thread.
// find_peak (correlate.rs:215-303) then runs on the plane as in the FP32 kernel.
//
// 64 px windows (two per tile, each on two warps) use a compact form to fit shared memory with
// two warpgroups per CTA: the complex DFTs F2 and I1 keep only [C | S] (cos and sin blocks along
// K) instead of the 2x2 real block matrix, and form the other output half as a second MMA chain
// over the other K half of the operand with B negated (the instruction descriptor's negate-B
// bit), e.g. Im F2 = Zi C^T - Zr S^T. Window reductions then cross the two warps through shared
// memory.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "tc.cuh"
#include "window.cuh"

namespace pivb200 {

// c / (N - 1) for c < N, the deformation ramps (correctly rounded, as the FP32 kernel computes
// them), set by corr_tc_init_device.
__constant__ float c_ramp16[16];
__constant__ float c_ramp32[32];
__constant__ float c_ramp64[64];
template <int N>
__device__ __forceinline__ const float* c_ramp() {
    if constexpr (N == 16) return c_ramp16;
    else if constexpr (N == 32) return c_ramp32;
    else return c_ramp64;
}

template <int N_>
struct TcCfg {
    static constexpr int N = N_, H2 = N / 2;
    static constexpr int WPT = 128 / N;  // windows (cells) per tile
    // 64 px: compact [C | S] DFT matrices and two warpgroups per CTA (shared memory); 16 and 32
    // px: the 2x2 real block matrices and four warpgroups per CTA
    static constexpr bool COMPACT = N >= 64;
    static constexpr int NWG = COMPACT ? 2 : 4;  // warpgroups per CTA, each on its own tiles
    static constexpr int THREADS = 128 * NWG;
    // DFT matrices, B operands (rows = outputs, K-major), element offsets of hi (or lo) parts
    static constexpr int R1_OFF = 0;                                     // N x N
    static constexpr int R2_OFF = R1_OFF + N * N;                        // 2N x 2N, compact N x 2N
    static constexpr int R3_OFF = R2_OFF + (COMPACT ? 2 : 4) * N * N;    // N x 2N, compact N/2 x 2N
    static constexpr int R4_OFF = R3_OFF + (COMPACT ? 1 : 2) * N * N;    // N x N
    static constexpr int RMAT = R4_OFF + N * N;
    static constexpr size_t MAT_BYTES = (size_t)RMAT * 2;
    static constexpr int ABUF = 128 * 2 * N;  // operand elements per part per warpgroup
    static constexpr size_t A_BYTES = (size_t)ABUF * 2;
    static constexpr int TCOLS = (2 * N < 32) ? 32 : 2 * N;  // TMEM columns per warpgroup
    static constexpr int PLD = N + 4;  // FP32 plane row pitch (floats): 16-byte rows, 8 rows on distinct banks
    static constexpr size_t BAR_OFF = 2 * MAT_BYTES + (size_t)NWG * 2 * A_BYTES;
    // cross-warp window reductions (64 px): per warpgroup, 4 warps x 4 floats
    static constexpr size_t RED_OFF = (BAR_OFF + 8 * NWG + 16 + sizeof(int) * NWG * WPT * 4 + 15) / 16 * 16;
    // staged DC + i*Nyquist spectra: per warpgroup, window and frame, 2N floats
    static constexpr size_t ZST_OFF = (RED_OFF + sizeof(float) * NWG * 16 + 15) / 16 * 16;
    static constexpr size_t SMEM = ZST_OFF + sizeof(float) * NWG * WPT * 4 * N + 64;
    static_assert((size_t)128 * PLD * 4 <= 2 * A_BYTES, "plane fits in the operand buffers");
    static_assert(N % 16 == 0 && 128 % N == 0, "tile shape");
    static_assert(SMEM <= 232448, "shared memory");
    // CTAs per SM: two at 16 px (83 KB of shared memory and 128 TMEM columns each, registers
    // capped at 64 per thread), one otherwise
    static constexpr int CTAS_PER_SM = N == 16 ? 2 : 1;
    // fixed operand factors (see the top of the file) and the plane's exact rescale
    static constexpr int LOG2N = N == 16 ? 4 : (N == 32 ? 5 : 6);
    static constexpr float CROSS_SCALE = (4 * LOG2N > 12) ? 1.0f / (float)(1 << (4 * LOG2N - 12)) : 1.0f;
    // plane = I2 / (CROSS_SCALE * (1/N)) / N^4, the unit-variance factors N/sqrt(E) included
    static constexpr float PLANE_SCALE = (float)N / (CROSS_SCALE * (float)N * (float)N * (float)N * (float)N);
};

// K-major operand of `rows` rows: byte offset of the 16-byte chunk holding (row, k..k+7).
__device__ __forceinline__ uint32_t kmaj_chunk(int rows, int row, int k) {
    return (uint32_t)((k >> 3) * (rows >> 3) * 128 + (row >> 3) * 128 + (row & 7) * 16);
}
// MN-major operand of `rows` rows: byte offset of the chunk holding (m..m+7, k), m % 8 == 0.
__device__ __forceinline__ uint32_t mnmaj_chunk(int rows, int m, int k) {
    return (uint32_t)((k >> 3) * (rows >> 3) * 128 + (m >> 3) * 128 + (k & 7) * 16);
}

// Window sampling for the tensor-core tier (correlate.rs:182-202 semantics: integer copy when
// both fractional parts are < 1e-4, bilinear otherwise), one lane per column streaming down the
// rows. Each lane loads both taps of every row itself from one row pointer (the right-hand tap
// is the next float, or the same one at the right image border), with no shuffles and no
// conditional loads; the row below is carried to the next iteration. The bilinear weights are
// applied as two linear interpolations with FMA (rounding differs from the reference's weight
// sum by an ulp, far below the split-BF16 precision); zero fractions make it an exact copy.
template <int N, bool IMAG>
__device__ __forceinline__ void sample_rows(const float* __restrict__ img, int H, int W, float ox, float oy, int x,
                                            float2 (&z)[N]) {
    const float fx0 = floorf(ox), fy0 = floorf(oy);
    const int x0 = min(max((int)fx0, 0), W - 1), y0 = min(max((int)fy0, 0), H - 1);
    float tx = ox - fx0, ty = oy - fy0;
    if (tx < 1e-4f && ty < 1e-4f) tx = ty = 0.0f;
    const int c0 = min(x0 + x, W - 1);
    const int dc = min(x0 + x + 1, W - 1) - c0;  // 1, or 0 at the right border
    const float* base = img + (size_t)y0 * W + c0;
    const int last = H - 1 - y0;                  // rows below y0 that exist
    float top = __ldg(base), topr = __ldg(base + dc);
    float ht = fmaf(tx, topr - top, top);
#pragma unroll
    for (int p = 0; p < N; ++p) {
        const float* row = base + (size_t)min(p + 1, last) * W;
        const float bot = __ldg(row), botr = __ldg(row + dc);
        const float hb = fmaf(tx, botr - bot, bot);
        const float v = fmaf(ty, hb - ht, ht);
        if (IMAG) z[p].y = v; else z[p].x = v;
        ht = hb;
    }
}

__device__ __forceinline__ void wg_sync(int wg) { asm volatile("bar.sync %0, 128;" ::"r"(wg + 1) : "memory"); }

template <bool F16>
__device__ __forceinline__ void store_split(uint8_t* hi, uint8_t* lo, uint32_t off, const float (&v)[8]) {
    uint4 h, l;
    if constexpr (F16) tc::split8_f16(v, h, l); else tc::split8_bf16(v, h, l);
    *reinterpret_cast<uint4*>(hi + off) = h;
    *reinterpret_cast<uint4*>(lo + off) = l;
}

// Issues D (+)= A * B^T over `ksteps` K=16 steps for the three split products; with
// `accumulate` the chain adds to what D holds.
__device__ __forceinline__ void mma_split(uint32_t d, uint32_t a_hi, uint32_t a_lo, uint32_t a_lbo, uint32_t b_hi,
                                          uint32_t b_lo, uint32_t b_lbo, int ksteps, uint32_t idesc,
                                          bool accumulate = false) {
    uint32_t acc = accumulate ? 1u : 0u;
    const uint32_t as[3] = {a_hi, a_lo, a_hi};
    const uint32_t bs[3] = {b_hi, b_hi, b_lo};
#pragma unroll
    for (int part = 0; part < 3; ++part)
        for (int s = 0; s < ksteps; ++s) {
            const uint64_t ad = tc::smem_desc(as[part] + 2 * s * a_lbo, a_lbo, 128);
            const uint64_t bd = tc::smem_desc(bs[part] + 2 * s * b_lbo, b_lbo, 128);
            tc::mma_f16(d, ad, bd, idesc, acc);
            acc = 1;
        }
}

// Instruction-descriptor bit that negates the B operand (kind::f16 with FP32 accumulation).
constexpr uint32_t kNegateB = 1u << 14;

// Reductions over the N lanes of one window (a tile holds 128/N windows of N consecutive rows).
// Up to 32 lanes the window is a segment of one warp; a 64 px window spans two warps, whose
// partials meet in shared memory (`red`: 4 warps x 4 floats of this warpgroup), combined in the
// same order by every lane.
template <int N>
__device__ __forceinline__ float2 win_sum2(float2 v, float* red, int i, int wg) {
#pragma unroll
    for (int o = (N < 32 ? N : 32) / 2; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if constexpr (N > 32) {
        const int w = i >> 5, w0 = w & ~1;
        if ((i & 31) == 0) {
            red[4 * w] = v.x;
            red[4 * w + 1] = v.y;
        }
        wg_sync(wg);
        v = make_float2(red[4 * w0] + red[4 * w0 + 4], red[4 * w0 + 1] + red[4 * w0 + 5]);
        wg_sync(wg);
    }
    return v;
}

template <int N>
__device__ __forceinline__ void win_argmax(float& best, int& bi, float* red, int i, int wg) {
#pragma unroll
    for (int o = (N < 32 ? N : 32) / 2; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        amax_combine(best, bi, ob, oi);
    }
    if constexpr (N > 32) {
        const int w = i >> 5, w0 = w & ~1;
        if ((i & 31) == 0) {
            red[4 * w] = best;
            red[4 * w + 1] = __int_as_float(bi);
        }
        wg_sync(wg);
        best = red[4 * w0];
        bi = __float_as_int(red[4 * w0 + 1]);
        amax_combine(best, bi, red[4 * w0 + 4], __float_as_int(red[4 * w0 + 5]));
        wg_sync(wg);
    }
}

template <int N>
__device__ __forceinline__ float win_max(float v, float* red, int i, int wg) {
#pragma unroll
    for (int o = (N < 32 ? N : 32) / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if constexpr (N > 32) {
        const int w = i >> 5, w0 = w & ~1;
        if ((i & 31) == 0) red[4 * w] = v;
        wg_sync(wg);
        v = fmaxf(red[4 * w0], red[4 * w0 + 4]);
        wg_sync(wg);
    }
    return v;
}

template <int N, bool F16, bool DEFORM>
__global__ void __launch_bounds__(TcCfg<N>::THREADS, TcCfg<N>::CTAS_PER_SM)
    correlate_tc_kernel(const __grid_constant__ CorrBatch batch, const uint4* __restrict__ mats, int total_tiles,
                        unsigned int* err) {
    using C = TcCfg<N>;
    constexpr int H2 = C::H2;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* mat_hi = smem;
    uint8_t* mat_lo = smem + C::MAT_BYTES;
    const int wg = threadIdx.x >> 7;
    const int i = threadIdx.x & 127;  // row of the tile, TMEM lane
    uint8_t* a_hi = smem + 2 * C::MAT_BYTES + (size_t)wg * 2 * C::A_BYTES;
    uint8_t* a_lo = a_hi + C::A_BYTES;
    float* plane = reinterpret_cast<float*>(a_hi);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + C::BAR_OFF) + wg;
    uint32_t* tbase = reinterpret_cast<uint32_t*>(smem + C::BAR_OFF + 8 * C::NWG);
    int* s_hw = reinterpret_cast<int*>(smem + C::BAR_OFF + 8 * C::NWG + 16) + wg * C::WPT * 4;
    float* zst = reinterpret_cast<float*>(smem + C::ZST_OFF) + (size_t)wg * C::WPT * 4 * N;
    float* red = reinterpret_cast<float*>(smem + C::RED_OFF) + wg * 16;

    for (int j = threadIdx.x; j < (int)(2 * C::MAT_BYTES / 16); j += C::THREADS)
        reinterpret_cast<uint4*>(smem)[j] = mats[j];
    if (threadIdx.x == 0) {
        for (int g = 0; g < C::NWG; ++g) tc::mbar_init(reinterpret_cast<uint64_t*>(smem + C::BAR_OFF) + g, 1);
        tc::fence_mbar_init();
    }
    if (threadIdx.x < 32) {
        tc::tmem_alloc(tbase, C::NWG * C::TCOLS);
        tc::tmem_relinquish();
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tbase + (uint32_t)(wg * C::TCOLS);
    const uint32_t trow = tmem + ((uint32_t)(i & ~31) << 16);  // this warp's lane quarter
    uint32_t phase = 0;

    const uint32_t mh = tc::smem_u32(mat_hi), ml = tc::smem_u32(mat_lo);
    const uint32_t ah = tc::smem_u32(a_hi), al = tc::smem_u32(a_lo);
    constexpr uint32_t LBO_A = (128 / 8) * 128;  // 128-row operands
    const int c = i / N;                          // window of the tile for this thread
    const int q = i % N;                          // column (sampling) / row (later stages) in the window

    auto mma_wait = [&]() {
        tc::mbar_wait(bar, phase, err);
        phase ^= 1u;
        tc::fence_after_sync();
    };
    auto sync_for_mma = [&]() {
        tc::fence_async_smem();
        tc::fence_before_sync();
        wg_sync(wg);
    };

    for (int tile = blockIdx.x * C::NWG + wg; tile < total_tiles; tile += gridDim.x * C::NWG) {
        const int item = batch_item(batch.block_start, batch.n, tile);
        const CorrParams& prm = batch.item[item];
        const long long cell = (long long)(tile - batch.block_start[item]) * C::WPT + c;
        const bool active = cell < prm.ncells;
        float4 org = make_float4(0.f, 0.f, 0.f, 0.f);  // deformed: (D(centre).x, D(centre).y, -, -)
        if constexpr (!DEFORM) {
            if (active) org = prm.origins[cell];
        }
        bool ok = active && prm.status[cell] != 0;

        // ------------------------------------------------ sampling (lane = column q of window c)
        float2 z[N];
        if constexpr (DEFORM) {
            // Deformed windows (the FP32 kernel's sampling): the predictor's bilinear blend D of
            // the four window corners, frame A at -D/2 and frame B at +D/2 from the base position.
            const int ci = active ? (int)cell : 0;
            const float4 k0 = active ? prm.corners[2 * (size_t)ci] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 k1 = active ? prm.corners[2 * (size_t)ci + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
            const int gx = min(prm.gx0 + (ci % prm.gnx) * prm.gstep, max(prm.W - N - 1, 0));
            const int gy = min(prm.gy0 + (ci / prm.gnx) * prm.gstep, max(prm.H - N - 1, 0));
            org = make_float4(corner_blend(k0.x, k0.z, k1.x, k1.z, 0.5f, 0.5f),
                              corner_blend(k0.y, k0.w, k1.y, k1.w, 0.5f, 0.5f), 0.f, 0.f);
            sample_deformed<N, 1>(prm.img_a, prm.img_b, prm.H, prm.W, gx, gy, k0, k1, q, 0, c_ramp<N>(), z);
        } else {
            sample_rows<N, false>(prm.img_a, prm.H, prm.W, org.x, org.y, q, z);
            sample_rows<N, true>(prm.img_b, prm.H, prm.W, org.z, org.w, q, z);
        }
        float2 e;
        {
            float2 s = make_float2(0.f, 0.f);
#pragma unroll
            for (int p = 0; p < N; ++p) {
                s.x += z[p].x;
                s.y += z[p].y;
            }
            s = win_sum2<N>(s, red, i, wg);
            constexpr float inv = 1.0f / (float)(N * N);
            const float ma = s.x * inv, mb = s.y * inv;
            e = make_float2(0.f, 0.f);
#pragma unroll
            for (int p = 0; p < N; ++p) {
                z[p].x = __fsub_rn(z[p].x, ma);
                z[p].y = __fsub_rn(z[p].y, mb);
                e.x += z[p].x * z[p].x;
                e.y += z[p].y * z[p].y;
            }
            e = win_sum2<N>(e, red, i, wg);
        }
        ok = ok && e.x > 1e-12f && e.y > 1e-12f;
        {  // unit-variance windows (a flat or masked window is zeroed: its result is discarded)
            const float ka = ok ? (float)N / sqrtf(e.x) : 0.0f, kb = ok ? (float)N / sqrtf(e.y) : 0.0f;
#pragma unroll
            for (int p = 0; p < N; ++p) {
                z[p].x *= ka;
                z[p].y *= kb;
            }
        }
        // F1 operands, MN-major (m = c*N + r, k = column q); frame b after frame a.
#pragma unroll
        for (int j = 0; j < N / 8; ++j) {
            float va[8], vb[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                va[t] = z[8 * j + t].x;
                vb[t] = z[8 * j + t].y;
            }
            const uint32_t off = mnmaj_chunk(128, c * N + 8 * j, q);
            store_split<F16>(a_hi, a_lo, off, va);
            store_split<F16>(a_hi + 128 * N * 2, a_lo + 128 * N * 2, off, vb);
        }
        sync_for_mma();
        if (i == 0) {
            tc::fence_after_sync();
            constexpr uint32_t id = tc::idesc_f16(128, N, !F16, true);
            constexpr uint32_t lb = (N / 8) * 128;
            for (int f = 0; f < 2; ++f)
                mma_split(tmem + f * N, ah + f * 128 * N * 2, al + f * 128 * N * 2, LBO_A, mh + C::R1_OFF * 2,
                          ml + C::R1_OFF * 2, lb, N / 16, id);
            tc::mma_commit(bar);
        }
        mma_wait();

        // ------------------------------------------------ F1 -> F2 operand (row r = q of window c)
        {
            float d[2 * N];
#pragma unroll
            for (int j = 0; j < 2 * N; j += 16) tc::tmem_ld16(trow + j, d + j);
            tc::wait_ld();
            // m = c*N + 2*kx' + f; k = r (real parts), N + r (imaginary parts)
#pragma unroll
            for (int j = 0; j < N / 8; ++j) {
                float vr[8], vi[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    vr[t] = d[(t & 1) * N + 4 * j + (t >> 1)];
                    vi[t] = d[(t & 1) * N + H2 + 4 * j + (t >> 1)];
                }
                store_split<F16>(a_hi, a_lo, mnmaj_chunk(128, c * N + 8 * j, q), vr);
                store_split<F16>(a_hi, a_lo, mnmaj_chunk(128, c * N + 8 * j, N + q), vi);
            }
        }
        sync_for_mma();
        if (i == 0) {
            tc::fence_after_sync();
            if constexpr (C::COMPACT) {
                // B = [C | S] (N rows, K = 2N); A = [Zr | Zi] (K = 2N), MN-major
                constexpr uint32_t id = tc::idesc_f16(128, N, !F16, true);
                constexpr uint32_t lb = (N / 8) * 128;
                constexpr uint32_t akoff = (N / 8) * LBO_A, bkoff = (N / 8) * lb;  // K offset N
                const uint32_t bh = mh + C::R2_OFF * 2, bl = ml + C::R2_OFF * 2;
                // Re = Zr C^T + Zi S^T
                mma_split(tmem, ah, al, LBO_A, bh, bl, lb, 2 * N / 16, id);
                // Im = Zi C^T - Zr S^T
                mma_split(tmem + N, ah + akoff, al + akoff, LBO_A, bh, bl, lb, N / 16, id);
                mma_split(tmem + N, ah, al, LBO_A, bh + bkoff, bl + bkoff, lb, N / 16, id | kNegateB, true);
            } else {
                constexpr uint32_t id = tc::idesc_f16(128, 2 * N, !F16, true);
                constexpr uint32_t lb = (2 * N / 8) * 128;
                mma_split(tmem, ah, al, LBO_A, mh + C::R2_OFF * 2, ml + C::R2_OFF * 2, lb, 2 * N / 16, id);
            }
            tc::mma_commit(bar);
        }
        mma_wait();

        // ------------------------------------------------ spectra -> cross spectrum -> I1 operand
        {
            const int fr = q & 1;  // row (w, kx' = q/2, frame fr)
            const bool dcrow = q < 2;
            float zr[N], zi[N];
#pragma unroll
            for (int j = 0; j < N; j += 16) {
                tc::tmem_ld16(trow + j, zr + j);
                tc::tmem_ld16(trow + N + j, zi + j);
            }
            tc::wait_ld();
            if (dcrow) {  // DC + i*Nyquist rows: staged for the separation below
                float* st = zst + (c * 2 + fr) * 2 * N;
#pragma unroll
                for (int j = 0; j < N; j += 4) {
                    *reinterpret_cast<float4*>(st + j) = make_float4(zr[j], zr[j + 1], zr[j + 2], zr[j + 3]);
                    *reinterpret_cast<float4*>(st + N + j) = make_float4(zi[j], zi[j + 1], zi[j + 2], zi[j + 3]);
                }
            }
            // conj(FA) * FB with FA from the frame-0 lane and FB from the frame-1 lane (lane ^ 1)
#pragma unroll
            for (int j = 0; j < N / 8; ++j) {
                float pr[8], pi[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int ky = 8 * j + t;
                    const float oar = __shfl_xor_sync(0xffffffffu, zr[ky], 1);
                    const float oai = __shfl_xor_sync(0xffffffffu, zi[ky], 1);
                    const float far_ = fr ? oar : zr[ky], fai = fr ? oai : zi[ky];
                    const float fbr = fr ? zr[ky] : oar, fbi = fr ? zi[ky] : oai;
                    const float sg = (fr && (ky & 1)) ? -C::CROSS_SCALE : C::CROSS_SCALE;  // frame-1 lane: (-1)^ky
                    pr[t] = sg * (far_ * fbr + fai * fbi);
                    pi[t] = sg * (far_ * fbi - fai * fbr);
                }
                if (!dcrow) {
                    store_split<F16>(a_hi, a_lo, kmaj_chunk(128, i, 8 * j), pr);
                    store_split<F16>(a_hi, a_lo, kmaj_chunk(128, i, N + 8 * j), pi);
                }
            }
        }
        wg_sync(wg);  // staged DC rows complete
        {
            // Lane q of window c separates column ky = q of the DC + i*Nyquist rows of both frames:
            // F(0, ky) = (Z + conj Z[-ky]) / 2, F(N/2, ky) = (Z - conj Z[-ky]) / 2i, the DC bin
            // zeroed (mean removal), and writes C(0, ky) + i C(N/2, ky) into rows (w, 0, 0) and,
            // times (-1)^ky, (w, 0, 1).
            const int ky = q, my = (N - q) % N;
            const float* sa = zst + (c * 2 + 0) * 2 * N;
            const float* sb = zst + (c * 2 + 1) * 2 * N;
            float a0r = 0.5f * (sa[ky] + sa[my]), a0i = 0.5f * (sa[N + ky] - sa[N + my]);
            const float anr = 0.5f * (sa[N + ky] + sa[N + my]), ani = 0.5f * (sa[my] - sa[ky]);
            float b0r = 0.5f * (sb[ky] + sb[my]), b0i = 0.5f * (sb[N + ky] - sb[N + my]);
            const float bnr = 0.5f * (sb[N + ky] + sb[N + my]), bni = 0.5f * (sb[my] - sb[ky]);
            if (ky == 0) a0r = a0i = b0r = b0i = 0.0f;
            const float c0r = a0r * b0r + a0i * b0i, c0i = a0r * b0i - a0i * b0r;
            const float cnr = anr * bnr + ani * bni, cni = anr * bni - ani * bnr;
            const float prr = (c0r - cni) * C::CROSS_SCALE, pri = (c0i + cnr) * C::CROSS_SCALE;
            const float sg = (ky & 1) ? -1.0f : 1.0f;
            const float vals[4] = {prr, pri, sg * prr, sg * pri};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int row = c * N + (u >> 1), k = (u & 1) * N + ky;
                const uint32_t off = kmaj_chunk(128, row, k) + (k & 7) * 2;
                if constexpr (F16) {
                    const __half h = __float2half_rn(vals[u]);
                    const __half l = __float2half_rn(vals[u] - __half2float(h));
                    *reinterpret_cast<__half*>(a_hi + off) = h;
                    *reinterpret_cast<__half*>(a_lo + off) = l;
                } else {
                    const __nv_bfloat16 h = __float2bfloat16_rn(vals[u]);
                    const __nv_bfloat16 l = __float2bfloat16_rn(vals[u] - __bfloat162float(h));
                    *reinterpret_cast<__nv_bfloat16*>(a_hi + off) = h;
                    *reinterpret_cast<__nv_bfloat16*>(a_lo + off) = l;
                }
            }
        }
        sync_for_mma();
        if (i == 0) {
            tc::fence_after_sync();
            if constexpr (C::COMPACT) {
                // B = [C | S] (N/2 rows: outputs y < N/2, K = 2N); A = [Pr | Pi] (K = 2N), K-major
                constexpr uint32_t id = tc::idesc_f16(128, H2, !F16, false);
                constexpr uint32_t lb = (H2 / 8) * 128;
                constexpr uint32_t akoff = (N / 8) * LBO_A, bkoff = (N / 8) * lb;  // K offset N
                const uint32_t bh = mh + C::R3_OFF * 2, bl = ml + C::R3_OFF * 2;
                // Re = Pr C^T - Pi S^T
                mma_split(tmem, ah, al, LBO_A, bh, bl, lb, N / 16, id);
                mma_split(tmem, ah + akoff, al + akoff, LBO_A, bh + bkoff, bl + bkoff, lb, N / 16, id | kNegateB, true);
                // Im = Pr S^T + Pi C^T
                mma_split(tmem + H2, ah, al, LBO_A, bh + bkoff, bl + bkoff, lb, N / 16, id);
                mma_split(tmem + H2, ah + akoff, al + akoff, LBO_A, bh, bl, lb, N / 16, id, true);
            } else {
                constexpr uint32_t id = tc::idesc_f16(128, N, !F16, false);
                constexpr uint32_t lb = (N / 8) * 128;
                mma_split(tmem, ah, al, LBO_A, mh + C::R3_OFF * 2, ml + C::R3_OFF * 2, lb, 2 * N / 16, id);
            }
            tc::mma_commit(bar);
        }
        mma_wait();

        // ------------------------------------------------ I1 -> I2 operand
        {
            const int kxp = q >> 1, fr = q & 1;
            float g[N];
#pragma unroll
            for (int j = 0; j < N; j += 16) tc::tmem_ld16(trow + j, g + j);
            tc::wait_ld();
            // m = c*N + y with y = fr*N/2 + j; k = kx' (real), N/2 + kx' (imaginary)
#pragma unroll
            for (int j = 0; j < H2 / 8; ++j) {
                float vr[8], vi[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    vr[t] = g[8 * j + t] * (1.0f / (float)N);
                    vi[t] = g[H2 + 8 * j + t] * (1.0f / (float)N);
                }
                const int m = c * N + fr * H2 + 8 * j;
                store_split<F16>(a_hi, a_lo, mnmaj_chunk(128, m, kxp), vr);
                store_split<F16>(a_hi, a_lo, mnmaj_chunk(128, m, H2 + kxp), vi);
            }
        }
        sync_for_mma();
        if (i == 0) {
            tc::fence_after_sync();
            constexpr uint32_t id = tc::idesc_f16(128, N, !F16, true);
            constexpr uint32_t lb = (N / 8) * 128;
            mma_split(tmem, ah, al, LBO_A, mh + C::R4_OFF * 2, ml + C::R4_OFF * 2, lb, N / 16, id);
            tc::mma_commit(bar);
        }
        mma_wait();

        // ------------------------------------------------ correlation plane, row y = q
        float v[N];
#pragma unroll
        for (int j = 0; j < N; j += 16) tc::tmem_ld16(trow + j, v + j);
        tc::wait_ld();
        tc::fence_before_sync();
        const int y = q;
        float* prow = plane + (size_t)(c * N) * C::PLD;  // window c's plane
#pragma unroll
        for (int x = 0; x < N; x += 4) {
            v[x] *= C::PLANE_SCALE;
            v[x + 1] *= C::PLANE_SCALE;
            v[x + 2] *= C::PLANE_SCALE;
            v[x + 3] *= C::PLANE_SCALE;
            *reinterpret_cast<float4*>(prow + y * C::PLD + x) = make_float4(v[x], v[x + 1], v[x + 2], v[x + 3]);
        }
        // argmax, lowest row-major index on ties
        float best = -INFINITY;
        int bi = 0x7fffffff;
#pragma unroll
        for (int x = 0; x < N; ++x)
            if (v[x] > best) {
                best = v[x];
                bi = y * N + x;
            }
        win_argmax<N>(best, bi, red, i, wg);
        if (!(best > -INFINITY)) bi = 0;
        const int by = bi / N, bx = bi % N;
        wg_sync(wg);  // plane complete
        auto at = [&](int yy, int xx) -> float { return prow[((yy + N) % N) * C::PLD + (xx + N) % N]; };
        if (q < 4) {  // footprint (correlate.rs:242-254): half-width along +y, -y, +x, -x
            const int sy = q == 0 ? 1 : (q == 1 ? N - 1 : 0);
            const int sx = q == 2 ? 1 : (q == 3 ? N - 1 : 0);
            const float half = 0.5f * best;
            int k = 0;
            while (k < N / 2 && at(by + k * sy, bx + k * sx) > half) ++k;
            s_hw[c * 4 + q] = k;
        }
        // vertical 3-maximum from the neighbouring rows
        float vm[N];
        {
            const float* up = prow + ((y + N - 1) % N) * C::PLD;
            const float* dn = prow + ((y + 1) % N) * C::PLD;
#pragma unroll
            for (int x = 0; x < N; x += 4) {
                const float4 a4 = *reinterpret_cast<const float4*>(up + x), b4 = *reinterpret_cast<const float4*>(dn + x);
                vm[x] = fmaxf(fmaxf(a4.x, b4.x), v[x]);
                vm[x + 1] = fmaxf(fmaxf(a4.y, b4.y), v[x + 1]);
                vm[x + 2] = fmaxf(fmaxf(a4.z, b4.z), v[x + 2]);
                vm[x + 3] = fmaxf(fmaxf(a4.w, b4.w), v[x + 3]);
            }
        }
        wg_sync(wg);  // footprints written
        const int hw = max(max(s_hw[c * 4 + 0], s_hw[c * 4 + 1]), max(s_hw[c * 4 + 2], s_hw[c * 4 + 3]));
        const int ex = max((int)ceilf(1.5f * (float)hw), 2);
        float second = -INFINITY;
        {
            // columns outside the footprint: circular distance from bx above ex, or every column
            // when this row is already farther than ex from by
            using Mask = std::conditional_t<(N > 32), unsigned long long, uint32_t>;
            constexpr int MB = 8 * (int)sizeof(Mask);
            const int dy = abs(y - by), cy = min(dy, N - dy);
            Mask allowed = ~Mask(0);
            if (cy <= ex) {
                Mask band = ~Mask(0);  // columns bx - ex .. bx + ex (circular)
                if (2 * ex + 1 < N) {
                    const Mask run = (Mask(1) << (2 * ex + 1)) - Mask(1);
                    const int s0 = (bx - ex + N) % N;
                    band = (run << s0) | (s0 ? run >> (N - s0) : Mask(0));
                    if constexpr (N < MB) band &= (Mask(1) << (N % MB)) - Mask(1);
                }
                allowed = ~band;
            }
#pragma unroll
            for (int x = 0; x < N; ++x) {
                const float h = fmaxf(fmaxf(vm[(x + N - 1) % N], vm[(x + 1) % N]), vm[x]);
                if (v[x] == h && ((allowed >> x) & Mask(1))) second = fmaxf(second, v[x]);
            }
        }
        second = win_max<N>(second, red, i, wg);
        if (q == 0 && active) {
            if (ok) {
                const float sx = subpixel(at(by, bx - 1), best, at(by, bx + 1));
                const float sy = subpixel(at(by - 1, bx), best, at(by + 1, bx));
                const float wx = bx >= N / 2 ? (float)bx - (float)N : (float)bx;
                const float wy = by >= N / 2 ? (float)by - (float)N : (float)by;
                const float pdx = __fadd_rn(wx, sx), pdy = __fadd_rn(wy, sy);
                if constexpr (DEFORM) {
                    prm.raw_dx[cell] = __fadd_rn(org.x, pdx);  // D(centre) + peak
                    prm.raw_dy[cell] = __fadd_rn(org.y, pdy);
                } else {
                    prm.raw_dx[cell] = __fadd_rn(__fsub_rn(org.z, org.x), pdx);
                    prm.raw_dy[cell] = __fadd_rn(__fsub_rn(org.w, org.y), pdy);
                }
                prm.raw_ppr[cell] = second > 0.0f ? fminf(__fdiv_rn(best, second), MAX_PPR) : MAX_PPR;
                prm.raw_flags[cell] = 0;
            } else {
                prm.raw_dx[cell] = NAN;
                prm.raw_dy[cell] = NAN;
                prm.raw_ppr[cell] = 0.0f;
                prm.raw_flags[cell] = F_NO_SIGNAL;
            }
        }
        wg_sync(wg);  // plane and footprints read before the next tile reuses them
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after_sync();
        tc::tmem_dealloc(*tbase, C::NWG * C::TCOLS);
    }
}

// ---------------------------------------------------------------------------------------------
// Host side: DFT matrices (split into bf16 hi / lo, laid out as the K-major shared-memory image).
// ---------------------------------------------------------------------------------------------
static uint16_t bf16_rne(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40);  // NaN
    const uint32_t r = 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)((u + r) >> 16);
}
static float bf16_f(uint16_t h) {
    const uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// cos / sin of 2*pi*k/n with the phase reduced exactly first.
static double cs(long long k, int n, bool sine) {
    const long long r = ((k % n) + n) % n;
    const double a = 2.0 * M_PI * (double)r / (double)n;
    return sine ? std::sin(a) : std::cos(a);
}

static uint16_t f16_rn(float f) {
    const __half h = __float2half_rn(f);
    uint16_t u;
    std::memcpy(&u, &h, 2);
    return u;
}
static float f16_f(uint16_t u) {
    __half h;
    std::memcpy(&h, &u, 2);
    return __half2float(h);
}

template <int N, bool F16>
static std::vector<uint16_t> build_mats() {
    using C = TcCfg<N>;
    constexpr int H2 = N / 2;
    std::vector<uint16_t> img(2 * (size_t)C::RMAT, 0);  // [hi image | lo image]
    auto put = [&](int off, int rows, int row, int k, double val) {
        const size_t e = (size_t)off + (size_t)(k >> 3) * (rows >> 3) * 64 + (size_t)(row >> 3) * 64 + (row & 7) * 8 +
                         (k & 7);  // element index of the K-major layout (64 elements per core)
        const uint16_t h = F16 ? f16_rn((float)val) : bf16_rne((float)val);
        const uint16_t l = F16 ? f16_rn((float)(val - (double)f16_f(h))) : bf16_rne((float)(val - (double)bf16_f(h)));
        img[e] = h;
        img[(size_t)C::RMAT + e] = l;
    };
    for (int n = 0; n < N; ++n)  // R1: r2c along x, packed half spectrum
        for (int x = 0; x < N; ++x) {
            double v;
            if (n < H2) v = cs((long long)n * x, N, false);
            else if (n == H2) v = (x & 1) ? -1.0 : 1.0;
            else v = -cs((long long)(n - H2) * x, N, true);
            put(C::R1_OFF, N, n, x, v);
        }
    if constexpr (C::COMPACT) {
        // [C | S] blocks: row = output (ky for F2, y < N/2 for I1), K = [cos terms | sin terms];
        // the kernel forms the other output half with B negated (see the top of the file)
        for (int n = 0; n < N; ++n)  // R2: forward complex DFT along y
            for (int k = 0; k < 2 * N; ++k)
                put(C::R2_OFF, N, n, k, cs((long long)n * (k % N), N, k >= N));
        for (int n = 0; n < H2; ++n)  // R3: inverse complex DFT along ky, outputs y < N/2
            for (int k = 0; k < 2 * N; ++k)
                put(C::R3_OFF, H2, n, k, cs((long long)(k % N) * n, N, k >= N));
    } else {
        for (int n = 0; n < 2 * N; ++n)  // R2: forward complex DFT along y
            for (int k = 0; k < 2 * N; ++k) {
                const int ky = n % N, r = k % N;
                const bool out_im = n >= N, in_im = k >= N;
                double v;
                if (!out_im) v = in_im ? cs((long long)ky * r, N, true) : cs((long long)ky * r, N, false);
                else v = in_im ? cs((long long)ky * r, N, false) : -cs((long long)ky * r, N, true);
                put(C::R2_OFF, 2 * N, n, k, v);
            }
        for (int n = 0; n < N; ++n)  // R3: inverse complex DFT along ky, outputs y < N/2
            for (int k = 0; k < 2 * N; ++k) {
                const int yy = n % H2, ky = k % N;
                const bool out_im = n >= H2, in_im = k >= N;
                double v;
                if (!out_im) v = in_im ? -cs((long long)ky * yy, N, true) : cs((long long)ky * yy, N, false);
                else v = in_im ? cs((long long)ky * yy, N, false) : cs((long long)ky * yy, N, true);
                put(C::R3_OFF, N, n, k, v);
            }
    }
    for (int x = 0; x < N; ++x)  // R4: c2r along kx from the packed half spectrum
        for (int k = 0; k < N; ++k) {
            double v;
            if (k == 0) v = 1.0;
            else if (k < H2) v = 2.0 * cs((long long)k * x, N, false);
            else if (k == H2) v = (x & 1) ? -1.0 : 1.0;
            else v = -2.0 * cs((long long)(k - H2) * x, N, true);
            put(C::R4_OFF, N, x, k, v);
        }
    return img;
}

namespace {
constexpr int kMaxDevices = 64;
// DFT matrix images per device: [size 16 | 32 | 64][BF16 | FP16]
const uint4* g_mats[kMaxDevices][3][2] = {};
int size_slot(int n) { return n == 16 ? 0 : (n == 32 ? 1 : 2); }
unsigned int* g_err_host[kMaxDevices] = {};
unsigned int* g_err_dev[kMaxDevices] = {};

template <int N, bool F16>
cudaError_t upload(const uint4** slot) {
    if (*slot) return cudaSuccess;
    const std::vector<uint16_t> img = build_mats<N, F16>();
    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, img.size() * 2);
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(d, img.data(), img.size() * 2, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return e;
    }
    *slot = reinterpret_cast<const uint4*>(d);
    return cudaSuccess;
}
}  // namespace

bool corr_tc_supported(int n) { return n == 16 || n == 32 || n == 64; }

cudaError_t corr_tc_init_device() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    e = upload<16, false>(&g_mats[dev][0][0]);
    if (e == cudaSuccess) e = upload<16, true>(&g_mats[dev][0][1]);
    if (e == cudaSuccess) e = upload<32, false>(&g_mats[dev][1][0]);
    if (e == cudaSuccess) e = upload<32, true>(&g_mats[dev][1][1]);
    if (e == cudaSuccess) e = upload<64, false>(&g_mats[dev][2][0]);
    if (e == cudaSuccess) e = upload<64, true>(&g_mats[dev][2][1]);
    if (e == cudaSuccess) {
        float r16[16], r32[32], r64[64];
        for (int i = 0; i < 16; ++i) r16[i] = (float)i / 15.0f;
        for (int i = 0; i < 32; ++i) r32[i] = (float)i / 31.0f;
        for (int i = 0; i < 64; ++i) r64[i] = (float)i / 63.0f;
        e = cudaMemcpyToSymbol(c_ramp16, r16, sizeof(r16));
        if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_ramp32, r32, sizeof(r32));
        if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_ramp64, r64, sizeof(r64));
    }
    if (e == cudaSuccess && !g_err_host[dev]) {
        e = cudaHostAlloc(reinterpret_cast<void**>(&g_err_host[dev]), sizeof(unsigned int), cudaHostAllocMapped);
        if (e == cudaSuccess) {
            *g_err_host[dev] = 0;
            e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&g_err_dev[dev]), g_err_host[dev], 0);
        }
    }
    return e;
}

unsigned int corr_tc_error(int device) {
    return (device >= 0 && device < kMaxDevices && g_err_host[device]) ? *(volatile unsigned int*)g_err_host[device] : 0u;
}

template <int N, bool F16, bool DEFORM>
static cudaError_t launch_tc(CorrBatch b, cudaStream_t s, const uint4* mats, unsigned int* err) {
    using C = TcCfg<N>;
    long long total = 0;
    for (int i = 0; i < b.n; ++i) {
        b.block_start[i] = (int)total;
        total += (b.item[i].ncells + C::WPT - 1) / C::WPT;
    }
    b.block_start[b.n] = (int)total;
    if (total <= 0) return cudaSuccess;
    if (total > 0x7fffffffll) return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    auto kern = correlate_tc_kernel<N, F16, DEFORM>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (e != cudaSuccess) return e;
    const long long ctas = std::min<long long>((total + C::NWG - 1) / C::NWG, (long long)sms * C::CTAS_PER_SM);
    kern<<<(unsigned)ctas, C::THREADS, C::SMEM, s>>>(b, mats, (int)total, err);
    return cudaGetLastError();
}

cudaError_t launch_correlate_tc_items(int n, bool f16, const CorrParams* items, int count, cudaStream_t s,
                                      int* launches) {
    if (count <= 0) return cudaSuccess;
    if (!corr_tc_supported(n)) return cudaErrorInvalidValue;
    const bool deform = items[0].corners != nullptr;
    for (int i = 0; i < count; ++i)
        if ((items[i].corners != nullptr) != deform) return cudaErrorInvalidValue;  // one kind per launch
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices || !g_err_dev[dev]) return cudaErrorInitializationError;
    for (int off = 0; off < count; off += kMaxBatch) {
        CorrBatch b;
        b.n = count - off < kMaxBatch ? count - off : kMaxBatch;
        for (int i = 0; i < b.n; ++i) b.item[i] = items[off + i];
        const uint4* m = g_mats[dev][size_slot(n)][f16 ? 1 : 0];
        unsigned int* err = g_err_dev[dev];
        if (n == 16) {
            if (deform) e = f16 ? launch_tc<16, true, true>(b, s, m, err) : launch_tc<16, false, true>(b, s, m, err);
            else e = f16 ? launch_tc<16, true, false>(b, s, m, err) : launch_tc<16, false, false>(b, s, m, err);
        } else if (n == 32) {
            if (deform) e = f16 ? launch_tc<32, true, true>(b, s, m, err) : launch_tc<32, false, true>(b, s, m, err);
            else e = f16 ? launch_tc<32, true, false>(b, s, m, err) : launch_tc<32, false, false>(b, s, m, err);
        } else {
            if (deform) e = f16 ? launch_tc<64, true, true>(b, s, m, err) : launch_tc<64, false, true>(b, s, m, err);
            else e = f16 ? launch_tc<64, true, false>(b, s, m, err) : launch_tc<64, false, false>(b, s, m, err);
        }
        if (e != cudaSuccess) return e;
        if (launches) ++*launches;
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------------------------------------
// Self-test of the tensor-core building blocks: D (128 x n) = A (128 x k) * B (n x k)^T with
// BF16 operands (the inputs are rounded to bf16 on the way in) and FP32 accumulation, A stored
// K-major or MN-major exactly as the correlation kernel stores its operands.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1)
    tc_selftest_kernel(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ d, int n, int k,
                       int a_mn, unsigned int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    // A: 128 x k, B: n x k (bf16), then the barrier and the TMEM address
    uint8_t* sa = smem;
    uint8_t* sb = smem + 128 * k * 2;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sb + n * k * 2);
    uint32_t* tbase = reinterpret_cast<uint32_t*>(bar + 1);
    const int i = threadIdx.x;
    // element writes (scalar; this is a test)
    for (int e = i; e < 128 * k; e += 128) {
        const int m = e / k, kk = e % k;
        const uint32_t off = a_mn ? mnmaj_chunk(128, m & ~7, kk) + (m & 7) * 2 : kmaj_chunk(128, m, kk & ~7) + (kk & 7) * 2;
        *reinterpret_cast<__nv_bfloat16*>(sa + off) = __float2bfloat16_rn(a[e]);
    }
    for (int e = i; e < n * k; e += 128) {
        const int r = e / k, kk = e % k;
        *reinterpret_cast<__nv_bfloat16*>(sb + kmaj_chunk(n, r, kk & ~7) + (kk & 7) * 2) = __float2bfloat16_rn(b[e]);
    }
    if (i == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    if (i < 32) {
        tc::tmem_alloc(tbase, 256);
        tc::tmem_relinquish();
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tbase;
    if (i == 0) {
        const uint32_t id = tc::idesc_f16(128, n, true, a_mn != 0);
        const uint32_t la = 16 * 128, lb = (uint32_t)(n / 8) * 128;
        const uint32_t a0 = tc::smem_u32(sa), b0 = tc::smem_u32(sb);
        for (int s = 0; s < k / 16; ++s)
            tc::mma_f16(tmem, tc::smem_desc(a0 + 2 * s * la, la, 128), tc::smem_desc(b0 + 2 * s * lb, lb, 128), id,
                        s > 0 ? 1u : 0u);
        tc::mma_commit(bar);
    }
    tc::mbar_wait(bar, 0, err);
    tc::fence_after_sync();
    for (int j = 0; j < n; j += 16) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(i & ~31) << 16) + j, v);
        tc::wait_ld();
        for (int t = 0; t < 16; ++t) d[i * n + j + t] = v[t];
    }
    tc::fence_before_sync();
    __syncthreads();
    if (i < 32) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 256);
    }
}

// The bounded wait of the correlation kernel on an mbarrier that nothing arrives on: the wait
// runs out after 2^log2_iters try_wait rounds and records that in `err`.
__global__ void tc_wait_probe_kernel(unsigned int* err, int log2_iters) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) tc::mbar_wait(&bar, 0, err, log2_iters);
}

cudaError_t tc_wait_probe(int log2_iters, unsigned int* timed_out, float* ms) {
    if (log2_iters < 0 || log2_iters > tc::kWaitLog2Iters) return cudaErrorInvalidValue;
    unsigned int* word = nullptr;  // host-mapped, private to the probe
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&word), sizeof(unsigned int), cudaHostAllocMapped);
    if (e != cudaSuccess) return e;
    *word = 0;
    unsigned int* dword = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&dword), word, 0);
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    if (e == cudaSuccess) e = cudaEventRecord(t0, 0);
    if (e == cudaSuccess) {
        tc_wait_probe_kernel<<<1, 32>>>(dword, log2_iters);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(t1, 0);
    if (e == cudaSuccess) e = cudaEventSynchronize(t1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, t0, t1);
    if (e == cudaSuccess) *timed_out = *(volatile unsigned int*)word;
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFreeHost(word);
    return e;
}

cudaError_t tc_selftest(int a_mn, int n, int k, const float* a, const float* b, float* d) {
    if (n < 16 || n > 256 || n % 16 || k < 16 || k > 256 || k % 16) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices || !g_err_dev[dev]) return cudaErrorInitializationError;
    const size_t smem = (size_t)128 * k * 2 + (size_t)n * k * 2 + 64;
    e = cudaFuncSetAttribute(tc_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    tc_selftest_kernel<<<1, 128, smem>>>(a, b, d, n, k, a_mn, g_err_dev[dev]);
    return cudaGetLastError();
}

}  // namespace pivb200
