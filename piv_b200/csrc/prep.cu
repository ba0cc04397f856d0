// Frame preparation: PreparedFrame::new (preprocess.rs:138-158) on the device.
//
//   raw u8/u16 -> f32 as v/255 or v/65535 (decode.rs:227-234); f32 frames pass through
//   optional percentile clip of the integer codes (not in the reference; see below)
//   base = max(raw - background, 0)                     preprocess.rs:140-142
//   integral tables of base for the signal mask          preprocess.rs:76-125 (exact int64 here)
//   separable Gaussian blur, radius ceil(3 sigma), clamped edges, f32 sums in kernel order
//                                                        preprocess.rs:161-195
//   local mean/std normalization over the clipped (2r+1)^2 box    preprocess.rs:199-216
//
// The blur repeats the reference's f32 operations in order (no FMA), so it is bit-exact given
// the same kernel weights. The normalization's box statistics are exact integer sums turned into
// f32 mean/std by the reference's steps (mean = s/n, var = sq/n - mean^2, sqrt) in double-float
// arithmetic (fix_stats in common.cuh; no FP64 instruction). These sums are exact where the
// reference's f64 integral image can round, and double-float carries ~48 of f64's 53 bits, so a
// result can differ from the reference's in a rounding-boundary case.
//
// Percentile clip (an addition, parity unpinned against the reference, pinned against the
// oracle): the clip code is the smallest code c with #(codes <= c) >= ceil(p/100 * H*W); codes
// above it are set to it before conversion. Found with two 256-bin histogram passes.
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace pivb200 {

constexpr int kMaxBlurTaps = 65;  // radius <= 32
constexpr int kMaxNormRadius = 16;

struct BlurKernel {
    float w[kMaxBlurTaps];
    int radius;
};

// ------------------------------------------------------------------------------- percentile
template <typename CodeT>
__global__ void hist_kernel(const CodeT* __restrict__ raw, long long n, unsigned int* hist, int level,
                            const unsigned int* sel) {
    __shared__ unsigned int h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const unsigned int coarse = level ? sel[0] : 0u;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned int c = raw[i];
        if (level == 0)
            atomicAdd(&h[c >> 8], 1u);
        else if ((c >> 8) == coarse)
            atomicAdd(&h[c & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

// sel[0] = coarse bin, sel[1] = remaining rank inside it; level 1 writes sel[2] = clip code.
__global__ void select_kernel(const unsigned int* hist, unsigned int* sel, unsigned long long target, int level) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long acc = 0, want = level == 0 ? target : sel[1];
    for (int b = 0; b < 256; ++b) {
        if (acc + hist[b] >= want) {
            if (level == 0) {
                sel[0] = b;
                sel[1] = (unsigned int)(want - acc);
            } else {
                sel[2] = (sel[0] << 8) | (unsigned int)b;
            }
            return;
        }
        acc += hist[b];
    }
    if (level == 0) {
        sel[0] = 255;
        sel[1] = 0;
    } else {
        sel[2] = (sel[0] << 8) | 255u;
    }
}

// ------------------------------------------------------------------------------- conversion
// Integer codes to f32 as decode.rs:227-234 divides them: c / 255 (u8) or c / 65535 (u16),
// correctly rounded. The quotient is c * RN(1/d) corrected once by its exact residual
// (Markstein's method): q0 = RN(c r), e = fma(-q0, d, c), q = fma(e, r, q0); for these two
// divisors it equals the correctly rounded quotient for every code (checked exhaustively against
// exact rational arithmetic, and on the GPU against IEEE division).
template <typename CodeT>
struct CodeDivisor;
template <>
struct CodeDivisor<uint8_t> {
    static constexpr float d = 255.0f;
};
template <>
struct CodeDivisor<uint16_t> {
    static constexpr float d = 65535.0f;
};

__device__ __forceinline__ float div_code(float x, float d, float r) {
    const float q0 = __fmul_rn(x, r);
    return __fmaf_rn(__fmaf_rn(-q0, d, x), r, q0);
}

// The background-subtracted intensity of one sample (preprocess.rs:144-151): an integer code
// clipped to the percentile code, divided as above, then the background subtracted and clamped
// at zero. `begin()` reads the clip code on the device once per thread.
template <typename CodeT>
struct CodeSamples {
    const CodeT* raw;
    const float* bg;  // nullable
    const unsigned int* clip;  // nullable; clip[2] is the clip code
    unsigned int cl;
    float d, r;
    __device__ __forceinline__ void begin() {
        cl = clip ? clip[2] : 0xffffffffu;
        d = CodeDivisor<CodeT>::d;
        r = __frcp_rn(d);
    }
    __device__ __forceinline__ float value(unsigned int c, float b) const {
        if (c > cl) c = cl;
        float v = div_code((float)c, d, r);
        if (bg) v = fmaxf(__fsub_rn(v, b), 0.0f);
        return v;
    }
    __device__ __forceinline__ float operator()(size_t i) const { return value(raw[i], bg ? bg[i] : 0.0f); }
};

// f32 samples, background-subtracted and clamped at zero when a background is given.
struct FloatSamples {
    const float* raw;
    const float* bg;  // nullable
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ float operator()(size_t i) const {
        float v = raw[i];
        if (bg) v = fmaxf(__fsub_rn(v, bg[i]), 0.0f);
        return v;
    }
};

// Streams codes 16 bytes per load (8 u16 or 16 u8) when the buffers are 16-byte aligned; the
// rest of the frame (or an unaligned one) one code at a time.
template <typename CodeT>
__global__ void convert_kernel(const CodeT* __restrict__ raw, long long n, const float* __restrict__ bg,
                               const unsigned int* clip, float* __restrict__ out) {
    constexpr int V = 16 / (int)sizeof(CodeT);
    CodeSamples<CodeT> src{raw, bg, clip, 0u, 0.0f, 0.0f};
    src.begin();
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    auto value = [&](unsigned int c, float b) { return src.value(c, b); };
    long long head = 0;
    const bool aligned = (reinterpret_cast<uintptr_t>(raw) | reinterpret_cast<uintptr_t>(out) |
                          reinterpret_cast<uintptr_t>(bg)) % 16 == 0;
    if (aligned) {
        const long long nv = n / V;
        for (long long j = tid; j < nv; j += stride) {
            union {
                uint4 w;
                CodeT c[V];
            } u;
            u.w = __ldg(reinterpret_cast<const uint4*>(raw) + j);
#pragma unroll
            for (int k = 0; k < V; k += 4) {
                float4 b = make_float4(0.f, 0.f, 0.f, 0.f);
                if (bg) b = __ldg(reinterpret_cast<const float4*>(bg + j * V + k));
                float4 o;
                o.x = value(u.c[k], b.x);
                o.y = value(u.c[k + 1], b.y);
                o.z = value(u.c[k + 2], b.z);
                o.w = value(u.c[k + 3], b.w);
                *reinterpret_cast<float4*>(out + j * V + k) = o;
            }
        }
        head = nv * V;
    }
    for (long long i = head + tid; i < n; i += stride) out[i] = value(raw[i], bg ? bg[i] : 0.0f);
}

__global__ void convert_f32_kernel(const float* __restrict__ raw, long long n, const float* __restrict__ bg,
                                   float* __restrict__ out) {
    const FloatSamples src{raw, bg};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = src((size_t)i);
}

// ------------------------------------------------------------------------------- max |v|
// One atomic per block (the block's warps reduce through shared memory first); launched with
// 256 threads.
// Folds each thread's running max |v| into *out: one atomic per block of <= 256 threads. Every
// thread of the block calls it.
__device__ __forceinline__ void block_max_to(float m, unsigned int* out) {
    __shared__ float wmax[8];
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? wmax[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) atomicMax(out, __float_as_uint(m));  // non-negative floats order as uints
    }
}

__global__ void maxabs_kernel(const float* __restrict__ v, long long n, unsigned int* out) {
    float m = 0.0f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(v[i]));
    block_max_to(m, out);
}

// ------------------------------------------------------------------------------- integral tables
// Row pass: T[y+1][x+1] = sum_{x' <= x} q(v[y][x']) for both tables; T[y+1][0] = 0.
__global__ void integral_rows_kernel(const float* __restrict__ v, int H, int W, long long* sum, long long* sumsq,
                                     const unsigned int* maxbits, int* scales) {
    const int y = blockIdx.x;
    const FixScale fs = fix_scale(__uint_as_float(*maxbits), (long long)H * W);
    if (y == 0 && threadIdx.x == 0) {
        scales[0] = fs.s1;
        scales[1] = fs.s2;
    }
    const int stride = W + 1;
    long long* r1 = sum + (size_t)(y + 1) * stride;
    long long* r2 = sumsq + (size_t)(y + 1) * stride;
    const float* row = v + (size_t)y * W;
    __shared__ long long c1[32], c2[32];
    __shared__ long long carry1, carry2;
    if (threadIdx.x == 0) {
        r1[0] = 0;
        r2[0] = 0;
        carry1 = 0;
        carry2 = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < W; base += blockDim.x) {
        const int x = base + threadIdx.x;
        long long a = 0, b = 0;
        if (x < W) {
            const float f = row[x];
            a = fix_q1(f, fs);
            b = fix_q2(f, fs);
        }
        for (int o = 1; o < 32; o <<= 1) {
            const long long ua = __shfl_up_sync(0xffffffffu, a, o), ub = __shfl_up_sync(0xffffffffu, b, o);
            if (lane >= o) {
                a += ua;
                b += ub;
            }
        }
        if (lane == 31) {
            c1[warp] = a;
            c2[warp] = b;
        }
        __syncthreads();
        if (warp == 0) {
            long long wa = lane < nw ? c1[lane] : 0, wb = lane < nw ? c2[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const long long ua = __shfl_up_sync(0xffffffffu, wa, o), ub = __shfl_up_sync(0xffffffffu, wb, o);
                if (lane >= o) {
                    wa += ua;
                    wb += ub;
                }
            }
            if (lane < nw) {
                c1[lane] = wa;
                c2[lane] = wb;
            }
        }
        __syncthreads();
        const long long off1 = carry1 + (warp > 0 ? c1[warp - 1] : 0);
        const long long off2 = carry2 + (warp > 0 ? c2[warp - 1] : 0);
        if (x < W) {
            r1[x + 1] = a + off1;
            r2[x + 1] = b + off2;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry1 += c1[nw - 1];
            carry2 += c2[nw - 1];
        }
        __syncthreads();
    }
}

// Column pass: cumulative sums down each column of both tables (rows 1..H). Row 0 is zero.
__global__ void integral_cols_kernel(int H, int W, long long* sum, long long* sumsq) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = W + 1;
    if (x > W) return;
    sum[x] = 0;
    sumsq[x] = 0;
    long long a = 0, b = 0;
    int y = 1;
    for (; y + 4 <= H + 1; y += 4) {
        long long va[4], vb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            va[i] = sum[(size_t)(y + i) * stride + x];
            vb[i] = sumsq[(size_t)(y + i) * stride + x];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            a += va[i];
            b += vb[i];
            sum[(size_t)(y + i) * stride + x] = a;
            sumsq[(size_t)(y + i) * stride + x] = b;
        }
    }
    for (; y <= H; ++y) {
        a += sum[(size_t)y * stride + x];
        b += sumsq[(size_t)y * stride + x];
        sum[(size_t)y * stride + x] = a;
        sumsq[(size_t)y * stride + x] = b;
    }
}

// ------------------------------------------------------------------------------- blur
constexpr int BT_X = 32, BT_Y = 32;
constexpr int kBlurThreads = 256;  // the blur's launch width; its loops stride by it

// The tile load reads samples through `Src`: the previous stage's f32 image, or (when nothing
// else needs the background-subtracted image) the raw frame decoded on the fly, which saves the
// conversion kernel and its H x W f32 round trip. With a non-null `maxout` the kernel also folds
// max |output| into *maxout for the local normalisation's fixed-point scale (launched with 256
// threads).
// RC > 0 fixes the radius at compile time (the taps unroll; the summation order is unchanged);
// RC = 0 takes it from k.
template <typename Src, int RC>
__global__ void blur_kernel(Src src, int H, int W, const BlurKernel k, float* __restrict__ out,
                            unsigned int* maxout) {
    extern __shared__ float sm[];
    src.begin();
    const int R = RC > 0 ? RC : k.radius;
    const int TW = BT_X + 2 * R, TH = BT_Y + 2 * R;
    float* tin = sm;             // TH x TW
    float* trow = sm + TH * TW;  // TH x BT_X
    const int gx0 = blockIdx.x * BT_X, gy0 = blockIdx.y * BT_Y;
    // i / TW as a multiply-high by ceil(2^32 / TW), exact for i * TW < 2^32.
    const unsigned int tw_magic = 0xffffffffu / (unsigned int)TW + 1u;
#pragma unroll 2
    for (int i = threadIdx.x; i < TH * TW; i += kBlurThreads) {
        const int ty = (int)__umulhi((unsigned int)i, tw_magic), tx = i - ty * TW;
        const int gy = min(max(gy0 + ty - R, 0), H - 1);
        const int gx = min(max(gx0 + tx - R, 0), W - 1);
        tin[i] = src((size_t)gy * W + gx);
    }
    __syncthreads();
    // Row pass over every tile row (vertical halo included): sum in kernel order from -0.0.
#pragma unroll
    for (int i = threadIdx.x; i < TH * BT_X; i += kBlurThreads) {
        const int ty = i / BT_X, tx = i % BT_X;
        float s = -0.0f;
#pragma unroll
        for (int j = 0; j <= 2 * R; ++j) s = __fadd_rn(s, __fmul_rn(k.w[j], tin[ty * TW + tx + j]));
        trow[i] = s;
    }
    __syncthreads();
    // Column pass: out starts at 0.0 and accumulates kernel terms in order (preprocess.rs:186-193).
    float m = 0.0f;
#pragma unroll
    for (int i = threadIdx.x; i < BT_X * BT_Y; i += kBlurThreads) {
        const int ty = i / BT_X, tx = i % BT_X;
        const int gx = gx0 + tx, gy = gy0 + ty;
        if (gx >= W || gy >= H) continue;
        float o = 0.0f;
#pragma unroll
        for (int j = 0; j <= 2 * R; ++j) o = __fadd_rn(o, __fmul_rn(k.w[j], trow[(ty + j) * BT_X + tx]));
        out[(size_t)gy * W + gx] = o;
        m = fmaxf(m, fabsf(o));
    }
    if (maxout) block_max_to(m, maxout);
}

// ------------------------------------------------------------------------------- normalize
constexpr int NT_X = 32, NT_Y = 32;
constexpr int NT_RUN = 4;  // output rows per thread in the column pass (256 threads = 32 columns x 8 runs)
constexpr int NT_XRUN = 4;  // outputs per thread in the row pass
constexpr int NT_HW = NT_X + 1;  // row stride of the row-pass sums (odd, in 8-byte words)
constexpr int kNormThreads = 256;  // the launch width; the loops stride by it

// RC > 0 fixes the radius at compile time; RC = 0 takes it from r_arg.
template <int RC>
__global__ void normalize_kernel(const float* __restrict__ src, int H, int W, int r_arg, float eps,
                                 const unsigned int* maxbits, float* __restrict__ out) {
    extern __shared__ long long smq[];
    const int r = RC > 0 ? RC : r_arg;
    const int TW = NT_X + 2 * r, TH = NT_Y + 2 * r;
    // Row strides in 8-byte words are odd (QW, NT_HW), so 16 lanes on 16 consecutive rows of one
    // column hit 16 different bank pairs.
    const int QW = TW | 1;
    long long* q1 = smq;                 // TH x QW
    long long* q2 = q1 + TH * QW;        // TH x QW
    long long* h1 = q2 + TH * QW;        // TH x NT_HW
    long long* h2 = h1 + TH * NT_HW;     // TH x NT_HW
    const FixScale fs = fix_scale(__uint_as_float(*maxbits), (long long)(2 * r + 1) * (2 * r + 1));
    const int gx0 = blockIdx.x * NT_X, gy0 = blockIdx.y * NT_Y;
    // i / TW as a multiply-high by ceil(2^32 / TW): exact while i * TW < 2^32, which the tile's
    // shared-memory size guarantees by far.
    const unsigned int tw_magic = 0xffffffffu / (unsigned int)TW + 1u;
#pragma unroll 2
    for (int i = threadIdx.x; i < TH * TW; i += kNormThreads) {
        const int ty = (int)__umulhi((unsigned int)i, tw_magic), tx = i - ty * TW;
        const int gy = gy0 + ty - r, gx = gx0 + tx - r;
        long long a = 0, b = 0;
        if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
            const float f = src[(size_t)gy * W + gx];
            a = fix_q1(f, fs);
            b = fix_q2(f, fs);
        }
        q1[ty * QW + tx] = a;
        q2[ty * QW + tx] = b;
    }
    __syncthreads();
    // Row pass: each thread slides a (2r+1)-tap window along NT_XRUN outputs of one tile row;
    // consecutive threads take consecutive rows. The sums are exact integers, so sliding gives
    // the same totals as summing afresh.
    const unsigned int th_magic = 0xffffffffu / (unsigned int)TH + 1u;
    for (int i = threadIdx.x; i < TH * (NT_X / NT_XRUN); i += kNormThreads) {
        const int run = (int)__umulhi((unsigned int)i, th_magic), row = i - run * TH;
        const long long* p1 = q1 + row * QW + run * NT_XRUN;
        const long long* p2 = q2 + row * QW + run * NT_XRUN;
        long long* o1 = h1 + row * NT_HW + run * NT_XRUN;
        long long* o2 = h2 + row * NT_HW + run * NT_XRUN;
        // Two accumulators per table shorten the first sum's add chains.
        long long a0 = p1[0], b0 = p2[0], a1 = 0, b1 = 0;
        int j = 1;
#pragma unroll
        for (; j + 1 <= 2 * r; j += 2) {
            a0 += p1[j];
            a1 += p1[j + 1];
            b0 += p2[j];
            b1 += p2[j + 1];
        }
        if (j <= 2 * r) {
            a0 += p1[j];
            b0 += p2[j];
        }
        long long a = a0 + a1, b = b0 + b1;
        o1[0] = a;
        o2[0] = b;
#pragma unroll
        for (int k = 1; k < NT_XRUN; ++k) {
            a += p1[k + 2 * r] - p1[k - 1];
            b += p2[k + 2 * r] - p2[k - 1];
            o1[k] = a;
            o2[k] = b;
        }
    }
    __syncthreads();
    // Column pass: each thread slides a (2r+1)-row window down NT_RUN output rows of one column
    // (the sums are exact integers, so sliding gives the same totals as summing afresh).
    for (int i = threadIdx.x; i < NT_X * (NT_Y / NT_RUN); i += kNormThreads) {
        const int tx = i % NT_X, ty0 = (i / NT_X) * NT_RUN;
        const int gx = gx0 + tx;
        long long a = 0, b = 0;
#pragma unroll
        for (int j = 0; j <= 2 * r; ++j) {
            a += h1[(ty0 + j) * NT_HW + tx];
            b += h2[(ty0 + j) * NT_HW + tx];
        }
        for (int k = 0; k < NT_RUN; ++k) {
            const int ty = ty0 + k, gy = gy0 + ty;
            if (k > 0) {
                a += h1[(ty + 2 * r) * NT_HW + tx] - h1[(ty - 1) * NT_HW + tx];
                b += h2[(ty + 2 * r) * NT_HW + tx] - h2[(ty - 1) * NT_HW + tx];
            }
            if (gx >= W || gy >= H) continue;
            const int x0 = max(gx - r, 0), x1 = min(gx + r + 1, W);
            const int y0 = max(gy - r, 0), y1 = min(gy + r + 1, H);
            float mean, sd;
            fix_stats(a, b, fs, (float)((x1 - x0) * (y1 - y0)), &mean, &sd);
            const float v = src[(size_t)gy * W + gx];
            out[(size_t)gy * W + gx] = __fdiv_rn(__fsub_rn(v, mean), __fadd_rn(sd, eps));
        }
    }
}

// ------------------------------------------------------------------------------- drivers
// Launches the blur through sample source `src`: the radius-3 instantiation (sigma 1, the
// default) or the general one, which is opted into more than 48 KB of dynamic shared memory when
// its tile needs it.
template <typename Src>
static cudaError_t run_blur(dim3 grid, size_t sm, cudaStream_t s, const Src& src, int H, int W, const BlurKernel& k,
                            float* dst, unsigned int* mx) {
    if (k.radius == 3) {
        blur_kernel<Src, 3><<<grid, kBlurThreads, sm, s>>>(src, H, W, k, dst, mx);
        return cudaSuccess;
    }
    if (sm > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(blur_kernel<Src, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
    }
    blur_kernel<Src, 0><<<grid, kBlurThreads, sm, s>>>(src, H, W, k, dst, mx);
    return cudaSuccess;
}

static int grid_for(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

// ------------------------------------------------------------------------------- reference tables
// IntegralImage's f64 summed-area tables (preprocess.rs:76-103), handed over by a caller that
// prepared its frames on the host, are turned into this library's int64 fixed-point tables in
// place (each f64 entry's 8 bytes become its int64 entry): q = round(T * 2^s), with s chosen per
// table from its largest |entry| so that every entry and every 4-term box difference fits in
// int64. Only integer operations on the f64 bit patterns are used (no FP64 instruction). Entries
// whose f64 spacing is below 2^-s are rounded to the nearest multiple of 2^-s (ties to even);
// box sums are then exact differences of these entries.
__global__ void table_maxbits_kernel(const unsigned long long* __restrict__ t, long long n, unsigned long long* out,
                                     unsigned int* nonfinite) {
    unsigned long long m = 0;
    bool bad = false;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long b = t[i] & 0x7fffffffffffffffull;
        if ((b >> 52) == 0x7ffull) bad = true;
        else m = b > m ? b : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, m, o);
        m = v > m ? v : m;
    }
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(nonfinite, 1u);
}

// Scale exponent s with max|T| * 2^s < 2^61 (headroom for the box differences).
__device__ __forceinline__ int table_scale(unsigned long long maxbits) {
    if (!maxbits) return 0;
    const int e = (int)(maxbits >> 52) - 1022;  // max|T| < 2^e
    return 61 - e;
}

__device__ __forceinline__ long long f64_bits_to_fixed(unsigned long long bits, int s) {
    const bool neg = bits >> 63;
    const int be = (int)((bits >> 52) & 0x7ff);
    if (be == 0x7ff) return 0;  // non-finite: reported through the flag, never used
    unsigned long long m = bits & 0x000fffffffffffffull;
    int k;  // |value| = m * 2^k
    if (be) {
        m |= 1ull << 52;
        k = be - 1075;
    } else {
        k = -1074;
    }
    k += s;
    unsigned long long q;
    if (k >= 0) {
        q = m << k;  // the scale keeps |value| * 2^s below 2^61
    } else if (-k >= 64) {
        q = 0;  // below half a quantum
    } else {
        const int r = -k;
        q = m >> r;
        const unsigned long long rem = m & ((1ull << r) - 1), half = 1ull << (r - 1);
        if (rem > half || (rem == half && (q & 1))) ++q;
    }
    return neg ? -(long long)q : (long long)q;
}

__global__ void table_to_fixed_kernel(unsigned long long* t, long long n, const unsigned long long* maxbits,
                                      int* scale_out) {
    const int s = table_scale(*maxbits);
    if (blockIdx.x == 0 && threadIdx.x == 0) *scale_out = s;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        t[i] = (unsigned long long)f64_bits_to_fixed(t[i], s);
}

cudaError_t launch_stats(const float* base, int H, int W, long long* sum, long long* sumsq, int* scales,
                         unsigned int* maxbits, cudaStream_t s, int* launches) {
    const long long n = (long long)H * W;
    cudaError_t e = cudaMemsetAsync(maxbits, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    maxabs_kernel<<<grid_for(n), 256, 0, s>>>(base, n, maxbits);
    integral_rows_kernel<<<H, 256, 0, s>>>(base, H, W, sum, sumsq, maxbits, scales);
    integral_cols_kernel<<<(W + 1 + 127) / 128, 128, 0, s>>>(H, W, sum, sumsq);
    if (launches) *launches += 3;
    return cudaGetLastError();
}

// Blur weights exactly as preprocess.rs:162-168 computes them (f32 exp of an f32 argument,
// normalised by their f32 sum in order).
static BlurKernel make_blur(float sigma) {
    BlurKernel k{};
    const int radius = (int)std::max(std::ceil(3.0f * sigma), 1.0f);
    k.radius = radius;
    float total = 0.0f;
    for (int i = -radius; i <= radius; ++i) {
        const float v = std::exp(-(float)(i * i) / (2.0f * sigma * sigma));
        k.w[i + radius] = v;
    }
    for (int j = 0; j <= 2 * radius; ++j) total += k.w[j];
    for (int j = 0; j <= 2 * radius; ++j) k.w[j] /= total;
    return k;
}

cudaError_t launch_tables_to_fixed(long long* sum, long long* sumsq, int H, int W, int* scales,
                                   unsigned long long* maxbits2, unsigned int* nonfinite, cudaStream_t s, int* launches) {
    const long long n = (long long)(H + 1) * (W + 1);
    cudaError_t e = cudaMemsetAsync(maxbits2, 0, 2 * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(nonfinite, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    unsigned long long* t1 = reinterpret_cast<unsigned long long*>(sum);
    unsigned long long* t2 = reinterpret_cast<unsigned long long*>(sumsq);
    table_maxbits_kernel<<<grid_for(n), 256, 0, s>>>(t1, n, maxbits2, nonfinite);
    table_maxbits_kernel<<<grid_for(n), 256, 0, s>>>(t2, n, maxbits2 + 1, nonfinite);
    table_to_fixed_kernel<<<grid_for(n), 256, 0, s>>>(t1, n, maxbits2, scales);
    table_to_fixed_kernel<<<grid_for(n), 256, 0, s>>>(t2, n, maxbits2 + 1, scales + 1);
    if (launches) *launches += 4;
    return cudaGetLastError();
}

cudaError_t launch_prepare(const PrepParams& p, cudaStream_t s, int* launches) {
    const long long n = (long long)p.H * p.W;
    cudaError_t e;
    int nl = 0;
    const unsigned int* clip = nullptr;
    if (p.clip_percentile_on && (p.raw_type == RAW_U8 || p.raw_type == RAW_U16)) {
        e = cudaMemsetAsync(p.hist, 0, sizeof(unsigned int) * (512 + 4), s);
        if (e != cudaSuccess) return e;
        double pc = std::min(std::max(p.clip_percentile, 0.0), 100.0);
        unsigned long long target = (unsigned long long)std::ceil(pc / 100.0 * (double)n);
        if (target < 1) target = 1;
        unsigned int* h0 = p.hist;
        unsigned int* h1 = p.hist + 256;
        unsigned int* sel = p.hist + 512;
        if (p.raw_type == RAW_U16) {
            hist_kernel<uint16_t><<<grid_for(n), 256, 0, s>>>((const uint16_t*)p.raw, n, h0, 0, sel);
            select_kernel<<<1, 32, 0, s>>>(h0, sel, target, 0);
            hist_kernel<uint16_t><<<grid_for(n), 256, 0, s>>>((const uint16_t*)p.raw, n, h1, 1, sel);
        } else {
            hist_kernel<uint8_t><<<grid_for(n), 256, 0, s>>>((const uint8_t*)p.raw, n, h0, 0, sel);
            select_kernel<<<1, 32, 0, s>>>(h0, sel, target, 0);
            hist_kernel<uint8_t><<<grid_for(n), 256, 0, s>>>((const uint8_t*)p.raw, n, h1, 1, sel);
        }
        select_kernel<<<1, 32, 0, s>>>(h1, sel, target, 1);
        nl += 4;
        clip = sel;
    }
    const bool blur = p.smooth_sigma > 0.0f;
    const bool norm = p.normalize_radius > 0;
    // base goes straight to `image` when no further stage follows. When the blur follows and no
    // integral tables are wanted, the blur decodes the raw samples itself and base is not written.
    float* base = p.base;
    const bool fused = blur && !p.build_stats;
    if (!fused) switch (p.raw_type) {
        case RAW_U8:
            convert_kernel<uint8_t><<<grid_for(n), 256, 0, s>>>((const uint8_t*)p.raw, n, p.background, clip, base);
            break;
        case RAW_U16:
            convert_kernel<uint16_t><<<grid_for(n), 256, 0, s>>>((const uint16_t*)p.raw, n, p.background, clip, base);
            break;
        default:
            convert_f32_kernel<<<grid_for(n), 256, 0, s>>>((const float*)p.raw, n, p.background, base);
            break;
    }
    if (!fused) nl += 1;
    if (p.build_stats) {
        e = launch_stats(base, p.H, p.W, p.sum, p.sumsq, p.scales, p.maxbits, s, &nl);
        if (e != cudaSuccess) return e;
    }
    const float* cur = base;
    if (blur) {
        const BlurKernel k = make_blur(p.smooth_sigma);
        if (k.radius > (kMaxBlurTaps - 1) / 2) return cudaErrorInvalidValue;
        const int R = k.radius;
        const size_t sm = sizeof(float) * ((size_t)(BT_Y + 2 * R) * (BT_X + 2 * R) + (size_t)(BT_Y + 2 * R) * BT_X);
        float* dst = norm ? p.tmp : p.image;
        unsigned int* mx = norm ? p.maxbits + 1 : nullptr;
        if (norm) {
            e = cudaMemsetAsync(mx, 0, sizeof(unsigned int), s);
            if (e != cudaSuccess) return e;
        }
        dim3 grid((p.W + BT_X - 1) / BT_X, (p.H + BT_Y - 1) / BT_Y);
        if (!fused) {
            e = run_blur(grid, sm, s, FloatSamples{cur, nullptr}, p.H, p.W, k, dst, mx);
        } else if (p.raw_type == RAW_U8) {
            e = run_blur(grid, sm, s, CodeSamples<uint8_t>{(const uint8_t*)p.raw, p.background, clip, 0u, 0.0f, 0.0f},
                         p.H, p.W, k, dst, mx);
        } else if (p.raw_type == RAW_U16) {
            e = run_blur(grid, sm, s, CodeSamples<uint16_t>{(const uint16_t*)p.raw, p.background, clip, 0u, 0.0f, 0.0f},
                         p.H, p.W, k, dst, mx);
        } else {
            e = run_blur(grid, sm, s, FloatSamples{(const float*)p.raw, p.background}, p.H, p.W, k, dst, mx);
        }
        if (e != cudaSuccess) return e;
        nl += 1;
        cur = dst;
    }
    if (norm) {
        const int r = p.normalize_radius;
        if (r > kMaxNormRadius) return cudaErrorInvalidValue;
        if (!blur) {
            e = cudaMemsetAsync(p.maxbits + 1, 0, sizeof(unsigned int), s);
            if (e != cudaSuccess) return e;
            maxabs_kernel<<<grid_for(n), 256, 0, s>>>(cur, n, p.maxbits + 1);
            nl += 1;
        }
        const size_t sm = sizeof(long long) * (2 * (size_t)(NT_Y + 2 * r) * ((NT_X + 2 * r) | 1) + 2 * (size_t)(NT_Y + 2 * r) * NT_HW);
        dim3 grid((p.W + NT_X - 1) / NT_X, (p.H + NT_Y - 1) / NT_Y);
        if (r == 4) {  // the default radius: 46.3 KB of tile, under the 48 KB default
            normalize_kernel<4><<<grid, kNormThreads, sm, s>>>(cur, p.H, p.W, r, p.normalize_eps, p.maxbits + 1, p.image);
        } else {
            if (sm > 48 * 1024) {
                e = cudaFuncSetAttribute(normalize_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                if (e != cudaSuccess) return e;
            }
            normalize_kernel<0><<<grid, kNormThreads, sm, s>>>(cur, p.H, p.W, r, p.normalize_eps, p.maxbits + 1, p.image);
        }
        nl += 1;
        cur = p.image;
    }
    if (cur != p.image) {
        e = cudaMemcpyAsync(p.image, cur, sizeof(float) * n, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
    }
    if (launches) *launches += nl;
    return cudaGetLastError();
}

}  // namespace pivb200
