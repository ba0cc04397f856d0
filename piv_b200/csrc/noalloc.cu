// Field validation without any device allocation.
//
// Who needs this: callers that cannot call cudaMalloc once they are running. Two kinds are
// common. An acquisition or control loop that must hand back each field on a deadline cannot
// afford an allocation call: cudaFree waits for the whole device, and a first cudaMalloc of a
// size can take milliseconds. A process whose device memory is already handed out by another
// allocator (a framework's caching pool that reserved most of the GPU) can see a plain
// cudaMalloc fail even though the pool has room. Such callers own every buffer they pass in and
// need the library to allocate nothing.
//
// The validation stages need two per-cell flag snapshots (validate.rs:81 and :103 take them).
// Here they live in one file-scope device array of fixed size, kNoAllocMaxCells cells per
// snapshot (2 x 2,097,152 bytes = 4 MiB). Every GPU that loads this library holds that array
// until the process exits. Fields with more cells are rejected.
//
// Host code cannot use the array's name as a device address (it names a host-side stand-in),
// so the address is taken with cudaGetSymbolAddress once per device, with that device current,
// on the first call of the entry point on that device. Make that first call before any stream
// capture begins. The address is kept for the life of the process, so the entry point must not
// be used on a device after cudaDeviceReset (or any reset of its primary context). Every call
// shares the same array, and the kernels overwrite every snapshot byte they later read, so
// nothing needs clearing between calls; two calls whose work overlaps on the GPU (different
// streams, or different host threads on one device) race on it.
//
// Outputs must not overlap inputs: the median test reads neighbours' dx/dy while other threads
// write theirs, so in-place validation would race. Overlapping buffers are rejected.
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/piv_b200.h"
#include "kernels.h"

using namespace pivb200;

namespace {

constexpr long long kNoAllocMaxCells = 1ll << 21;

static __device__ __align__(256) uint8_t g_validate_scratch[2 * kNoAllocMaxCells];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint8_t* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (taken once per device).
cudaError_t scratch_for_current_device(uint8_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_validate_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<uint8_t*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

int reject(int code, const std::string& msg) {
    set_last_error(msg.c_str());
    return code;
}

// Whether the byte ranges [a, a + na) and [b, b + nb) share a byte.
bool overlap(const void* a, size_t na, const void* b, size_t nb) {
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x < y + nb && y < x + na;
}

}  // namespace

extern "C" {

int32_t piv_validate_field_noalloc(int64_t ny, int64_t nx, const float* dx, const float* dy, const float* peak_ratio,
                                   const uint8_t* flags, float max_displacement, float ppr_threshold,
                                   float median_threshold, float median_eps, int32_t replace, float* out_dx,
                                   float* out_dy, uint8_t* out_flags, void* stream) {
    if (!dx || !dy || !peak_ratio || !flags || !out_dx || !out_dy || !out_flags)
        return reject(PIV_ERR_ARGUMENT, "piv_validate_field_noalloc: null pointer");
    if (ny <= 0 || nx <= 0) return reject(PIV_ERR_ARGUMENT, "piv_validate_field_noalloc: empty field");
    // nx > max / ny rather than ny * nx > max: the product of two huge sizes would overflow.
    if (nx > kNoAllocMaxCells / ny) {
        char buf[200];
        snprintf(buf, sizeof(buf),
                 "piv_validate_field_noalloc: a %lld x %lld field exceeds the fixed scratch of %lld cells",
                 (long long)ny, (long long)nx, kNoAllocMaxCells);
        return reject(PIV_ERR_UNSUPPORTED, buf);
    }
    const size_t n = (size_t)(ny * nx), nf = n * sizeof(float);
    const void* ins[4] = {dx, dy, peak_ratio, flags};
    const size_t in_bytes[4] = {nf, nf, nf, n};
    const void* outs[3] = {out_dx, out_dy, out_flags};
    const size_t out_bytes[3] = {nf, nf, n};
    for (int o = 0; o < 3; ++o) {
        for (int i = 0; i < 4; ++i)
            if (overlap(outs[o], out_bytes[o], ins[i], in_bytes[i]))
                return reject(PIV_ERR_ARGUMENT, "piv_validate_field_noalloc: an output buffer overlaps an input "
                                                "(in-place validation would race)");
        for (int q = o + 1; q < 3; ++q)
            if (overlap(outs[o], out_bytes[o], outs[q], out_bytes[q]))
                return reject(PIV_ERR_ARGUMENT, "piv_validate_field_noalloc: output buffers overlap");
    }
    uint8_t* scratch = nullptr;
    cudaError_t e = scratch_for_current_device(&scratch);
    if (e != cudaSuccess)
        return reject(PIV_ERR_CUDA, std::string("piv_validate_field_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    ValidateParams vp{(int)nx, (int)ny, dx, dy, peak_ratio, flags, scratch, scratch + kNoAllocMaxCells,
                      out_dx, out_dy, out_flags, max_displacement, ppr_threshold, median_threshold, median_eps,
                      replace};
    e = launch_validate(vp, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return reject(PIV_ERR_CUDA, std::string("piv_validate_field_noalloc: ") + cudaGetErrorString(e));
    return PIV_OK;
}

}  // extern "C"
