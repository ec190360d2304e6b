// propagate_static.cuh -- fixed device scratch for the connection propagation that allocates nothing.
//
// The split GEMV of propagate.cuh needs splits x N_post floats between its two kernels.  This file
// provides that scratch as one module-scope device array per device instead of a per-call
// allocation.  Every float the reduction reads is written by the partial kernel of the same call,
// so the array never has to start at zero.  All calls on one device share it: two calls that
// overlap in time (different streams or host threads) race on it.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>

namespace bsnn {
namespace prop {

constexpr size_t kStaticScratchFloats = size_t(1) << 20;  // 4 MiB per device
constexpr int kMaxStaticDevices = 64;

static __device__ __align__(256) float g_static_scratch[kStaticScratchFloats];

// Device address of g_static_scratch on device `dev`, which must be the current device.  The first
// call for a device looks the symbol up (and may load this library's device code); later calls
// return the cached address.
inline cudaError_t static_scratch(int dev, float** out) {
    static std::mutex mu;
    static float* addr[kMaxStaticDevices] = {};
    if (dev < 0 || dev >= kMaxStaticDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        addr[dev] = static_cast<float*>(p);
    }
    *out = addr[dev];
    return cudaSuccess;
}

// Row chunks for the static scratch: the same count as the allocating path whenever
// splits x n_post fits, never more than fits.  On a 148-SM B200 choose_splits keeps
// splits x n_post below 4 * 148 * 256 + 256 * ceil(n_post / 256) for n_post < 151553 and equal to
// n_post (one split) above, so every n_post up to kStaticScratchFloats gets the same chunks, and
// the same result bits, as the allocating path.
inline uint32_t static_splits(uint32_t n_pre, uint32_t n_post, int sm_count) {
    uint32_t splits = choose_splits(n_pre, n_post, sm_count);
    const size_t fit = kStaticScratchFloats / n_post;
    if (splits > fit) splits = static_cast<uint32_t>(fit);
    return splits;
}

}  // namespace prop
}  // namespace bsnn
