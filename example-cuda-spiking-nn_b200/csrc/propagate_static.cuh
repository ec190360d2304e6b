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

// The calling thread's current CUDA context (a driver handle), or null when none is current yet.
// Looked up through the runtime's driver entry point, so the library needs no link to libcuda.
inline cudaError_t current_context(void** ctx) {
    using CtxGetCurrent = int (*)(void**);
    static CtxGetCurrent fn = nullptr;
    static cudaError_t lookup = cudaSuccess;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        lookup = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
        if (lookup == cudaSuccess && (q != cudaDriverEntryPointSuccess || f == nullptr)) lookup = cudaErrorNotSupported;
        fn = reinterpret_cast<CtxGetCurrent>(f);
    });
    if (lookup != cudaSuccess) return lookup;
    *ctx = nullptr;
    return fn(ctx) == 0 ? cudaSuccess : cudaErrorDeviceUninitialized;
}

// Device address of g_static_scratch on device `dev`, which must be the current device.  The first
// call for a device looks the symbol up (and may load this library's device code) and caches the
// address together with the context it belongs to.  When the current context of the device changes
// (after cudaDeviceReset, or when a caller makes another context current) the address is looked up
// again, so a call never launches on an address of a context that no longer exists.
inline cudaError_t static_scratch(int dev, float** out) {
    static std::mutex mu;
    static float* addr[kMaxStaticDevices] = {};
    static void* owner[kMaxStaticDevices] = {};
    if (dev < 0 || dev >= kMaxStaticDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    void* ctx = nullptr;
    cudaError_t e = current_context(&ctx);
    if (e != cudaSuccess) return e;
    if (!addr[dev] || ctx == nullptr || ctx != owner[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);  // initialises the device's context if needed
        if (e != cudaSuccess) return e;
        e = current_context(&ctx);
        if (e != cudaSuccess) return e;
        addr[dev] = static_cast<float*>(p);
        owner[dev] = ctx;
    }
    *out = addr[dev];
    return cudaSuccess;
}

// Row chunks for the static scratch: the same count as the allocating path whenever
// splits x n_post fits, never more than fits.  With the same count the two paths add the same
// floats in the same order and give the same result bits.  On a 148-SM B200 choose_splits keeps
// splits x n_post below 4 * 148 * 256 + 256 * ceil(n_post / 256) for n_post < 151553 and equal to
// n_post (one split) above, so there every n_post up to kStaticScratchFloats gets the same chunks.
// On a GPU whose SM count makes splits x n_post exceed the array, fewer chunks are used: the sums
// are then added in another order and agree with the allocating path to float rounding only.
inline uint32_t static_splits(uint32_t n_pre, uint32_t n_post, int sm_count) {
    uint32_t splits = choose_splits(n_pre, n_post, sm_count);
    const size_t fit = kStaticScratchFloats / n_post;
    if (splits > fit) splits = static_cast<uint32_t>(fit);
    return splits;
}

}  // namespace prop
}  // namespace bsnn
