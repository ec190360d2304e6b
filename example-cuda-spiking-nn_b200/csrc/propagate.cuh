// propagate.cuh -- stand-alone connection propagation on caller-owned device buffers.
//
// The work of kernel_connection_propagate_launch (cpp_src/connections/kernel_connection_propagate.cu:64-111)
// for one ConnectionView: decay the presynaptic r and d traces (flushing values below 1e-30), add
// the normalisation value on a presynaptic spike, form x = d - r, then add W^T x into the
// postsynaptic conductance the connection drives (g_inhibitory for an inhibitory presynaptic
// group, g_excitatory otherwise).  The GEMV is split over `splits` row chunks: each chunk's column
// sums go to scratch[split][post], and a second kernel adds them in split order, so the result
// does not depend on scheduling.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bsnn.h"

namespace bsnn {
namespace prop {

constexpr unsigned kThreads = 256;

__global__ void traces_kernel(float r_decay, float d_decay, float norm, uint32_t n_pre, float* __restrict__ r,
                              float* __restrict__ d, float* __restrict__ x, const uint32_t* __restrict__ spikes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pre) return;
    // Each operation rounded on its own (no contraction), as the reference's separate kernels do.
    float dd = __fmul_rn(d[i], d_decay);  // kernel_connection_decay_d_traces (:22-33)
    if (dd < 1e-30f) dd = 0.0f;
    float rr = __fmul_rn(r[i], r_decay);  // kernel_connection_decay_r_traces (:8-20)
    if (rr < 1e-30f) rr = 0.0f;
    if (spikes[i] == 1u) {  // kernel_connection_update_conductances_with_spikes (:35-46)
        rr = __fadd_rn(rr, norm);
        dd = __fadd_rn(dd, norm);
    }
    r[i] = rr;
    d[i] = dd;
    x[i] = __fsub_rn(dd, rr);
}

// partial[s][q] = sum over rows p in chunk s of W[p * n_post + q] * x[p] (ascending p).
__global__ void gemv_partial_kernel(const float* __restrict__ w, const float* __restrict__ x, uint32_t n_pre,
                                    uint32_t n_post, uint32_t chunk, float* __restrict__ partial) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t s = blockIdx.y;
    if (q >= n_post) return;
    const uint32_t p0 = s * chunk;
    const uint32_t p1 = p0 + chunk < n_pre ? p0 + chunk : n_pre;
    float acc = 0.0f;
    uint32_t p = p0;
    for (; p + 4 <= p1; p += 4) {  // four independent loads in flight per iteration
        const float w0 = __ldg(w + static_cast<size_t>(p) * n_post + q);
        const float w1 = __ldg(w + static_cast<size_t>(p + 1) * n_post + q);
        const float w2 = __ldg(w + static_cast<size_t>(p + 2) * n_post + q);
        const float w3 = __ldg(w + static_cast<size_t>(p + 3) * n_post + q);
        acc = fmaf(w0, x[p], acc);
        acc = fmaf(w1, x[p + 1], acc);
        acc = fmaf(w2, x[p + 2], acc);
        acc = fmaf(w3, x[p + 3], acc);
    }
    for (; p < p1; ++p) acc = fmaf(__ldg(w + static_cast<size_t>(p) * n_post + q), x[p], acc);
    partial[static_cast<size_t>(s) * n_post + q] = acc;
}

// g[q] = (sum over splits of partial[s][q]) + g[q]  (cublasSgemv with alpha = beta = 1)
__global__ void gemv_reduce_kernel(const float* __restrict__ partial, uint32_t n_post, uint32_t splits,
                                   float* __restrict__ g) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_post) return;
    float dot = 0.0f;
    for (uint32_t s = 0; s < splits; ++s) dot += partial[static_cast<size_t>(s) * n_post + q];
    g[q] = dot + g[q];
}

// Row chunks of the split GEMV: enough blocks to cover the SMs a few times over.
inline uint32_t choose_splits(uint32_t n_pre, uint32_t n_post, int sm_count) {
    const uint32_t col_blocks = (n_post + kThreads - 1) / kThreads;
    uint32_t splits = (4u * static_cast<uint32_t>(sm_count > 0 ? sm_count : 1) + col_blocks - 1) / col_blocks;
    if (splits > n_pre) splits = n_pre;
    if (splits < 1) splits = 1;
    return splits;
}

// Validates a view; returns a message or nullptr.
inline const char* check_view(const bsnn_connection_view* v) {
    if (!v) return "null view";
    if (v->pre_group_num_neurons == 0 || v->post_group_num_neurons == 0) return "empty connection";
    if (!v->weight_matrix || !v->postsynaptic_r_traces || !v->postsynaptic_d_traces ||
        !v->summed_postsynaptic_conductances || !v->spikes)
        return "null device pointer in view";
    float* g = v->pre_group_is_inhibtory ? v->post_group_g_inhibitory : v->post_group_g_excitatory;
    if (!g) return "null postsynaptic conductance pointer";
    return nullptr;
}

// Enqueues the three kernels on `stream` with `splits` row chunks and the given scratch
// (splits * n_post floats).
inline cudaError_t enqueue(const bsnn_connection_view* v, uint32_t splits, float* scratch, cudaStream_t stream) {
    const uint32_t n_pre = v->pre_group_num_neurons, n_post = v->post_group_num_neurons;
    float* g = v->pre_group_is_inhibtory ? v->post_group_g_inhibitory : v->post_group_g_excitatory;
    traces_kernel<<<(n_pre + kThreads - 1) / kThreads, kThreads, 0, stream>>>(
        v->postsynaptic_r_trace_decay, v->postsynaptic_d_trace_decay, v->postsynaptic_kernel_normalization_value,
        n_pre, v->postsynaptic_r_traces, v->postsynaptic_d_traces, v->summed_postsynaptic_conductances, v->spikes);
    const uint32_t chunk = (n_pre + splits - 1) / splits;
    const uint32_t used = (n_pre + chunk - 1) / chunk;
    gemv_partial_kernel<<<dim3((n_post + kThreads - 1) / kThreads, used), kThreads, 0, stream>>>(
        v->weight_matrix, v->summed_postsynaptic_conductances, n_pre, n_post, chunk, scratch);
    gemv_reduce_kernel<<<(n_post + kThreads - 1) / kThreads, kThreads, 0, stream>>>(scratch, n_post, used, g);
    return cudaGetLastError();
}

}  // namespace prop
}  // namespace bsnn
