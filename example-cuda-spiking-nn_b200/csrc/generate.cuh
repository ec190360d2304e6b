// generate.cuh -- network generation on the GPU: distance-dependent weights (a flagged
// alternative to the reference's generator, cpp_src/generation/generate_weights.cpp:10-103).
//
// The rule is the reference's: a pair (pre i, post q) is a candidate unless it is on the diagonal
// (when diagonals are excluded) or farther apart than max_distance on the periodic 2-D layout;
// a candidate exists with probability p = probability_multiplier (times exp(-d^2 / spread_scale)
// when the probability is normal), and weighs max_weight_value (times the same Gaussian when the
// value drops off normally).  The distance and the candidate test are computed exactly as on the
// host (IEEE fabs, min, square root), so the candidate sets are identical.  The random draws are
// not: the reference draws one mt19937 number per candidate in row-major order, a sequential
// stream; here every pair draws from Philox4x32-10 keyed by (seed, pre, post), so the matrix is
// the same in distribution, not bit for bit.  Uniform value mode (w ~ U[0, max_weight_value) on
// each existing synapse) takes the second uniform of the same draw.
#pragma once

#include "step_kernel.cuh"

namespace bsnn {

struct GenParams {
    float max_weight_value, max_distance, spread_scale, probability_multiplier, lx, ly;
    uint32_t value_dropoff, normal_probability, no_diagonal, uniform_values;
    uint32_t seed_lo, seed_hi;
};

__device__ __forceinline__ float gen_uniform(uint32_t r) {  // [0, 1) on the 24-bit grid
    return __uint2float_rn(r >> 8) * 5.9604644775390625e-8f;
}

// One thread per (pre, post) pair, posts fastest; w row-major [n_pre][n_post].
__global__ void bsnn_generate_weights_kernel(const float* __restrict__ pre_xy, uint32_t n_pre,
                                             const float* __restrict__ post_xy, uint32_t n_post, GenParams P,
                                             float* __restrict__ w) {
    const uint64_t idx = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<uint64_t>(n_pre) * n_post) return;
    const uint32_t i = static_cast<uint32_t>(idx / n_post), q = static_cast<uint32_t>(idx % n_post);
    float dx = fabsf(pre_xy[2 * i] - post_xy[2 * q]);
    float dy = fabsf(pre_xy[2 * i + 1] - post_xy[2 * q + 1]);
    dx = fminf(dx, P.lx - dx);
    dy = fminf(dy, P.ly - dy);
    const float d = sqrtf(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));  // no contraction: the host's rounding
    float v = 0.0f;
    const bool candidate = !(P.no_diagonal && i == q) && !(fabsf(d) > P.max_distance);
    if (candidate) {
        uint32_t c0 = q, c1 = i, c2 = P.seed_hi, c3 = 0x57E16u;
        philox4x32_10(c0, c1, c2, c3, P.seed_lo, 0x5EEDu);
        float prob = P.probability_multiplier;
        const float gauss = expf(-1.0f * __fmul_rn(d, d) / P.spread_scale);
        if (P.normal_probability) prob *= gauss;
        if (gen_uniform(c0) < prob) {
            v = P.uniform_values ? gen_uniform(c1) * P.max_weight_value : P.max_weight_value;
            if (P.value_dropoff) v *= gauss;
        }
    }
    w[idx] = v;
}

}  // namespace bsnn
