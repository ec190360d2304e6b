// adjoint_kernel.cuh -- the differentiation form: a surrogate-gradient adjoint (backpropagation
// through time) of the two-group network with frozen weights, for the gradient of a loss on the
// excitatory population rate (and, optionally, on the mean excitatory voltage) with respect to the
// E->E weights and g_leak.
//
// The forward model is the reference's step (background Poisson shot noise, conductance-EIF Euler
// step with refractoriness, difference-of-exponentials traces, the four propagations, stimulus)
// without plasticity, as simple per-step kernels that record what the backward pass needs:
//   u_t  the pre-threshold potential v_t + dt/C * F(v_t, g_e, g_i) (non-refractory steps),
//   s_t  the spike (u_t >= v_th), r_t whether the neuron was refractory, v_t, g_e(t), g_i(t),
//   x_t  the connection trace d - r each presynaptic neuron fed the step-t propagation with.
// State is checkpointed every `checkpoint` steps; the backward pass replays each segment from its
// checkpoint (the noise is a counter-based function of (seed, neuron, step), so the replay is
// exact), then walks the segment backwards:
//   spikes: ds/du = psi(u - v_th), psi(z) = 1 / (1 + |z| / beta)^2 (fast sigmoid, width beta);
//   v_{t+1} = s v_th + (1 - s) u (the reset is not differentiated); refractory steps block;
//   u = v + dt/C (-gL (v - v_rest) + gL dT exp((v - v_T)/dT) - g_e (v - E_e) - g_i (v - E_i) + I);
//   traces d' = a_d d + n s, r' = a_r r + n s, x = d - r;
//   g_e(t) = b_e(t) + sum_pre W_E[pre, post] x_t[pre] (E presynaptic), g_i likewise with W_I.
// The adjoints of g_e / g_i are pulled back through the weights by a GEMV per step
// (lambda_x = W lambda_g), and dL/dW_EE accumulates x_t lambda_ge(t)^T per segment by a GEMM over
// the segment's steps.  All arithmetic is FP32.
#pragma once

#include "step_kernel.cuh"

namespace bsnn {

struct AdjGroupP {
    float timestep, g_leak, cap, delta_t, v_eff, e_exc, e_inh, v_th, v_reset, v_rest;
    float exp_neg_mean_e, exp_neg_mean_i, bg_er_decay, bg_ed_decay, bg_ir_decay, bg_id_decay, bg_scale_e, bg_scale_i;
    uint32_t refractory_steps, has_bg_e, has_bg_i;
};

struct ADev {
    uint32_t E, I, N, seed, noise_on;
    AdjGroupP g[2];
    float r_decay[2], d_decay[2], norm[2];  // E-presynaptic and I-presynaptic connection traces
    const float* WE;  // [E][N] row-major: E->E | E->I
    const float* WI;  // [I][N]: I->E | I->I
    // state
    float *v, *ge, *gi, *istim, *er, *ed, *ir, *id, *tr, *td;
    uint32_t* refrac;
    // stimulus CSR over steps, events sorted by neuron
    uint32_t stim_len;
    const uint32_t* stim_off;
    const uint32_t* ev_neuron;
    const float* ev_delta;
};

// Propagation partial sums: part[(side * chunks + c) * N + post] holds the chunk-c share of
// sum_pre W_side[pre, post] x[pre] (side 0: E presynaptic rows, side 1: I rows).  The neuron
// kernel adds the chunks in order, so g is the same on every pass over a step.
constexpr uint32_t kAdjChunks = 16;
constexpr uint32_t kAdjBlock = 256;

__device__ __forceinline__ float adj_chunk_sum(const float* part, uint32_t side, uint32_t chunks, uint32_t N,
                                               uint32_t n) {
    float s = 0.0f;
    for (uint32_t c = 0; c < chunks; ++c) s += part[(static_cast<size_t>(side) * chunks + c) * N + n];
    return s;
}

// One forward step t for every neuron: g_e / g_i of the step are the background of the previous
// step plus the propagation partials; writes x_{t+1} (the trace value the next propagation uses)
// and, when the tape pointers are set, the step's tape row.  Optional: the step's E spike count
// and this block's sum of the E voltages after the step.
__global__ void __launch_bounds__(kAdjBlock) bsnn_adj_neuron_fwd(ADev A, uint32_t t, const float* __restrict__ part,
                                                                 float* tape_v, float* tape_u, float* tape_ge,
                                                                 float* tape_gi, uint8_t* tape_s, uint8_t* tape_ref,
                                                                 float* x_next, uint32_t* e_spike_count,
                                                                 double* vsum_out) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    double vpart = 0.0;
    if (n < A.N) {
        const uint32_t side = n < A.E ? 0u : 1u;
        const AdjGroupP& G = A.g[side];
        const float ge_used = A.ge[n] + adj_chunk_sum(part, 0, kAdjChunks, A.N, n);
        const float gi_used = A.gi[n] + adj_chunk_sum(part, 1, kAdjChunks, A.N, n);
        float er = flush_tiny(A.er[n] * G.bg_er_decay);
        float ir = flush_tiny(A.ir[n] * G.bg_ir_decay);
        float ed = flush_tiny(A.ed[n] * G.bg_ed_decay);
        float id = flush_tiny(A.id[n] * G.bg_id_decay);
        uint32_t ne = 0, ni = 0;
        if (A.noise_on) {
            if (G.has_bg_e) ne = poisson_knuth(G.exp_neg_mean_e, A.seed, n, t, 0u);
            if (G.has_bg_i) ni = poisson_knuth(G.exp_neg_mean_i, A.seed, n, t, 1u);
        }
        if (ne > 0u) {
            const float inc = static_cast<float>(ne);
            er += inc;
            ed += inc;
        }
        const float bg_ge = (ed - er) * G.bg_scale_e;
        if (ni > 0u) {
            const float inc = static_cast<float>(ni);
            ir += inc;
            id += inc;
        }
        const float bg_gi = (id - ir) * G.bg_scale_i;
        const float v_in = A.v[n];
        float v = v_in, istim = A.istim[n];
        uint32_t refrac = A.refrac[n], spike = 0;
        float u = v;
        const bool was_refractory = refrac > 0;
        if (refrac > 0) {
            --refrac;
            v = G.v_reset;
        } else {
            const float linear_leak_term = -1.0f * G.g_leak * (v - G.v_rest);
            const float exponential_depolarization_term = G.g_leak * G.delta_t * expf((v - G.v_eff) / G.delta_t);
            const float excitatory_synaptic_term = -1.0f * ge_used * (v - G.e_exc);
            const float inhibitory_synaptic_term = -1.0f * gi_used * (v - G.e_inh);
            const float dv = (G.timestep / G.cap) * (linear_leak_term + exponential_depolarization_term +
                                                     excitatory_synaptic_term + inhibitory_synaptic_term + istim);
            u = v + dv;
            if (u >= G.v_th) {
                refrac = G.refractory_steps;
                spike = 1;
                v = G.v_th;
            } else {
                v = u;
            }
        }
        if (tape_v) {
            tape_v[n] = v_in;
            tape_ge[n] = ge_used;
            tape_gi[n] = gi_used;
            tape_ref[n] = was_refractory ? 1 : 0;
            tape_u[n] = u;
            tape_s[n] = static_cast<uint8_t>(spike);
        }
        if (spike && side == 0 && e_spike_count) atomicAdd(e_spike_count, 1u);
        A.er[n] = er;
        A.ed[n] = ed;
        A.ir[n] = ir;
        A.id[n] = id;
        A.v[n] = v;
        A.refrac[n] = refrac;
        A.ge[n] = bg_ge;  // the next step adds the propagation of x_{t+1}
        A.gi[n] = bg_gi;
        if (t < A.stim_len) {
            for (uint32_t k = A.stim_off[t]; k < A.stim_off[t + 1]; ++k)
                if (A.ev_neuron[k] == n) istim = istim + A.ev_delta[k];
            A.istim[n] = istim;
        }
        float d = flush_tiny(A.td[n] * A.d_decay[side]);
        float r = flush_tiny(A.tr[n] * A.r_decay[side]);
        if (spike) {
            r += A.norm[side];
            d += A.norm[side];
        }
        A.tr[n] = r;
        A.td[n] = d;
        x_next[n] = d - r;
        if (side == 0) vpart = static_cast<double>(v);
    }
    if (vsum_out) {  // block sum of the E voltages, in a fixed order
        __shared__ double red[kAdjBlock];
        red[threadIdx.x] = vpart;
        __syncthreads();
        for (uint32_t o = kAdjBlock / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) vsum_out[blockIdx.x] = red[0];
    }
}

// The propagation of x for both presynaptic sides: blockIdx.y = side * chunks + chunk, each block
// a contiguous range of presynaptic rows for kAdjBlock postsynaptic columns.  The block first
// lists the range's rows with x != 0 in shared memory (in row order), then accumulates over them
// with kAdjRowsInFlight weight loads in flight per thread.  A zero-x row would add exactly 0, so
// the sum is the dense one, in row order, on every pass.
constexpr uint32_t kAdjRowsInFlight = 8;
__global__ void __launch_bounds__(kAdjBlock) bsnn_adj_propagate(const float* __restrict__ WE,
                                                                const float* __restrict__ WI, uint32_t E, uint32_t I,
                                                                uint32_t N, uint32_t ld, const float* __restrict__ x,
                                                                float* __restrict__ part) {
    __shared__ uint32_t srow[kAdjBlock];
    __shared__ float sx[kAdjBlock];
    __shared__ uint32_t wcount[kAdjBlock / 32];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t post = blockIdx.x * blockDim.x + tid;
    const uint32_t side = blockIdx.y / kAdjChunks, c = blockIdx.y % kAdjChunks;
    const uint32_t rows = side ? I : E;
    const float* W = side ? WI : WE;
    const float* xs = x + (side ? E : 0u);
    const uint32_t per = (rows + kAdjChunks - 1) / kAdjChunks;
    const uint32_t r0 = c * per < rows ? c * per : rows, r1 = r0 + per < rows ? r0 + per : rows;
    const bool col = post < N;
    const float* wcol = W + (col ? post : 0u);
    float acc = 0.0f;
    for (uint32_t base = r0; base < r1; base += kAdjBlock) {
        const uint32_t r = base + tid;
        const float xv = r < r1 ? xs[r] : 0.0f;
        const bool live = xv != 0.0f;
        const uint32_t bal = __ballot_sync(kFull, live);
        if (lane == 0) wcount[warp] = __popc(bal);
        __syncthreads();
        uint32_t off = __popc(bal & ((1u << lane) - 1u)), total = 0;
#pragma unroll
        for (uint32_t w = 0; w < kAdjBlock / 32; ++w) {
            off += w < warp ? wcount[w] : 0u;
            total += wcount[w];
        }
        if (live) {
            srow[off] = r;
            sx[off] = xv;
        }
        __syncthreads();
        if (col) {
            uint32_t k = 0;
            for (; k + kAdjRowsInFlight <= total; k += kAdjRowsInFlight) {
                float w[kAdjRowsInFlight];
#pragma unroll
                for (uint32_t q = 0; q < kAdjRowsInFlight; ++q) w[q] = __ldg(wcol + static_cast<size_t>(srow[k + q]) * ld);
#pragma unroll
                for (uint32_t q = 0; q < kAdjRowsInFlight; ++q) acc = fmaf(w[q], sx[k + q], acc);
            }
            for (; k < total; ++k) acc = fmaf(__ldg(wcol + static_cast<size_t>(srow[k]) * ld), sx[k], acc);
        }
        __syncthreads();
    }
    if (col) part[static_cast<size_t>(blockIdx.y) * N + post] = acc;
}

// Checkpoint slot layout: 12 arrays of N: v, g_e and g_i as the next step uses them, i_stimulus,
// the four background traces, the connection r and d traces, the refractory counters (as bits)
// and x (the trace value the next step's propagation used).
constexpr uint32_t kAdjCkptArrays = 12;

__global__ void bsnn_adj_save(ADev A, const float* __restrict__ part, const float* __restrict__ x, float* slot) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.N) return;
    const size_t N = A.N;
    slot[n] = A.v[n];
    slot[N + n] = A.ge[n] + adj_chunk_sum(part, 0, kAdjChunks, A.N, n);
    slot[2 * N + n] = A.gi[n] + adj_chunk_sum(part, 1, kAdjChunks, A.N, n);
    slot[3 * N + n] = A.istim[n];
    slot[4 * N + n] = A.er[n];
    slot[5 * N + n] = A.ed[n];
    slot[6 * N + n] = A.ir[n];
    slot[7 * N + n] = A.id[n];
    slot[8 * N + n] = A.tr[n];
    slot[9 * N + n] = A.td[n];
    slot[10 * N + n] = __uint_as_float(A.refrac[n]);
    slot[11 * N + n] = x[n];
}

// Restores a checkpoint (slot non-null) or the initial state (v = v_rest, all else 0); the
// partials are zeroed, so the next step's g is exactly the saved one.
__global__ void bsnn_adj_restore(ADev A, float* __restrict__ part, float* __restrict__ x, const float* slot) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.N) return;
    const size_t N = A.N;
    for (uint32_t c = 0; c < 2 * kAdjChunks; ++c) part[c * N + n] = 0.0f;
    if (slot) {
        A.v[n] = slot[n];
        A.ge[n] = slot[N + n];
        A.gi[n] = slot[2 * N + n];
        A.istim[n] = slot[3 * N + n];
        A.er[n] = slot[4 * N + n];
        A.ed[n] = slot[5 * N + n];
        A.ir[n] = slot[6 * N + n];
        A.id[n] = slot[7 * N + n];
        A.tr[n] = slot[8 * N + n];
        A.td[n] = slot[9 * N + n];
        A.refrac[n] = __float_as_uint(slot[10 * N + n]);
        x[n] = slot[11 * N + n];
    } else {
        A.v[n] = A.g[n < A.E ? 0 : 1].v_rest;
        A.ge[n] = A.gi[n] = A.istim[n] = 0.0f;
        A.er[n] = A.ed[n] = A.ir[n] = A.id[n] = A.tr[n] = A.td[n] = 0.0f;
        A.refrac[n] = 0u;
        x[n] = 0.0f;
    }
}

__device__ __forceinline__ float surrogate(float z, float beta) {
    if (!(beta > 0.0f)) return 0.0f;
    const float a = 1.0f + fabsf(z) / beta;
    return 1.0f / (a * a);
}

// One backward step t for every neuron.  In: lambda_v(t+1) (lam_v), the trace adjoints carried
// from step t+1 (lam_d, lam_r: dL/dd_{t+1}, dL/dr_{t+1} before adding lambda_x(t+1)), lambda_x(t+1)
// (lam_x, the pull-back of step t+1's g adjoints), *c_s_t (dL/ds_t from the rate loss, E neurons)
// and *c_v_t (dL/dv_{t+1} from the voltage loss, E neurons).  Out: lambda_v(t), the carried trace
// adjoints for step t, lambda_ge(t) / lambda_gi(t), and this block's share of dL/dg_leak.
__global__ void bsnn_adj_neuron_bwd(ADev A, const float* tape_v, const float* tape_u, const float* tape_ge,
                                    const float* tape_gi, const uint8_t* tape_s, const uint8_t* tape_ref,
                                    float* lam_v, float* lam_d, float* lam_r, const float* lam_x,
                                    const float* __restrict__ c_s_t, const float* __restrict__ c_v_t, float beta,
                                    float* lam_ge, float* lam_gi, double* gleak_acc) {
    const float c_s = *c_s_t, c_v = *c_v_t;
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    double gl = 0.0;
    if (n < A.N) {
        const uint32_t side = n < A.E ? 0u : 1u;
        const AdjGroupP& G = A.g[side];
        // traces produced at step t (x_{t+1} = d_{t+1} - r_{t+1}); lam_x is dL/dx_{t+1}
        const float Ld = lam_d[n] + lam_x[n], Lr = lam_r[n] - lam_x[n];
        const float s = tape_s[n] ? 1.0f : 0.0f;
        float dLds = A.norm[side] * (Ld + Lr);
        if (side == 0) dLds += c_s;
        float Lv_next = lam_v[n] + (side == 0 ? c_v : 0.0f);
        float lv = 0.0f, lge = 0.0f, lgi = 0.0f;
        if (!tape_ref[n]) {
            const float v = tape_v[n], u = tape_u[n], ge = tape_ge[n], gi = tape_gi[n];
            const float lu = Lv_next * (1.0f - s) + dLds * surrogate(u - G.v_th, beta);
            const float k = G.timestep / G.cap;
            const float ex = expf((v - G.v_eff) / G.delta_t);
            lv = lu * (1.0f + k * (-G.g_leak + G.g_leak * ex - ge - gi));
            lge = lu * k * (G.e_exc - v);
            lgi = lu * k * (G.e_inh - v);
            gl = static_cast<double>(lu) * static_cast<double>(k * (-(v - G.v_rest) + G.delta_t * ex));
        }
        lam_v[n] = lv;
        lam_d[n] = A.d_decay[side] * Ld;  // dL/dd_t
        lam_r[n] = A.r_decay[side] * Lr;
        lam_ge[n] = lge;
        lam_gi[n] = lgi;
    }
    // block reduction of the g_leak share, in a fixed order
    __shared__ double red[kAdjBlock];
    red[threadIdx.x] = gl;
    __syncthreads();
    for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) gleak_acc[blockIdx.x] += red[0];
}

// lambda_x[pre] = sum_post W[pre, post] lambda_g[post] for both sides (one warp per presynaptic
// row: rows < E use W_E and lambda_ge, the others W_I and lambda_gi).  Rows are ld floats (ld a
// multiple of 4, zero beyond N), read as float4; lambda_g is zero beyond N as well.
__global__ void bsnn_adj_pullback(const float* __restrict__ WE, const float* __restrict__ WI, uint32_t E, uint32_t N,
                                  uint32_t ld, const float* __restrict__ lam_ge, const float* __restrict__ lam_gi,
                                  float* __restrict__ lam_x) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (warp >= N) return;
    const float4* row = reinterpret_cast<const float4*>(warp < E ? WE + static_cast<size_t>(warp) * ld
                                                                  : WI + static_cast<size_t>(warp - E) * ld);
    const float4* lam = reinterpret_cast<const float4*>(warp < E ? lam_ge : lam_gi);
    const uint32_t n4 = ld >> 2;
    float acc = 0.0f;
#pragma unroll 4
    for (uint32_t q = lane; q < n4; q += 32u) {
        const float4 w = __ldg(row + q), l = __ldg(lam + q);
        acc = fmaf(w.x, l.x, acc);
        acc = fmaf(w.y, l.y, acc);
        acc = fmaf(w.z, l.z, acc);
        acc = fmaf(w.w, l.w, acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane == 0) lam_x[warp] = acc;
}

// dW[pre, post] += sum_t X[t, pre] L[t, post] over one segment's steps (X: x_t of the E
// presynaptic neurons, rows of ldx floats; L: lambda_ge(t) of the E postsynaptic neurons, rows of
// ldl floats).
// 32 x 32 output tiles, the steps staged through shared memory 32 at a time.
__global__ void bsnn_adj_outer(const float* __restrict__ X, uint32_t ldx, const float* __restrict__ L, uint32_t ldl,
                               uint32_t steps, uint32_t E, float* __restrict__ dW) {
    __shared__ float xs[32][33], ls[32][33];
    const uint32_t pre0 = blockIdx.y * 32u, post0 = blockIdx.x * 32u;
    const uint32_t tx = threadIdx.x & 31u, ty = threadIdx.x >> 5;  // 32 x 8 threads, 4 outputs each
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (uint32_t t0 = 0; t0 < steps; t0 += 32u) {
        for (uint32_t k = ty; k < 32u; k += 8u) {
            const uint32_t t = t0 + k;
            xs[k][tx] = t < steps && pre0 + tx < E ? X[static_cast<size_t>(t) * ldx + pre0 + tx] : 0.0f;
            ls[k][tx] = t < steps && post0 + tx < E ? L[static_cast<size_t>(t) * ldl + post0 + tx] : 0.0f;
        }
        __syncthreads();
#pragma unroll 8
        for (uint32_t k = 0; k < 32u; ++k) {
            const float l = ls[k][tx];
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) acc[q] = fmaf(xs[k][ty + 8u * q], l, acc[q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (uint32_t q = 0; q < 4; ++q) {
        const uint32_t pre = pre0 + ty + 8u * q, post = post0 + tx;
        if (pre < E && post < E) dW[static_cast<size_t>(pre) * E + post] += acc[q];
    }
}

}  // namespace bsnn
