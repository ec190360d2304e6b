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

#include "batch_kernel.cuh"  // tensor-memory wrappers
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

// Programmatic dependent launch (the forward pass's per-step kernels are launched with it): let the
// next kernel in the stream launch now, then wait until the previous one has completed and its
// writes are visible, before reading anything.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ float adj_chunk_sum(const float* part, uint32_t side, uint32_t chunks, uint32_t N,
                                               uint32_t n) {
    float s = 0.0f;
    for (uint32_t c = 0; c < chunks; ++c) s += part[(static_cast<size_t>(side) * chunks + c) * N + n];
    return s;
}

// One forward step t for every neuron: g_e / g_i of the step are the background of the previous
// step plus the propagation partials; writes x_{t+1} (the trace value the next propagation uses)
// and, when the tape pointers are set, the step's tape row.  Optional: the step's E spike count
// and this block's sum of the E voltages after the step.  [ev_lo, ev_hi): the step's stimulus
// events (from the host's copy of the stimulus offsets, so a step without events reads nothing).
__global__ void __launch_bounds__(kAdjBlock) bsnn_adj_neuron_fwd(ADev A, uint32_t t, uint32_t ev_lo, uint32_t ev_hi,
                                                                 const float* __restrict__ part,
                                                                 float* tape_v, float* tape_u, float* tape_ge,
                                                                 float* tape_gi, uint8_t* tape_s, uint8_t* tape_ref,
                                                                 float* x_next, uint32_t* e_spike_count,
                                                                 double* vsum_out) {
    pdl_enter();
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
            poisson_knuth_pair(G.exp_neg_mean_e, G.has_bg_e, G.exp_neg_mean_i, G.has_bg_i, A.seed, n, t, ne, ni);
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
        if (ev_lo < ev_hi) {
            for (uint32_t k = ev_lo; k < ev_hi; ++k)
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
    pdl_enter();
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

// One backward step t of neuron n.  In: lambda_v(t+1) (lv), the trace adjoints carried from step
// t+1 (ld_, lr_: dL/dd_{t+1}, dL/dr_{t+1} before adding lambda_x(t+1)), lambda_x(t+1) (lx, the
// pull-back of step t+1's g adjoints), c_s (dL/ds_t from the rate loss, E neurons) and c_v
// (dL/dv_{t+1} from the voltage loss, E neurons), and the step's tape row.  Out: lambda_v(t), the
// carried trace adjoints for step t, lambda_ge(t) / lambda_gi(t), and the neuron's share of
// dL/dg_leak.
__device__ __forceinline__ double adj_neuron_bwd_one(const ADev& A, uint32_t n, float tv, float tu, float tge, float tgi,
                                                     uint8_t ts, uint8_t tref, float& lv_io, float& ld_io, float& lr_io,
                                                     float lx, float c_s, float c_v, float beta, float& lge_out,
                                                     float& lgi_out) {
    const uint32_t side = n < A.E ? 0u : 1u;
    const AdjGroupP& G = A.g[side];
    // traces produced at step t (x_{t+1} = d_{t+1} - r_{t+1}); lx is dL/dx_{t+1}
    const float Ld = ld_io + lx, Lr = lr_io - lx;
    const float s = ts ? 1.0f : 0.0f;
    float dLds = A.norm[side] * (Ld + Lr);
    if (side == 0) dLds += c_s;
    const float Lv_next = lv_io + (side == 0 ? c_v : 0.0f);
    float lv = 0.0f, lge = 0.0f, lgi = 0.0f;
    double gl = 0.0;
    if (!tref) {
        const float v = tv, u = tu, ge = tge, gi = tgi;
        const float lu = Lv_next * (1.0f - s) + dLds * surrogate(u - G.v_th, beta);
        const float k = G.timestep / G.cap;
        const float ex = expf((v - G.v_eff) / G.delta_t);
        lv = lu * (1.0f + k * (-G.g_leak + G.g_leak * ex - ge - gi));
        lge = lu * k * (G.e_exc - v);
        lgi = lu * k * (G.e_inh - v);
        gl = static_cast<double>(lu) * static_cast<double>(k * (-(v - G.v_rest) + G.delta_t * ex));
    }
    lv_io = lv;
    ld_io = A.d_decay[side] * Ld;  // dL/dd_t
    lr_io = A.r_decay[side] * Lr;
    lge_out = lge;
    lgi_out = lgi;
    return gl;
}

// ---- the backward pass of a segment as one persistent kernel ------------------------------------
// The segment's steps walked backwards in one cooperative launch.  CTA b owns neurons [n0, n1) (an
// even split of N): their adjoint state (lambda_v, the carried trace adjoints and lambda_x) stays in
// shared memory for the launch, and the CTA computes both their neuron adjoints and their rows of
// the pull-back.  Per step t:
//   the own neurons' adjoints (adj_neuron_bwd_one): lambda_ge(t) into the segment's lambda_ge rows
//   (kept for dL/dW_EE), lambda_gi(t) into one of two buffers by step parity;
//   grid barrier (every CTA now needs every neuron's lambda_g);
//   lambda_ge(t) and lambda_gi(t) into shared memory, then the own rows' pull-back: lambda_x(t) of
//   the own neurons, which only this CTA's adjoints of step t - 1 read, so no second barrier is
//   needed.  A lambda_gi buffer is written again two steps later, after every CTA has passed the
//   barrier that follows its reads.
// The pull-back splits each own row into kPbChunks pieces, one (row, piece) per warp at a time,
// and adds a row's pieces in order.  The first `n_res` own rows of W are copied into shared memory
// at launch start (W does not change during the pass); the others stream from L2, and their
// pieces are taken first, so their loads are in flight while the resident rows are summed.
// The g_leak shares are summed per thread over the segment, then over the CTA in a fixed order.
// The barrier's wait is bounded (s_wait_limit_ns); a timeout sets the error word.
struct AdjBwd {
    const float *tv, *tu, *tge, *tgi;   // the segment's tape, [steps][N]
    const uint8_t *ts, *tref;
    float *lam_v, *lam_d, *lam_r, *lam_x;  // [N] carried between segments
    const float *c_s, *c_v;              // [T] the loss sensitivities
    float* lge_all;                      // [steps][ld] lambda_ge rows (zero beyond N)
    float* lgi2;                         // [2][ld] lambda_gi by step parity (zero beyond N)
    double* gl_acc;                      // [grid] g_leak shares, added to
    unsigned long long* barrier;
    int32_t* error;
    unsigned long long wait_limit_ns;
    uint32_t t0, steps, ld, max_own, n_res;
    float beta;
};
constexpr uint32_t kAdjBwdThreads = 512;
constexpr uint32_t kAdjTmemCols = 256;  // tensor memory of the backward kernel: W rows shared memory cannot hold

// One 32-bit column of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_st1(uint32_t taddr, float v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(__float_as_uint(v)) : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
constexpr uint32_t kPbChunks = 4;

// One warp: the piece [q0, q1) (in float4 units) of row `row` (ld floats) times lambda.
template <bool SMEM>
__device__ __forceinline__ float adj_pullback_piece(const float* row, const float* lam, uint32_t q0, uint32_t q1,
                                                    uint32_t lane) {
    const float4* r4 = reinterpret_cast<const float4*>(row);
    const float4* l4 = reinterpret_cast<const float4*>(lam);
    float acc = 0.0f;
#pragma unroll 8
    for (uint32_t q = q0 + lane; q < q1; q += 32u) {
        const float4 w = SMEM ? r4[q] : __ldg(r4 + q), l = l4[q];
        acc = fmaf(w.x, l.x, acc);
        acc = fmaf(w.y, l.y, acc);
        acc = fmaf(w.z, l.z, acc);
        acc = fmaf(w.w, l.w, acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    return acc;
}

__global__ void __launch_bounds__(kAdjBwdThreads, 1) bsnn_adj_backward_kernel(ADev A, AdjBwd B) {
    // lambda_ge [ld], lambda_gi [ld], own state [4][max_own], pieces [max_own][kPbChunks], rows [n_res][ld]
    extern __shared__ __align__(16) float adj_sm[];
    __shared__ int s_ok;
    __shared__ unsigned long long s_bar0;
    __shared__ double s_red[kAdjBwdThreads / 32];
    __shared__ uint32_t s_tmem;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u, nwarps = blockDim.x >> 5;
    const uint32_t N = A.N, ld = B.ld;
    const uint32_t n0 = static_cast<uint32_t>(static_cast<unsigned long long>(blockIdx.x) * N / gridDim.x);
    const uint32_t n1 = static_cast<uint32_t>(static_cast<unsigned long long>(blockIdx.x + 1u) * N / gridDim.x);
    const uint32_t own = n1 - n0;
    float* s_lge = adj_sm;
    float* s_lgi = adj_sm + ld;
    float* s_lv = adj_sm + 2u * ld;
    float* s_ld = s_lv + B.max_own;
    float* s_lr = s_ld + B.max_own;
    float* s_lx = s_lr + B.max_own;
    float* s_part = s_lx + B.max_own;
    float* s_w = adj_sm + 2u * ld + ((4u * B.max_own + kPbChunks * B.max_own + 3u) & ~3u);
    const uint32_t n_res = own < B.n_res ? own : B.n_res;
    for (uint32_t r = 0; r < n_res; ++r) {
        const uint32_t pre = n0 + r;
        const float4* src = reinterpret_cast<const float4*>(pre < A.E ? A.WE + static_cast<size_t>(pre) * ld
                                                                        : A.WI + static_cast<size_t>(pre - A.E) * ld);
        for (uint32_t q = tid; q < ld / 4u; q += blockDim.x)
            reinterpret_cast<float4*>(s_w + static_cast<size_t>(r) * ld)[q] = __ldg(src + q);
    }
    // Own rows n_res .. n_res + n_tm - 1 in tensor memory: element e of streamed row sr at lane
    // e mod 128, column sr * cpr + e / 128 (zero past ld).  Warp w reaches lanes 32 (w mod 4) ...
    // (a row spans cpr <= 32 columns, read as two 16-column loads that stay inside the allocation)
    const uint32_t cpr = (ld + 127u) / 128u, n_str = own - n_res;
    const uint32_t tm_max = cpr <= 32u ? (kAdjTmemCols - 32u) / cpr + 1u : 0u;
    const uint32_t n_tm = n_str < tm_max ? n_str : tm_max;
    if (warp == 0) {
        tmem_alloc(saddr(&s_tmem), kAdjTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    if (warp < 4u) {
        for (uint32_t sr = 0; sr < n_tm; ++sr) {
            const uint32_t pre = n0 + n_res + sr;
            const float* src = pre < A.E ? A.WE + static_cast<size_t>(pre) * ld : A.WI + static_cast<size_t>(pre - A.E) * ld;
            for (uint32_t c = 0; c < cpr; ++c) {
                const uint32_t e = c * 128u + 32u * warp + lane;
                tmem_st1(tmem + ((32u * warp) << 16) + sr * cpr + c, e < ld ? __ldg(src + e) : 0.0f);
            }
        }
        tmem_wait_st();
    }
    if (tid == 0) {
        s_wait_limit_ns = B.wait_limit_ns;
        s_bar0 = ld_acquire_u64(B.barrier) / gridDim.x * gridDim.x;
    }
    for (uint32_t i = tid; i < own; i += blockDim.x) {
        s_lv[i] = B.lam_v[n0 + i];
        s_ld[i] = B.lam_d[n0 + i];
        s_lr[i] = B.lam_r[n0 + i];
        s_lx[i] = B.lam_x[n0 + i];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned long long bar0 = s_bar0;
    double gl = 0.0;
    // Thread i steps own neuron i (own <= blockDim.x).  Its tape row and the loss sensitivities of
    // the next step to walk are loaded before the grid barrier, so their latency hides behind it.
    const bool mine = tid < own;
    const uint32_t n = n0 + tid;
    struct TapeRow {
        float v, u, ge, gi, cs, cv;
        uint8_t s, ref;
    };
    auto fetch = [&](uint32_t k) {
        TapeRow r{};
        const size_t o = static_cast<size_t>(k) * N + n;
        r.cs = B.c_s[B.t0 + k];
        r.cv = B.c_v[B.t0 + k];
        if (mine) {
            r.v = B.tv[o];
            r.u = B.tu[o];
            r.ge = B.tge[o];
            r.gi = B.tgi[o];
            r.s = B.ts[o];
            r.ref = B.tref[o];
        }
        return r;
    };
    TapeRow cur = fetch(B.steps - 1u);
    for (uint32_t kk = 0; kk < B.steps; ++kk) {
        const uint32_t k = B.steps - 1u - kk;
        float* lge_row = B.lge_all + static_cast<size_t>(k) * ld;
        float* lgi_buf = B.lgi2 + static_cast<size_t>(k & 1u) * ld;
        if (mine) {
            float lge, lgi;
            gl += adj_neuron_bwd_one(A, n, cur.v, cur.u, cur.ge, cur.gi, cur.s, cur.ref, s_lv[tid], s_ld[tid], s_lr[tid],
                                     s_lx[tid], cur.cs, cur.cv, B.beta, lge, lgi);
            lge_row[n] = lge;
            lgi_buf[n] = lgi;
        }
        if (k > 0u) cur = fetch(k - 1u);
        if (!grid_barrier(B.barrier, B.error, bar0 + (kk + 1ull) * gridDim.x, &s_ok)) break;
        // every neuron's lambda_g of step t (written by other CTAs: read from L2); only the side the
        // own rows pull back through (rows < E: lambda_ge, the others lambda_gi).  A thread issues
        // its loads of both sides, two float4 apart by blockDim each, before its first store, so
        // they cost one L2 round trip (ld / 4 <= 2 * blockDim here) instead of one per load.
        {
            const uint32_t n4 = ld / 4u;
            const bool use_e = n0 < A.E, use_i = n1 > A.E;
            const float4* src_e = reinterpret_cast<const float4*>(lge_row);
            const float4* src_i = reinterpret_cast<const float4*>(lgi_buf);
            for (uint32_t q = tid; q < n4; q += 2u * blockDim.x) {
                const uint32_t q2 = q + blockDim.x;
                const bool two = q2 < n4;
                const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                const float4 e0 = use_e ? __ldcg(src_e + q) : z, e1 = use_e && two ? __ldcg(src_e + q2) : z;
                const float4 i0 = use_i ? __ldcg(src_i + q) : z, i1 = use_i && two ? __ldcg(src_i + q2) : z;
                if (use_e) {
                    reinterpret_cast<float4*>(s_lge)[q] = e0;
                    if (two) reinterpret_cast<float4*>(s_lge)[q2] = e1;
                }
                if (use_i) {
                    reinterpret_cast<float4*>(s_lgi)[q] = i0;
                    if (two) reinterpret_cast<float4*>(s_lgi)[q2] = i1;
                }
            }
        }
        __syncthreads();
        {
            // the rows in tensor memory: the warps of lane quarter q = warp mod 4 take one row at a
            // time, a quarter of its elements each; the 4 quarter sums go where a row's pieces go
            const uint32_t q = warp & 3u;
            for (uint32_t sr = warp >> 2; sr < n_tm; sr += nwarps >> 2) {
                const float* lam = n0 + n_res + sr < A.E ? s_lge : s_lgi;
                float v[32];
                tmem_ld16(tmem + ((32u * q) << 16) + sr * cpr, v);
                tmem_ld16(tmem + ((32u * q) << 16) + sr * cpr + 16u, v + 16);
                float acc = 0.0f;
#pragma unroll
                for (uint32_t c = 0; c < 32u; ++c) {
                    const uint32_t e = c * 128u + 32u * q + lane;
                    if (c < cpr && e < ld) acc = fmaf(v[c], lam[e], acc);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
                if (lane == 0) s_part[(n_res + sr) * kPbChunks + q] = acc;
            }
            // the other rows in pieces: those streamed from L2 first, then those in shared memory
            const uint32_t n4 = ld / 4u, cq = (n4 + kPbChunks - 1u) / kPbChunks, n_l2 = own - n_res - n_tm;
            for (uint32_t p = warp; p < (n_res + n_l2) * kPbChunks; p += nwarps) {
                const uint32_t rr = p / kPbChunks, c = p % kPbChunks;
                const uint32_t r = rr < n_l2 ? n_res + n_tm + rr : rr - n_l2;
                const uint32_t pre = n0 + r;
                const float* lam = pre < A.E ? s_lge : s_lgi;
                const uint32_t q0 = c * cq < n4 ? c * cq : n4, q1 = q0 + cq < n4 ? q0 + cq : n4;
                float acc;
                if (r < n_res) {
                    acc = adj_pullback_piece<true>(s_w + static_cast<size_t>(r) * ld, lam, q0, q1, lane);
                } else {
                    const float* row = pre < A.E ? A.WE + static_cast<size_t>(pre) * ld
                                                 : A.WI + static_cast<size_t>(pre - A.E) * ld;
                    acc = adj_pullback_piece<false>(row, lam, q0, q1, lane);
                }
                if (lane == 0) s_part[r * kPbChunks + c] = acc;
            }
        }
        __syncthreads();
        if (mine) {
            float acc = 0.0f;
#pragma unroll
            for (uint32_t c = 0; c < kPbChunks; ++c) acc += s_part[tid * kPbChunks + c];
            s_lx[tid] = acc;
        }
    }
    // the CTA's g_leak share: warp sums, then the warps in order
    double v = gl;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (tid == 0) {
        double total = 0.0;
        for (uint32_t w = 0; w < nwarps; ++w) total += s_red[w];
        B.gl_acc[blockIdx.x] += total;
    }
    for (uint32_t i = tid; i < own; i += blockDim.x) {
        B.lam_v[n0 + i] = s_lv[i];
        B.lam_d[n0 + i] = s_ld[i];
        B.lam_r[n0 + i] = s_lr[i];
        B.lam_x[n0 + i] = s_lx[i];
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kAdjTmemCols);
}

// dW[pre, post] += sum_t X[t, pre] L[t, post] over one segment's steps (X: x_t of the E
// presynaptic neurons, rows of ldx floats; L: lambda_ge(t) of the E postsynaptic neurons, rows of
// ldl floats).  128 x 128 output tiles per block of 256 threads, 8 x 8 outputs per thread (pre =
// ty + 16 i, post = tx + 16 j); the steps pass through shared memory 8 at a time, the next 8
// loaded into registers while the current ones are used.  Each output adds its steps in order
// with fmaf, then adds the sum to dW.
constexpr uint32_t kOuterTile = 128, kOuterK = 8;
__global__ void __launch_bounds__(256) bsnn_adj_outer(const float* __restrict__ X, uint32_t ldx,
                                                      const float* __restrict__ L, uint32_t ldl, uint32_t steps,
                                                      uint32_t E, float* __restrict__ dW) {
    __shared__ float xs[2][kOuterK][kOuterTile], ls[2][kOuterK][kOuterTile];
    const uint32_t pre0 = blockIdx.y * kOuterTile, post0 = blockIdx.x * kOuterTile;
    const uint32_t tid = threadIdx.x, tx = tid & 15u, ty = tid >> 4;
    // this thread's loads of a k-tile: step row lr, columns lc .. lc + 3 of both operands
    const uint32_t lr = tid >> 5, lc = (tid & 31u) * 4u;
    float ra[4], rb[4];
    auto fetch = [&](uint32_t t0) {
        const uint32_t t = t0 + lr;
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            ra[q] = t < steps && pre0 + lc + q < E ? __ldg(X + static_cast<size_t>(t) * ldx + pre0 + lc + q) : 0.0f;
            rb[q] = t < steps && post0 + lc + q < E ? __ldg(L + static_cast<size_t>(t) * ldl + post0 + lc + q) : 0.0f;
        }
    };
    auto stash = [&](uint32_t buf) {
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            xs[buf][lr][lc + q] = ra[q];
            ls[buf][lr][lc + q] = rb[q];
        }
    };
    float acc[8][8];
#pragma unroll
    for (uint32_t i = 0; i < 8; ++i)
#pragma unroll
        for (uint32_t j = 0; j < 8; ++j) acc[i][j] = 0.0f;
    fetch(0);
    stash(0);
    __syncthreads();
    uint32_t buf = 0;
    for (uint32_t t0 = 0; t0 < steps; t0 += kOuterK) {
        const bool more = t0 + kOuterK < steps;
        if (more) fetch(t0 + kOuterK);
#pragma unroll
        for (uint32_t k = 0; k < kOuterK; ++k) {
            float a[8], b[8];
#pragma unroll
            for (uint32_t i = 0; i < 8; ++i) a[i] = xs[buf][k][ty + 16u * i];
#pragma unroll
            for (uint32_t j = 0; j < 8; ++j) b[j] = ls[buf][k][tx + 16u * j];
#pragma unroll
            for (uint32_t i = 0; i < 8; ++i)
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (more) stash(buf ^ 1u);
        __syncthreads();
        buf ^= 1u;
    }
#pragma unroll
    for (uint32_t i = 0; i < 8; ++i) {
        const uint32_t pre = pre0 + ty + 16u * i;
        if (pre >= E) continue;
#pragma unroll
        for (uint32_t j = 0; j < 8; ++j) {
            const uint32_t post = post0 + tx + 16u * j;
            if (post < E) dW[static_cast<size_t>(pre) * E + post] += acc[i][j];
        }
    }
}

}  // namespace bsnn
