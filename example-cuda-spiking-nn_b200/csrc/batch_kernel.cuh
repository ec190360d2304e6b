// batch_kernel.cuh -- the batched form: many independent networks ("instances") of uneven size,
// without plasticity, stepped together by one persistent cooperative kernel.
//
// Instances of one size class share one weight set, stored once in BF16, so the class's
// propagation for all its instances is a GEMM: for the excitatory presynaptic side
//     G_E[post, instance] = sum_pre W_E[pre, post] x_E[instance, pre]
// with W_E = [W_EE | W_EI] (E posts, then I posts), and likewise for the inhibitory side with
// W_I = [W_IE | W_II].  It runs on the 5th-generation tensor cores: D[128 posts x N] in tensor
// memory += A[128 posts x 64 pre] (W^T tile) * B[64 pre x N] (x tile), kind::f16 with BF16
// operands and FP32 accumulation.  x is split into a BF16 high part and a BF16 low part
// (x = hi + lo to about 2^-17), the two parts being the first and second halves of B's N
// columns, so the GEMM keeps x at nearly FP32 precision; the epilogue adds the two halves.
//
// Per clock step:
//   phase A (all neurons of all instances, grid-strided threads): g = g_base + the previous
//     step's GEMM partial sums (fixed order over K chunks), background Poisson shot noise
//     (the same counter-based Philox draw as the single-network kernel, keyed by the instance's
//     seed and the neuron's index in its instance), the conductance-EIF Euler step, the stimulus
//     events of the step, the connection traces, and x = d - r written as BF16 hi / lo into the
//     B operand tiles; spike counts per instance and group.
//   grid barrier
//   phase B (work units, a fixed list per CTA): one unit = (class, presynaptic side, 128-post
//     tile, a chunk of 64-pre K tiles).  One thread streams the unit's A and B tiles into a ring
//     of shared-memory stages by bulk asynchronous copies (one copy per operand tile; the
//     operands are stored pre-tiled in the canonical no-swizzle K-major core-matrix layout)
//     and issues the MMAs; tcgen05.commit releases each stage and finally signals the
//     accumulator; four warps read the 128 x N accumulator from tensor memory and write the
//     unit's partial sums.
//   grid barrier
//
// Each CTA steps a fixed contiguous range of neurons.  When the range's state fits beside the
// operand stages, it stays in shared memory for the whole launch (loaded at the start, written
// back at the end), so phase A's only global traffic is the partial sums in and x out, and the
// weight tiles have L2 to themselves; otherwise phase A reads and writes the state in global
// memory.  The stored background conductance is not kept: it is recomputed as (d - r) * scale
// from the background traces, the same expression that produced it.
//
// The background Poisson counts of a step depend only on (instance seed, neuron, step), so the
// warps that phase B leaves idle (5-15) draw the next step's counts for the CTA's neurons into
// shared memory while the GEMM runs, and phase A only reads them.
//
// Every wait is bounded (2 s): a timeout sets the error word and the kernel stops stepping,
// still releasing its tensor memory.
#pragma once

#include "step_kernel.cuh"

namespace bsnn {

constexpr uint32_t kBatchMaxClasses = 8;
constexpr uint32_t kBatchStages = 8;        // the largest shared-memory ring of operand stages
constexpr uint32_t kBatchTmemCols = 512;    // two accumulators of up to 256 columns (N <= 256)
constexpr uint32_t kAccCols = 256;
constexpr uint32_t kUnitRing = 4;           // units named ahead by the loader (phased form)
constexpr uint32_t kBatchThreads = 512;
constexpr uint32_t kATileBytes = 128u * 64u * 2u;  // one 128 x 64 BF16 A tile

// A size class: instances with the same numbers of neurons share its weights.
struct BClass {
    uint32_t E, I, N;        // neurons per instance (N = E + I)
    uint32_t n_inst, NP;     // instances; NP = n_inst rounded up to 8 (B has 2 NP rows: hi, lo)
    uint32_t nbase, nlen;    // the class's neurons: [nbase, nbase + nlen) (instances are numbered
                             // class by class, so a class's neurons are contiguous)
    uint32_t MT;             // 128-post tiles
    uint32_t KT[2];          // 64-pre K tiles of the E and I sides
    uint32_t nkc[2];         // K chunks per post tile (one unit each)
    size_t pbase[2];         // float offset of the partial sums of (side, post tile 0, chunk 0);
                             // unit (mt, kc) of a side holds NP x 128 floats at
                             // pbase + (mt * nkc + kc) * NP * 128
    const uint16_t* A[2];    // [MT][KT] tiles of W^T (BF16 bits), core-matrix layout
    uint16_t* X[2];          // [KT] tiles of x (2 NP rows), core-matrix layout
    float r_decay[2], d_decay[2], norm[2];  // connection traces of the E- and I-side connections
};

// The neuron-group parameters the neuron phase uses (NeuronGroupView, plus the Poisson means'
// exp(-mean)).
struct BGroupP {
    float dt_c;  // timestep / membrane_capacitance, divided once on the host (the same IEEE quotient)
    float g_leak, delta_t, v_eff, e_exc, e_inh, v_th, v_reset, v_rest;
    float exp_neg_mean_e, exp_neg_mean_i, bg_er_decay, bg_ed_decay, bg_ir_decay, bg_id_decay, bg_scale_e, bg_scale_i;
    uint32_t refractory_steps, has_bg_e, has_bg_i;
};

// One instance: its class, its row in the class's B operand, its first neuron, seed, its index in
// the order the instances were added (`id`, which indexes the spike counts) and its groups.  The
// table is sorted by first neuron.
struct BInst {
    uint32_t cls, row, nbase, seed, id, pad_;
    BGroupP g[2];  // E, I
};

struct BUnit {
    uint32_t cls, side, mt, k0, k1;
    size_t part;  // float offset of the unit's partial sums [NP][128]
};

struct BSim {
    uint32_t n_classes, n_inst, n_neurons, n_units;
    BClass cls[kBatchMaxClasses];
    const BInst* inst;
    uint32_t stage_bytes;         // one shared-memory operand stage (A tile + the largest B tile)
    uint32_t n_stages;            // operand stages in the ring (2 .. kBatchStages)
    uint32_t inst_in_smem;        // the instance table is copied into shared memory
    uint32_t state_in_smem;       // the CTA's neuron state lives in shared memory
    uint32_t per_cta;             // neurons per CTA (the last CTA may have fewer)
    uint32_t state_off;           // byte offset of the shared-memory state
    uint32_t noise_off;           // byte offset of the shared-memory noise counts [per_cta] (u16)
    const BUnit* units;           // longest first; CTAs take them in this order
    unsigned long long* unit_ctr; // unit dispenser: n_units takes per clock step
    float* partials;
    // neuron state [n_neurons]
    float *v, *istim, *er, *ed, *ir, *id, *tr, *td;
    uint32_t* refrac;
    uint32_t* spikes;
    unsigned long long* spike_counts;  // [n_inst][2]
    // stimulus: events of step t are ev_*[stim_off[t] .. stim_off[t+1]), sorted by neuron
    uint32_t stim_len;
    const uint32_t* stim_off;
    const uint32_t* ev_neuron;
    const float* ev_delta;
    int32_t noise_on;
    unsigned long long* phase_ns;  // [n_ctas][8] phase clock tallies (profiling builds)
    unsigned long long* barrier;
    int32_t* error;
    unsigned long long* steps_done;
    unsigned long long wait_limit_ns;  // bound of every device-side wait of a launch
    // the flow form (bsnn_batch_flow_kernel)
    uint32_t order[kBatchMaxClasses];     // classes in processing order (most GEMM work first)
    uint32_t units_of[kBatchMaxClasses];  // GEMM units per class
    unsigned long long* nready;           // [kBatchMaxClasses] CTA slices stepped (+1 per CTA per step)
    unsigned long long* udone;            // [kBatchMaxClasses] unit epilogue warps done (+4 per unit per step)
    // the phased form's class waits instead of grid barriers (classwait): a unit waits until every
    // CTA whose range holds neurons of its class has stepped them (nready[c] reaches
    // (t + 1) * ctas_of[c]), a CTA's phase A until its classes' units of the previous step are done
    uint32_t classwait;
    uint32_t ctas_of[kBatchMaxClasses];
};

// ---- tcgen05 / tensor-memory wrappers ---------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(cols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// D[tmem] (+)= A[smem] * B[smem], BF16 x BF16 -> FP32, M = 128.
__device__ __forceinline__ void tc_mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// 16 consecutive 32-bit accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* out) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) out[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
// An L2 policy that keeps the lines it touches (the weight tiles: every step reads all of them,
// and with the neuron state and the partial sums they fit in L2 together).
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void bulk_load_keep(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Shared-memory matrix descriptor, canonical K-major layout without swizzle: 8-row x 16-byte
// core matrices; `lbo` = bytes between the two core matrices of one K=16 step, `sbo` = bytes
// between consecutive 8-row groups; descriptor version 1 (bits 46-47).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t idesc_bf16_m128(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}
// Element offset of (row, k) in a [rows x 64] operand tile in core-matrix layout.
__host__ __device__ __forceinline__ uint32_t core_offset(uint32_t rows, uint32_t row, uint32_t k) {
    return ((((k >> 3) * (rows >> 3) + (row >> 3)) << 3) + (row & 7u)) * 8u + (k & 7u);
}

__device__ __forceinline__ uint16_t bf16_bits_rn(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }

// ---- phase A ------------------------------------------------------------------------------------
// Each CTA takes a contiguous range of neurons, one neuron per thread at a time, instance by
// instance: a range covers a few instances, and each instance's lookups (groups, B-operand row,
// partial-sum offsets, trace constants) are done once for its segment, not per neuron.  The
// phase is bound by instruction issue at 16 warps per SM: two neurons in flight per thread, or
// gathering the partial sums with many loads in flight first, measured slower or no faster.

// The state a CTA steps: shared-memory arrays indexed by n - base (base = the CTA's first
// neuron), or the global arrays (base = 0).  Spikes are bytes in shared memory, words in global.
struct BState {
    float *v, *istim, *er, *ed, *ir, *id, *tr, *td;
    uint32_t* refrac;
    uint8_t* spike8;
    uint32_t* spike32;
    uint32_t base;
};

template <bool SMEM>
__device__ __forceinline__ float st_ld(const float* p) {
    if constexpr (SMEM) return *p;
    else return __ldcg(p);
}
template <bool SMEM>
__device__ __forceinline__ uint32_t st_ld(const uint32_t* p) {
    if constexpr (SMEM) return *p;
    else return __ldcg(p);
}

__device__ __forceinline__ uint32_t instance_of(const BInst* P, uint32_t n_inst, uint32_t n) {
    uint32_t lo = 0, hi = n_inst;  // last instance whose first neuron is <= n
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (P[mid].nbase <= n) lo = mid;
        else hi = mid;
    }
    return lo;
}

// One instance's share of a CTA's neurons, with what every neuron of it needs, looked up once:
// its groups, its row in the class's B operand, the offsets of its partial sums and the class's
// connection traces.
struct SegCtx {
    const BGroupP* g;        // the instance's E and I groups (g[0], g[1])
    uint32_t nbase, E, id, NP, row;
    uint32_t pe, pi;         // float offsets of the partial sums of (side, post tile 0, chunk 0, row)
    uint32_t te, ti;         // floats per post tile of each side (nkc * NP * 128)
    uint32_t nkc0, nkc1, stride;
    uint16_t *X0, *X1;
    float r0, r1, d0, d1, m0, m1;  // connection trace decays and normalisation, by side
};

__device__ __forceinline__ SegCtx seg_ctx(const BInst& B, const BClass& C) {
    SegCtx c;
    c.g = B.g;
    c.nbase = B.nbase;
    c.E = C.E;
    c.id = B.id;
    c.NP = C.NP;
    c.row = B.row;
    c.stride = C.NP * 128u;
    c.pe = static_cast<uint32_t>(C.pbase[0]) + B.row * 128u;
    c.pi = static_cast<uint32_t>(C.pbase[1]) + B.row * 128u;
    c.nkc0 = C.nkc[0];
    c.nkc1 = C.nkc[1];
    c.te = C.nkc[0] * c.stride;
    c.ti = C.nkc[1] * c.stride;
    c.X0 = C.X[0];
    c.X1 = C.X[1];
    c.r0 = C.r_decay[0];
    c.r1 = C.r_decay[1];
    c.d0 = C.d_decay[0];
    c.d1 = C.d_decay[1];
    c.m0 = C.norm[0];
    c.m1 = C.norm[1];
    return c;
}

// What every neuron of a step reads from the launch descriptor, loaded once per step: the partial
// sums, the spike counters, whether the background noise is on, and the step's stimulus events
// [ev_lo, ev_hi) (sorted by neuron; empty on steps without events).
struct StepCtx {
    const float* partials;
    unsigned long long* spike_counts;
    uint32_t noise_on, ev_lo, ev_hi;
};

__device__ __forceinline__ StepCtx step_ctx(const BSim* S, unsigned long long t) {
    StepCtx k;
    k.partials = S->partials;
    k.spike_counts = S->spike_counts;
    k.noise_on = S->noise_on;
    k.ev_lo = k.ev_hi = 0;
    if (t < S->stim_len) {
        k.ev_lo = __ldg(S->stim_off + t);
        k.ev_hi = __ldg(S->stim_off + t + 1);
    }
    return k;
}

// One neuron's step (n: its index, i = n - X.base its state index): g = the background of the
// previous step (recomputed from its traces) + the previous step's propagation (K chunks in
// order), background Poisson shot noise, the conductance-EIF Euler step, the step's stimulus
// events, the connection traces, and x = d - r as BF16 hi / lo into the B operand.
// The previous step's partial sums of neuron j of an instance whose sides have at most 2 K chunks
// each, loaded but not yet added: the loads of the next neuron are issued before this one's
// update (a loop over a count known only at run time would wait for each load before issuing
// the next).
struct PartRaw {
    float e0, e1, g0, g1;
};
__device__ __forceinline__ PartRaw part_load(const StepCtx& sc, const SegCtx& c, uint32_t j) {
    const float* pe = sc.partials + c.pe + (j >> 7) * c.te + (j & 127u);
    const float* pi = sc.partials + c.pi + (j >> 7) * c.ti + (j & 127u);
    PartRaw r;
    r.e0 = __ldcg(pe);
    r.g0 = __ldcg(pi);
    r.e1 = c.nkc0 > 1u ? __ldcg(pe + c.stride) : 0.0f;
    r.g1 = c.nkc1 > 1u ? __ldcg(pi + c.stride) : 0.0f;
    return r;
}
// Their sums, K chunks in order from 0.
__device__ __forceinline__ float2 part_sum(const PartRaw& r, const SegCtx& c) {
    float dge = 0.0f, dgi = 0.0f;
    dge += r.e0;
    if (c.nkc0 > 1u) dge += r.e1;
    dgi += r.g0;
    if (c.nkc1 > 1u) dgi += r.g1;
    return make_float2(dge, dgi);
}
// The same sums for any number of K chunks.
__device__ __forceinline__ float2 part_sums_any(const StepCtx& sc, const SegCtx& c, uint32_t j) {
    const float* pe = sc.partials + c.pe + (j >> 7) * c.te + (j & 127u);
    const float* pi = sc.partials + c.pi + (j >> 7) * c.ti + (j & 127u);
    float dge = 0.0f, dgi = 0.0f;
    for (uint32_t kc = 0; kc < c.nkc0; ++kc) dge += __ldcg(pe + kc * c.stride);
    for (uint32_t kc = 0; kc < c.nkc1; ++kc) dgi += __ldcg(pi + kc * c.stride);
    return make_float2(dge, dgi);
}

// dg: the previous step's propagation onto the neuron (its partial sums; unused at t = 0).
template <bool SMEM>
__device__ __forceinline__ void neuron_step(const BSim* S, const StepCtx& sc, const SegCtx& c, const BState& X,
                                            const uint16_t* nz, uint32_t n0, uint32_t n, unsigned long long t,
                                            float2 dg) {
    const uint32_t i = n - X.base;
    const uint32_t j = n - c.nbase;  // index in the instance
    const uint32_t side = j < c.E ? 0u : 1u;
    const BGroupP& G = c.g[side];
    const uint32_t loc = j - (side ? c.E : 0u);
    const float dge = dg.x, dgi = dg.y;
    const float a_v = st_ld<SMEM>(X.v + i), a_istim = st_ld<SMEM>(X.istim + i);
    const float a_er = st_ld<SMEM>(X.er + i), a_ed = st_ld<SMEM>(X.ed + i);
    const float a_ir = st_ld<SMEM>(X.ir + i), a_id = st_ld<SMEM>(X.id + i);
    const float a_tr = st_ld<SMEM>(X.tr + i), a_td = st_ld<SMEM>(X.td + i);
    const uint32_t a_refrac = st_ld<SMEM>(X.refrac + i);
    // g = the background of the previous step (recomputed from its traces) + its propagation
    float ge_used = (a_ed - a_er) * G.bg_scale_e, gi_used = (a_id - a_ir) * G.bg_scale_i;
    if (t > 0) {
        ge_used = ge_used + dge;
        gi_used = gi_used + dgi;
    }

    float er = flush_tiny(a_er * G.bg_er_decay);
    float ir = flush_tiny(a_ir * G.bg_ir_decay);
    float ed = flush_tiny(a_ed * G.bg_ed_decay);
    float id = flush_tiny(a_id * G.bg_id_decay);
    uint32_t ne = 0, ni = 0;
    if (sc.noise_on) {
        const uint32_t cnt = nz[n - n0];
        ne = cnt & 0xFFu;
        ni = cnt >> 8;
    }
    if (ne > 0u) {
        const float inc = static_cast<float>(ne);
        er += inc;
        ed += inc;
    }
    if (ni > 0u) {
        const float inc = static_cast<float>(ni);
        ir += inc;
        id += inc;
    }

    float v = a_v, istim = a_istim;
    uint32_t refrac = a_refrac, spike = 0;
    if (refrac > 0) {
        --refrac;
        v = G.v_reset;
    } else {
        const float linear_leak_term = -1.0f * G.g_leak * (v - G.v_rest);
        const float exponential_depolarization_term = G.g_leak * G.delta_t * expf((v - G.v_eff) / G.delta_t);
        const float excitatory_synaptic_term = -1.0f * ge_used * (v - G.e_exc);
        const float inhibitory_synaptic_term = -1.0f * gi_used * (v - G.e_inh);
        const float dv = G.dt_c * (linear_leak_term + exponential_depolarization_term + excitatory_synaptic_term +
                                   inhibitory_synaptic_term + istim);
        const float v_next = v + dv;
        if (v_next >= G.v_th) {
            refrac = G.refractory_steps;
            spike = 1;
            v = G.v_th;
        } else {
            v = v_next;
        }
    }
    X.er[i] = er;
    X.ed[i] = ed;
    X.ir[i] = ir;
    X.id[i] = id;
    X.v[i] = v;
    X.refrac[i] = refrac;
    if constexpr (SMEM) X.spike8[i] = static_cast<uint8_t>(spike);
    else X.spike32[i] = spike;
    if (spike) atomicAdd(sc.spike_counts + 2u * c.id + side, 1ull);

    // stimulus events of this step act from the next step
    if (sc.ev_lo < sc.ev_hi) {
        uint32_t lo = sc.ev_lo, hi = sc.ev_hi;
        const uint32_t end = hi;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(S->ev_neuron + mid) < n) lo = mid + 1;
            else hi = mid;
        }
        bool any = false;
        for (uint32_t k = lo; k < end && __ldg(S->ev_neuron + k) == n; ++k) {
            istim = istim + __ldg(S->ev_delta + k);
            any = true;
        }
        if (any) X.istim[i] = istim;
    }

    // connection traces of the neuron's presynaptic side, and x as BF16 hi / lo in B
    float d = flush_tiny(a_td * (side ? c.d1 : c.d0));
    float r = flush_tiny(a_tr * (side ? c.r1 : c.r0));
    if (spike == 1) {
        const float m = side ? c.m1 : c.m0;
        r += m;
        d += m;
    }
    X.tr[i] = r;
    X.td[i] = d;
    const float x = d - r;
    const uint16_t xhi = bf16_bits_rn(x);
    const float lo_f = x - __uint_as_float(static_cast<uint32_t>(xhi) << 16);
    const uint16_t xlo = bf16_bits_rn(lo_f);
    uint16_t* Xt = (side ? c.X1 : c.X0) + static_cast<size_t>(loc >> 6) * (2u * c.NP * 64u);
    Xt[core_offset(2u * c.NP, c.row, loc & 63u)] = xhi;
    Xt[core_offset(2u * c.NP, c.NP + c.row, loc & 63u)] = xlo;
}

// Neurons [n0, n1), by `count` threads of the CTA, this one being number `me`: instance by
// instance (a CTA's range covers a few), the instance's lookups done once per segment.
template <bool SMEM>
__device__ __forceinline__ void batch_neurons(const BSim* S, const BInst* P, const BClass* s_cls, const BState& X,
                                              const uint16_t* nz, uint32_t n0, uint32_t n1, unsigned long long t,
                                              uint32_t me, uint32_t count) {
    if (n0 >= n1) return;
    const StepCtx sc = step_ctx(S, t);
    uint32_t inst = instance_of(P, S->n_inst, n0);
    for (uint32_t seg0 = n0; seg0 < n1; ++inst) {
        const BInst& B = P[inst];
        const BClass& C = s_cls[B.cls];
        const uint32_t seg1 = min(n1, B.nbase + C.N);
        const SegCtx c = seg_ctx(B, C);
        uint32_t n = seg0 + me;
        if (t > 0 && c.nkc0 <= 2u && c.nkc1 <= 2u) {
            PartRaw r{};
            if (n < seg1) r = part_load(sc, c, n - c.nbase);
            for (; n < seg1; n += count) {
                const uint32_t nn = n + count;
                PartRaw rn{};
                if (nn < seg1) rn = part_load(sc, c, nn - c.nbase);  // in flight during this update
                neuron_step<SMEM>(S, sc, c, X, nz, n0, n, t, part_sum(r, c));
                r = rn;
            }
        } else {
            for (; n < seg1; n += count)
                neuron_step<SMEM>(S, sc, c, X, nz, n0, n, t,
                                  t > 0 ? part_sums_any(sc, c, n - c.nbase) : make_float2(0.0f, 0.0f));
        }
        seg0 = seg1;
    }
}

// The background Poisson counts of step t for neurons [n0, n1), drawn by `count` threads of the
// CTA, this one being number `me`: nz[n - n0] = n_e | n_i << 8 (each saturates at 255).
__device__ __forceinline__ void noise_ahead(const BSim* S, const BInst* P, const BClass* s_cls, uint16_t* nz, uint32_t n0,
                                            uint32_t n1, unsigned long long t, uint32_t me, uint32_t count) {
    uint32_t cur = instance_of(P, S->n_inst, n0 + me < n1 ? n0 + me : n0);
    for (uint32_t n = n0 + me; n < n1; n += count) {
        while (cur + 1u < S->n_inst && P[cur + 1u].nbase <= n) ++cur;
        const BInst& B = P[cur];
        const uint32_t j = n - B.nbase;
        const BGroupP& G = B.g[j < s_cls[B.cls].E ? 0 : 1];
        uint32_t ne, ni;
        poisson_knuth_pair(G.exp_neg_mean_e, G.has_bg_e, G.exp_neg_mean_i, G.has_bg_i, B.seed, j, t, ne, ni);
        nz[n - n0] = static_cast<uint16_t>(ne | (ni << 8));
    }
}
// The warps idle in phase B that draw the noise: warps 5-15 except those on sub-partition 0 (8 and
// 12), where the loader thread (warp 4) and the MMA thread (warp 8) run: their single threads'
// issue latency gates the GEMM.
__device__ __forceinline__ bool noise_warp(uint32_t warp) { return warp >= 5u && (warp & 3u) != 0u; }
__device__ __forceinline__ uint32_t noise_rank(uint32_t warp) {  // among the noise warps
    return (warp - 5u) - (warp >= 8u ? 1u : 0u) - (warp >= 12u ? 1u : 0u);
}
constexpr uint32_t kNoiseWarps = 9u;

// The CTA's shared-memory state arrays (`per` neurons each, from `raw` on), from index `soff` on,
// for neurons numbered from `base`.
__device__ __forceinline__ BState smem_state(unsigned char* raw, uint32_t per, uint32_t soff, uint32_t base) {
    float* f = reinterpret_cast<float*>(raw);
    BState X{};
    X.v = f + soff;
    X.istim = f + per + soff;
    X.er = f + 2 * per + soff;
    X.ed = f + 3 * per + soff;
    X.ir = f + 4 * per + soff;
    X.id = f + 5 * per + soff;
    X.tr = f + 6 * per + soff;
    X.td = f + 7 * per + soff;
    X.refrac = reinterpret_cast<uint32_t*>(f + 8 * per) + soff;
    X.spike8 = reinterpret_cast<uint8_t*>(f + 9 * per) + soff;
    X.base = base;
    return X;
}
__device__ __forceinline__ BState global_state(const BSim* S) {
    BState X{};
    X.v = S->v;
    X.istim = S->istim;
    X.er = S->er;
    X.ed = S->ed;
    X.ir = S->ir;
    X.id = S->id;
    X.tr = S->tr;
    X.td = S->td;
    X.refrac = S->refrac;
    X.spike32 = S->spikes;
    X.base = 0;
    return X;
}

// Copies the state of neurons [n0, n1) between global memory and shared-memory arrays indexed by
// n - n0.
__device__ __forceinline__ void state_copy(const BSim* S, const BState& X, uint32_t n0, uint32_t n1, bool to_smem) {
    float* g[8] = {S->v, S->istim, S->er, S->ed, S->ir, S->id, S->tr, S->td};
    float* sm[8] = {X.v, X.istim, X.er, X.ed, X.ir, X.id, X.tr, X.td};
    for (uint32_t n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
        const uint32_t i = n - n0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (to_smem) sm[k][i] = g[k][n];
            else g[k][n] = sm[k][i];
        }
        if (to_smem) {
            X.refrac[i] = S->refrac[n];
            X.spike8[i] = static_cast<uint8_t>(S->spikes[n]);
        } else {
            S->refrac[n] = X.refrac[i];
            S->spikes[n] = X.spike8[i];
        }
    }
}

// ---- phase B ------------------------------------------------------------------------------------
struct BatchSmem {
    uint32_t tmem;          // tensor-memory base address
    uint32_t ok;
    uint64_t full[kBatchStages];
    uint64_t empty[kBatchStages];
    uint64_t accum;   // the MMA thread's commit: the unit's accumulator is complete
    uint64_t ready[2];  // the producer has taken a unit (or found none left) and named it in unit[]
    uint32_t unit[2];
    uint64_t tfree;   // the 4 epilogue warps: the accumulator has been read
    // the phased form's split producer: the loader names units in a ring (ufull: named; uempty:
    // the MMA thread and the 4 epilogue warps are done with the slot), and the MMA thread fills
    // two accumulators in turn (afull: committed; aempty: the 4 epilogue warps have read it)
    uint64_t ufull[kUnitRing];
    uint64_t uempty[kUnitRing];
    uint32_t uid[kUnitRing];
    uint64_t afull[2];
    uint64_t aempty[2];
};

// The producer's ring and accumulator state (one thread).
struct ProducerState {
    uint32_t full_ph = 0, empty_ph = 0, tfree_ph = 0;
    uint32_t empty_pend = 0;  // bit s: stage s holds tiles whose MMAs may still read it
    uint32_t full_pend = 0;   // bit s: stage s has copies in flight not yet waited for
    uint32_t load_s = 0, use_s = 0, units_issued = 0;
};

// One GEMM unit on the producer thread: streams the unit's A and B tiles into the ring of
// shared-memory stages (one bulk copy per operand tile), issues the MMAs into the accumulator
// (after the epilogue has read the previous unit's), and commits the accumulator.  Returns false
// when a wait timed out (the accumulator is committed all the same, to release the epilogue).
__device__ __forceinline__ bool issue_unit(BatchSmem& bs, ProducerState& ps, const BUnit& U, const BClass& C,
                                           uint32_t tmem, uint32_t smem_base, uint32_t stage_bytes, uint32_t n_stages,
                                           uint64_t keep) {
    const uint32_t N = 2u * C.NP, b_bytes = N * 128u, nk = U.k1 - U.k0;
    const unsigned char* a_src =
        reinterpret_cast<const unsigned char*>(C.A[U.side]) + (static_cast<size_t>(U.mt) * C.KT[U.side] + U.k0) * kATileBytes;
    const unsigned char* b_src = reinterpret_cast<const unsigned char*>(C.X[U.side]) + static_cast<size_t>(U.k0) * b_bytes;
    bool good = true;
    // K tile i of the unit into stage load_s, once the MMAs that read the stage last are done
    auto load = [&](uint32_t i) {
        const uint32_t s = ps.load_s;
        if ((ps.empty_pend >> s) & 1u) {
            if (!mbar_wait(saddr(&bs.empty[s]), (ps.empty_ph >> s) & 1u)) good = false;
            ps.empty_ph ^= 1u << s;
            ps.empty_pend &= ~(1u << s);
        }
        const uint32_t bar = saddr(&bs.full[s]);
        const uint32_t dst = smem_base + s * stage_bytes;
        mbar_expect_tx(bar, kATileBytes + b_bytes);
        bulk_load_keep(dst, a_src + static_cast<size_t>(i) * kATileBytes, kATileBytes, bar, keep);
        bulk_load(dst + kATileBytes, b_src + static_cast<size_t>(i) * b_bytes, b_bytes, bar);
        ps.full_pend |= 1u << s;
        ps.load_s = ps.load_s + 1u == n_stages ? 0u : ps.load_s + 1u;
    };
    const uint32_t idesc = idesc_bf16_m128(N);
    uint32_t next = 0;
    for (; next < nk && next < n_stages; ++next) load(next);
    // the epilogue of the previous unit has read the accumulator
    if (ps.units_issued > 0u) {
        if (!mbar_wait(saddr(&bs.tfree), ps.tfree_ph & 1u)) good = false;
        ps.tfree_ph ^= 1u;
    }
    for (uint32_t i = 0; i < nk && good; ++i) {
        const uint32_t s = ps.use_s;
        if (!mbar_wait(saddr(&bs.full[s]), (ps.full_ph >> s) & 1u)) {
            good = false;
            break;
        }
        ps.full_ph ^= 1u << s;
        ps.full_pend &= ~(1u << s);
        tc_fence_after();
        const uint32_t a = smem_base + s * stage_bytes, b = a + kATileBytes;
#pragma unroll
        for (uint32_t ks = 0; ks < 4; ++ks)
            tc_mma_bf16(tmem, smem_desc(a + ks * 2u * 2048u, 2048u, 128u), smem_desc(b + ks * 2u * (N * 16u), N * 16u, 128u),
                        idesc, (i | ks) != 0u);
        tc_commit(saddr(&bs.empty[s]));
        ps.empty_pend |= 1u << s;
        ps.use_s = ps.use_s + 1u == n_stages ? 0u : ps.use_s + 1u;
        // refill the stage of the previous iteration (its MMAs have had an MMA's time to finish;
        // load() waits for them)
        if (i > 0u && next < nk) load(next++);
    }
    tc_commit(saddr(&bs.accum));
    ++ps.units_issued;
    return good;
}

// After a timeout, on the producer thread: waits (each wait bounded) for the copies it issued and
// for its last MMAs, so that none is in flight when the CTA frees its tensor memory and exits.
__device__ __forceinline__ void producer_quiesce(BatchSmem& bs, ProducerState& ps, uint32_t n_stages) {
    for (uint32_t s = 0; s < n_stages; ++s)
        if ((ps.full_pend >> s) & 1u) mbar_wait(saddr(&bs.full[s]), (ps.full_ph >> s) & 1u);
    if (ps.units_issued > 0u) mbar_wait(saddr(&bs.accum), (ps.units_issued - 1u) & 1u);
}

// One GEMM unit on the epilogue warps 0-3 (warp w reads accumulator lanes 32w .. 32w + 31, one
// post each): waits for the accumulator, adds its hi and lo halves, writes the class's instances'
// partial sums of the unit, and frees the accumulator.
__device__ __forceinline__ void drain_unit(const BSim* S, BatchSmem& bs, const BUnit& U, const BClass& C, uint32_t tmem,
                                           uint32_t& accum_ph, uint32_t warp, uint32_t lane) {
    const uint32_t row = 32u * warp + lane;
    const bool got = mbar_wait(saddr(&bs.accum), accum_ph & 1u);
    accum_ph ^= 1u;
    if (!got) {
        atomicExch(S->error, kErrStageTimeout);
        bs.ok = 0u;
    }
    tc_fence_after();
    float* part = S->partials + U.part;
    for (uint32_t c0 = 0; c0 < C.NP; c0 += 16u) {
        float hi[16], lo[16];
        tmem_ld16(tmem + ((32u * warp) << 16) + c0, hi);
        tmem_ld16(tmem + ((32u * warp) << 16) + C.NP + c0, lo);
#pragma unroll
        for (uint32_t q = 0; q < 16; ++q)
            if (c0 + q < C.n_inst) part[static_cast<size_t>(c0 + q) * 128u + row] = hi[q] + lo[q];
    }
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(saddr(&bs.tfree));
}

// Copies the launch-invariant tables into shared memory: the class table, and the instance table
// when the placement keeps it there (returned; else the global one).
__device__ __forceinline__ const BInst* batch_tables(const BSim* S, unsigned char* table_smem, BClass* s_cls) {
    const BInst* P = S->inst;
    if (S->inst_in_smem) {
        BInst* s_inst = reinterpret_cast<BInst*>(table_smem);
        for (uint32_t i = threadIdx.x; i < S->n_inst * (sizeof(BInst) / 4u); i += blockDim.x)
            reinterpret_cast<uint32_t*>(s_inst)[i] = reinterpret_cast<const uint32_t*>(S->inst)[i];
        P = s_inst;
    }
    for (uint32_t i = threadIdx.x; i < S->n_classes * (sizeof(BClass) / 4u); i += blockDim.x)
        reinterpret_cast<uint32_t*>(s_cls)[i] = reinterpret_cast<const uint32_t*>(S->cls)[i];
    return P;
}

// Thread 0: the ring's, the accumulator's and the unit ring's mbarriers.
__device__ __forceinline__ void batch_init_barriers(BatchSmem& bs, uint32_t n_stages) {
    bs.ok = 1u;
    for (uint32_t s = 0; s < n_stages; ++s) {
        mbar_init(saddr(&bs.full[s]), 1u);
        mbar_init(saddr(&bs.empty[s]), 1u);
    }
    mbar_init(saddr(&bs.accum), 1u);
    mbar_init(saddr(&bs.ready[0]), 1u);
    mbar_init(saddr(&bs.ready[1]), 1u);
    mbar_init(saddr(&bs.tfree), 4u);
    for (uint32_t u = 0; u < kUnitRing; ++u) {
        mbar_init(saddr(&bs.ufull[u]), 1u);
        mbar_init(saddr(&bs.uempty[u]), 5u);
    }
    for (uint32_t b = 0; b < 2; ++b) {
        mbar_init(saddr(&bs.afull[b]), 1u);
        mbar_init(saddr(&bs.aempty[b]), 4u);
    }
    fence_mbar_init();
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// One thread: bounded wait until the counter reaches `target`.  It polls with gpu-scope relaxed
// loads and makes one acquire load once the target is reached: these waits run beside the other
// roles' work, and an acquire load per poll would keep invalidating the SM's L1 under them.  Gives
// up after s_wait_limit_ns, recording kErrBarrierTimeout, or when another CTA has given up.
__device__ __forceinline__ bool count_wait(const unsigned long long* ctr, int32_t* error, unsigned long long target) {
    unsigned long long t_start = 0;
    uint32_t spins = 0;
    while (static_cast<long long>(ld_relaxed_u64(ctr) - target) < 0) {
        if ((++spins & 63u) == 0u) {
            const unsigned long long now = globaltimer_ns();
            if (t_start == 0) {
                t_start = now;
            } else if (now - t_start > s_wait_limit_ns) {
                atomicExch(error, kErrBarrierTimeout);
                return false;
            }
            if (ld_relaxed_s32(error) != kErrNone) return false;
        }
    }
    ld_acquire_u64(ctr);  // orders this thread's later reads after the counted work
    return true;
}

// ---- phase B of the phased form: loader, MMA thread and epilogue as separate roles -------------
// The loader (thread 128) takes units from the dispenser, names each in the unit ring and streams
// its operand tiles into the stage ring.  The MMA thread (thread 256: warp 8, which draws no noise)
// issues a unit's MMAs as its tiles land, into accumulator buffer (its count) mod 2.  The epilogue
// warps 0-3 drain the buffers in the same order.  So the loader's copies, the MMA issue and the
// drain of the previous unit overlap, instead of one thread doing the first two in turn.  Each
// role keeps its own counters, carried across steps: the u-th fill of a ring slot or stage is
// phase u of its barriers.
struct SplitState {
    unsigned long long held = 0;  // class waits: the loader's ticket not yet processed
    uint32_t units = 0;  // units named (loader) or taken from the ring (MMA thread, epilogue)
    uint32_t stage = 0;  // the next stage, and how many times it was used before
    uint32_t use = 0;
    uint32_t accs = 0;   // accumulators filled (MMA thread) or drained (epilogue)
    uint32_t tiles = 0;  // k-tiles loaded (loader)
};
constexpr uint32_t kNoUnit = 0xFFFFFFFFu;

// The loader for one step: every processed unit is followed by exactly one take (units grid,
// grid + 1, ... after CTA b's first unit b), so a step makes n_units takes from t * n_units.
__device__ __forceinline__ bool split_loader(const BSim* S, BatchSmem& bs, const BClass* s_cls, SplitState& L,
                                             unsigned long long t, uint32_t smem_base, uint32_t stage_bytes,
                                             uint32_t n_stages, uint64_t keep) {
    const uint32_t n_units = S->n_units;
    const unsigned long long take0 = t * n_units;
    const bool classwait = S->classwait != 0u;
    bool good = true;
    // Grid barriers: CTA b starts with unit b, then takes from the dispenser (numbered from
    // t * n_units in the step).  Class waits: CTAs may be in different steps, so the dispenser is
    // one ticket sequence over the launch (ticket q: unit q mod n_units of step q / n_units), and
    // the loader holds its first ticket of a later step for that step's phase B.
    uint32_t ui = blockIdx.x;
    if (classwait) {
        const unsigned long long tq = L.held / n_units;
        ui = tq == t ? static_cast<uint32_t>(L.held - tq * n_units) : n_units;
    }
    for (;;) {
        const uint32_t slot = L.units % kUnitRing;
        if (L.units >= kUnitRing && !mbar_wait(saddr(&bs.uempty[slot]), ((L.units / kUnitRing) - 1u) & 1u)) good = false;
        bool none = ui >= n_units || !good || bs.ok == 0u;
        if (!none && classwait) {
            // every CTA holding neurons of the unit's class has stepped them (x tiles written by
            // generic stores, read by the bulk copies below)
            const uint32_t c = S->units[ui].cls;
            if (count_wait(S->nready + c, S->error, (t + 1ull) * S->ctas_of[c])) {
                fence_proxy_async_global();
            } else {
                good = false;
                none = true;
            }
        }
        bs.uid[slot] = none ? kNoUnit : ui;
        mbar_arrive(saddr(&bs.ufull[slot]));
        ++L.units;
        if (none) break;
        const BUnit U = S->units[ui];
        const BClass& C = s_cls[U.cls];
        const uint32_t b_bytes = 2u * C.NP * 128u, nk = U.k1 - U.k0;
        const unsigned char* a_src = reinterpret_cast<const unsigned char*>(C.A[U.side]) +
                                     (static_cast<size_t>(U.mt) * C.KT[U.side] + U.k0) * kATileBytes;
        const unsigned char* b_src =
            reinterpret_cast<const unsigned char*>(C.X[U.side]) + static_cast<size_t>(U.k0) * b_bytes;
        for (uint32_t i = 0; i < nk; ++i) {
            // the stage's previous tiles have been read by their MMAs
            if (L.use > 0u && !mbar_wait(saddr(&bs.empty[L.stage]), (L.use - 1u) & 1u)) {
                good = false;
                break;
            }
            const uint32_t bar = saddr(&bs.full[L.stage]), dst = smem_base + L.stage * stage_bytes;
            mbar_expect_tx(bar, kATileBytes + b_bytes);
            bulk_load_keep(dst, a_src + static_cast<size_t>(i) * kATileBytes, kATileBytes, bar, keep);
            bulk_load(dst + kATileBytes, b_src + static_cast<size_t>(i) * b_bytes, b_bytes, bar);
            ++L.tiles;
            if (++L.stage == n_stages) {
                L.stage = 0;
                ++L.use;
            }
        }
        if (classwait) {
            L.held = atomicAdd(S->unit_ctr, 1ull);
            const unsigned long long tq = L.held / n_units;
            ui = tq == t ? static_cast<uint32_t>(L.held - tq * n_units) : n_units;  // a later step's: held
        } else {
            ui = gridDim.x + static_cast<uint32_t>(atomicAdd(S->unit_ctr, 1ull) - take0);
        }
    }
    return good;
}

// The MMA thread for one step.  Descriptors: the stage's A and B base descriptors plus the K
// step's offset in the start-address field (shared-memory addresses stay below 256 KB).
__device__ __forceinline__ bool split_mma(const BSim* S, BatchSmem& bs, const BClass* s_cls, SplitState& M,
                                          uint32_t tmem, uint32_t smem_base, uint32_t stage_bytes, uint32_t n_stages) {
    bool good = true;
    for (;;) {
        const uint32_t slot = M.units % kUnitRing;
        if (!mbar_wait(saddr(&bs.ufull[slot]), (M.units / kUnitRing) & 1u)) return false;
        const uint32_t ui = bs.uid[slot];
        ++M.units;
        if (ui == kNoUnit) {
            mbar_arrive(saddr(&bs.uempty[slot]));
            break;
        }
        const BUnit U = S->units[ui];
        const BClass& C = s_cls[U.cls];
        const uint32_t N = 2u * C.NP, nk = U.k1 - U.k0, idesc = idesc_bf16_m128(N);
        const uint32_t buf = M.accs & 1u, fill = M.accs >> 1;
        // the epilogue has read this buffer's previous unit
        if (fill > 0u && !mbar_wait(saddr(&bs.aempty[buf]), (fill - 1u) & 1u)) good = false;
        tc_fence_after();
        const uint32_t d = tmem + buf * kAccCols;
        const uint64_t a0 = smem_desc(smem_base, 2048u, 128u), b0 = smem_desc(smem_base + kATileBytes, N * 16u, 128u);
        for (uint32_t i = 0; i < nk && good; ++i) {
            if (!mbar_wait(saddr(&bs.full[M.stage]), M.use & 1u)) {
                good = false;
                break;
            }
            tc_fence_after();
            const uint64_t so = (static_cast<uint64_t>(M.stage) * stage_bytes) >> 4;
#pragma unroll
            for (uint32_t ks = 0; ks < 4; ++ks)
                tc_mma_bf16(d, a0 + so + ks * 256u, b0 + so + ks * (2u * N), idesc, (i | ks) != 0u);
            tc_commit(saddr(&bs.empty[M.stage]));
            if (++M.stage == n_stages) {
                M.stage = 0;
                ++M.use;
            }
        }
        tc_commit(saddr(&bs.afull[buf]));  // also after a timeout, to release the epilogue
        ++M.accs;
        mbar_arrive(saddr(&bs.uempty[slot]));
        if (!good) break;
    }
    return good;
}

// The epilogue warps 0-3 for one step (warp w drains accumulator lanes 32w .. 32w + 31).  Every
// wait's outcome is made uniform over the warp before the warp-wide tensor-memory loads.
__device__ __forceinline__ bool split_epilogue(const BSim* S, BatchSmem& bs, const BClass* s_cls, SplitState& E,
                                               uint32_t tmem, uint32_t warp, uint32_t lane) {
    const uint32_t row = 32u * warp + lane;
    bool good = true;
    for (;;) {
        const uint32_t slot = E.units % kUnitRing;
        if (!__all_sync(kFull, mbar_wait(saddr(&bs.ufull[slot]), (E.units / kUnitRing) & 1u))) return false;
        const uint32_t ui = bs.uid[slot];
        ++E.units;
        if (ui == kNoUnit) {
            if (lane == 0) mbar_arrive(saddr(&bs.uempty[slot]));
            break;
        }
        const BUnit U = S->units[ui];
        const BClass& C = s_cls[U.cls];
        const uint32_t buf = E.accs & 1u, fill = E.accs >> 1;
        if (!__all_sync(kFull, mbar_wait(saddr(&bs.afull[buf]), fill & 1u))) good = false;
        ++E.accs;
        tc_fence_after();
        const uint32_t base = tmem + ((32u * warp) << 16) + buf * kAccCols;
        float* part = S->partials + U.part;
        for (uint32_t c0 = 0; c0 < C.NP; c0 += 16u) {
            float hi[16], lo[16];
            tmem_ld16(base + c0, hi);
            tmem_ld16(base + C.NP + c0, lo);
#pragma unroll
            for (uint32_t q = 0; q < 16; ++q)
                if (c0 + q < C.n_inst) part[static_cast<size_t>(c0 + q) * 128u + row] = hi[q] + lo[q];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(saddr(&bs.aempty[buf]));
            mbar_arrive(saddr(&bs.uempty[slot]));
            if (S->classwait) red_release_add_u64(S->udone + U.cls, 1ull);  // this warp's 32 posts are written
        }
        if (!good) break;
    }
    return good;
}

// After a timeout: the loader waits (each wait bounded) for its last copies and the MMA thread for
// its last MMAs, so that none is in flight when the CTA frees its tensor memory and exits.
__device__ __forceinline__ void split_quiesce(BatchSmem& bs, const SplitState& L, const SplitState& M, bool loader,
                                              uint32_t n_stages) {
    if (loader) {
        for (uint32_t j = 1; j <= n_stages && j <= L.tiles; ++j) {
            const uint32_t q = L.tiles - j;
            mbar_wait(saddr(&bs.full[q % n_stages]), (q / n_stages) & 1u);
        }
    } else if (M.accs > 0u) {
        mbar_wait(saddr(&bs.afull[(M.accs - 1u) & 1u]), ((M.accs - 1u) >> 1) & 1u);
    }
}

template <bool SMEM_STATE>
__global__ void __launch_bounds__(kBatchThreads, 1) bsnn_batch_kernel(const BSim* __restrict__ S, uint32_t n_steps) {
    extern __shared__ __align__(1024) unsigned char bsm_raw[];
    __shared__ BatchSmem bs;
    __shared__ BClass s_cls[kBatchMaxClasses];
    __shared__ int s_ok;
    __shared__ unsigned long long s_bar0, s_t0;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    if (tid == 0) s_wait_limit_ns = S->wait_limit_ns;  // read after the first __syncthreads below
    // stage s: A tile at s * stage_bytes, B tile after it; then the instance table (when it is
    // kept in shared memory), then the neuron state (when it is kept in shared memory)
    const uint32_t stage_bytes = S->stage_bytes, n_stages = S->n_stages;
    const uint32_t smem_base = saddr(bsm_raw);
    const BInst* P = batch_tables(S, bsm_raw + n_stages * stage_bytes, s_cls);
    const uint32_t n0 = min(blockIdx.x * S->per_cta, S->n_neurons);
    const uint32_t n1 = min(n0 + S->per_cta, S->n_neurons);
    BState X{};
    if constexpr (SMEM_STATE) {
        X = smem_state(bsm_raw + S->state_off, S->per_cta, 0u, n0);
        state_copy(S, X, n0, n1, true);
    } else {
        X = global_state(S);
    }

    if (tid == 0) {
        batch_init_barriers(bs, n_stages);
        s_bar0 = ld_acquire_u64(S->barrier) / gridDim.x * gridDim.x;
        s_t0 = *S->steps_done;
    }
    if (warp == 0) {
        tmem_alloc(saddr(&bs.tmem), kBatchTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = bs.tmem;
    const unsigned long long bar0 = s_bar0, t0 = s_t0;
    // phase B roles: thread 128 the loader, thread 256 the MMA thread, warps 0-3 the epilogue
    SplitState ls, ms, es;
    bool ok = true;
#ifdef BSNN_PHASE_TIMING
    __shared__ unsigned long long s_tally_[8];
    if (tid == 0)
        for (int i = 0; i < 8; ++i) s_tally_[i] = 0;
    unsigned long long t_mark_ = static_cast<unsigned long long>(clock64());
#endif

    uint16_t* s_nz = reinterpret_cast<uint16_t*>(bsm_raw + S->noise_off);
    if (S->noise_on) noise_ahead(S, P, s_cls, s_nz, n0, n1, t0, tid, blockDim.x);
    __syncthreads();

    // the size classes this CTA's neurons belong to (bit c)
    __shared__ uint32_t s_cmask;
    if (tid == 0) {
        uint32_t m = 0;
        for (uint32_t c = 0; c < S->n_classes; ++c)
            if (n0 < s_cls[c].nbase + s_cls[c].nlen && s_cls[c].nbase < n1) m |= 1u << c;
        s_cmask = m;
    }
    __syncthreads();
    const uint32_t cmask = s_cmask;
    const bool classwait = S->classwait != 0u;
    const unsigned long long ticket_end = (t0 + n_steps) * static_cast<unsigned long long>(S->n_units);
    if (classwait && tid == 128u) ls.held = atomicAdd(S->unit_ctr, 1ull);  // this CTA's first ticket
    for (uint32_t k = 0; k < n_steps && ok; ++k) {
        const unsigned long long t = t0 + k;
        if (classwait && t > 0) {
            // the previous step's units of this CTA's classes are all done (4 counts per unit)
            if (tid == 0) {
                int good = 1;
                for (uint32_t c = 0; c < S->n_classes && good; ++c)
                    if ((cmask >> c) & 1u) good = count_wait(S->udone + c, S->error, 4ull * t * S->units_of[c]) ? 1 : 0;
                s_ok = good;
            }
            __syncthreads();
            if (!s_ok) {
                ok = false;
                break;
            }
        }
        BSNN_TMARK(3);
        batch_neurons<SMEM_STATE>(S, P, s_cls, X, s_nz, n0, n1, t, tid, blockDim.x);
        fence_proxy_async_global();
        __syncthreads();
        BSNN_TMARK(0);
        if (classwait) {
            if (tid == 0)
                for (uint32_t c = 0; c < S->n_classes; ++c)
                    if ((cmask >> c) & 1u) red_release_add_u64(S->nready + c, 1ull);
        } else if (!grid_barrier(S->barrier, S->error, bar0 + (2ull * k + 1ull) * gridDim.x, &s_ok)) {
            ok = false;
            break;
        }
        BSNN_TMARK(1);
        if (tid == 128u) {
            fence_proxy_async_global();
            if (!split_loader(S, bs, s_cls, ls, t, smem_base, stage_bytes, n_stages, l2_evict_last_policy())) {
                atomicExch(S->error, kErrStageTimeout);
                bs.ok = 0u;
            }
        } else if (tid == 256u) {
            if (!split_mma(S, bs, s_cls, ms, tmem, smem_base, stage_bytes, n_stages)) {
                atomicExch(S->error, kErrStageTimeout);
                bs.ok = 0u;
            }
        } else if (warp < 4) {
            if (!split_epilogue(S, bs, s_cls, es, tmem, warp, lane)) {
                atomicExch(S->error, kErrStageTimeout);
                bs.ok = 0u;
            }
        } else if (noise_warp(warp) && S->noise_on && k + 1u < n_steps) {
            noise_ahead(S, P, s_cls, s_nz, n0, n1, t + 1ull, 32u * noise_rank(warp) + lane, 32u * kNoiseWarps);
        }
        __syncthreads();
        ok = bs.ok != 0u;  // the same for every thread of the CTA
        if (!ok) break;
        BSNN_TMARK(2);
        if (!classwait && !grid_barrier(S->barrier, S->error, bar0 + (2ull * k + 2ull) * gridDim.x, &s_ok)) {
            ok = false;
            break;
        }
    }
#ifdef BSNN_PHASE_TIMING
    if (tid == 0)
        for (int i = 0; i < 8; ++i) S->phase_ns[blockIdx.x * 8u + i] += s_tally_[i];
#endif
    if ((tid == 128u || tid == 256u) && bs.ok == 0u) split_quiesce(bs, ls, ms, tid == 128u, n_stages);
    // class waits: the ticket past the launch's end is given back, so the next launch starts at
    // (t0 + n_steps) * n_units
    if (classwait && tid == 128u && ls.held >= ticket_end) atomicAdd(S->unit_ctr, ~0ull);
    tc_fence_before();
    __syncthreads();
    if constexpr (SMEM_STATE) state_copy(S, X, n0, n1, false);
    if (warp == 0) tmem_dealloc(tmem, kBatchTmemCols);
    if (blockIdx.x == 0 && tid == 0 && ok) *S->steps_done = t0 + n_steps;
}

// ---- the flow form -------------------------------------------------------------------------------
// The same per-neuron arithmetic and the same GEMM units as bsnn_batch_kernel, without grid
// barriers.  Each size class is a chain of its own (its neurons of step t, then its GEMM units of
// step t, then its neurons of step t + 1, ...), and the chains of different classes overlap, as
// do the neuron updates and the GEMMs inside a CTA.  Two monotonically increasing counters per
// class in global memory carry the dependencies:
//   nready[c]: +1 when a CTA has stepped its slice of class c (every CTA, every step, an empty
//              slice too), so the class's neurons of step t are all done at (t + 1) * grid;
//   udone[c]:  +1 when an epilogue warp has written its 32 posts of a GEMM unit of class c, so
//              the class's propagation of step t is complete at 4 * (t + 1) * units_of[c].
// Roles in a CTA:
//   warps 5-15, the neuron side: per step, per class in processing order (the classes with the
//     most GEMM work first), draw the Poisson counts of the CTA's slice of the class, wait until
//     the class's propagation of the previous step is complete, step the slice (its state in
//     shared memory for the launch, as in the phased form), and count the slice in nready[c];
//   thread 128, the producer: takes GEMM units from one dispenser over all steps of the launch
//     (ticket q is unit q mod n_units of step q / n_units; units in class processing order,
//     longest first within a class), waits until every CTA has stepped the unit's class at that
//     step, then streams the operands and issues the MMAs as in the phased form;
//   warps 0-3, the epilogue: drain the accumulator, write the unit's partial sums, and count them
//     in udone[c].
// Every role takes its work in one order (step, then class processing order) and every wait is
// for work earlier in that order, so the earliest unfinished piece of work can always run: with
// all CTAs resident (a cooperative launch) the chains cannot deadlock.  The write-after-read
// hazards are covered by the same counters: a class's neurons of step t + 1 (which overwrite its
// x tiles and read its partial sums) wait for all its units of step t (which read those tiles and
// wrote those sums), and its units of step t + 1 (which overwrite the sums) wait for all its
// neurons of step t + 1.  The dispenser ends a launch at exactly (t0 + n_steps) * n_units: each
// producer's last take is past the end and is given back.
constexpr uint32_t kFlowNeuronWarp0 = 5;
constexpr uint32_t kFlowNeuronThreads = kBatchThreads - 32u * kFlowNeuronWarp0;

// Bounded wait for an mbarrier phase with an explicit limit.
__device__ __forceinline__ bool mbar_wait_for(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity))
        if (globaltimer_ns() - t0 > limit_ns) return false;
    return true;
}

template <bool SMEM_STATE>
__global__ void __launch_bounds__(kBatchThreads, 1) bsnn_batch_flow_kernel(const BSim* __restrict__ S, uint32_t n_steps) {
    extern __shared__ __align__(1024) unsigned char bsm_raw[];
    __shared__ BatchSmem bs;
    __shared__ BClass s_cls[kBatchMaxClasses];
    __shared__ uint32_t s_order[kBatchMaxClasses];
    __shared__ uint32_t s_slice[kBatchMaxClasses][3];  // per processing position: first neuron, end, state index
    __shared__ int s_nok;
    __shared__ unsigned long long s_t0;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t stage_bytes = S->stage_bytes, n_stages = S->n_stages, nc = S->n_classes;
    const uint32_t smem_base = saddr(bsm_raw);
    const BInst* P = batch_tables(S, bsm_raw + n_stages * stage_bytes, s_cls);
    unsigned char* state_raw = bsm_raw + S->state_off;
    uint16_t* s_nz = reinterpret_cast<uint16_t*>(bsm_raw + S->noise_off);
    if (tid == 0) {
        s_wait_limit_ns = S->wait_limit_ns;
        // the CTA's slice of each class: an even share of the class's contiguous neurons
        uint32_t soff = 0;
        for (uint32_t p = 0; p < nc; ++p) {
            const uint32_t c = S->order[p];
            const BClass& C = S->cls[c];
            const uint32_t a = C.nbase + static_cast<uint32_t>((static_cast<unsigned long long>(blockIdx.x) * C.nlen) / gridDim.x);
            const uint32_t e =
                C.nbase + static_cast<uint32_t>((static_cast<unsigned long long>(blockIdx.x + 1u) * C.nlen) / gridDim.x);
            s_order[p] = c;
            s_slice[p][0] = a;
            s_slice[p][1] = e;
            s_slice[p][2] = soff;
            soff += e - a;
        }
        batch_init_barriers(bs, n_stages);
        s_t0 = *S->steps_done;
        s_nok = 1;
    }
    if (warp == 0) {
        tmem_alloc(saddr(&bs.tmem), kBatchTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if constexpr (SMEM_STATE) {
        for (uint32_t p = 0; p < nc; ++p)
            state_copy(S, smem_state(state_raw, S->per_cta, s_slice[p][2], s_slice[p][0]), s_slice[p][0], s_slice[p][1], true);
    }
#ifdef BSNN_PHASE_TIMING
    __shared__ unsigned long long s_tally_[8];
    if (tid < 8) s_tally_[tid] = 0;
#endif
    __syncthreads();
    const uint32_t tmem = bs.tmem;
    const unsigned long long t0 = s_t0;
    const uint32_t n_units = S->n_units;

    if (tid == 128u) {
        // the producer
        ProducerState ps;
        uint32_t ready_slot = 0;
        const uint64_t keep = l2_evict_last_policy();
        const unsigned long long end = (t0 + n_steps) * n_units;
        for (;;) {
            BSNN_TSTART(t_take_);
            uint32_t ui = 0xFFFFFFFFu;
            unsigned long long tq = 0;
            if (bs.ok != 0u) {
                const unsigned long long q = atomicAdd(S->unit_ctr, 1ull);
                if (q >= end) {
                    atomicAdd(S->unit_ctr, ~0ull);  // the take past the launch's end is given back
                } else {
                    tq = q / n_units;
                    ui = static_cast<uint32_t>(q - tq * n_units);
                }
            }
            BSNN_TSPAN(6, t_take_);
            if (ui != 0xFFFFFFFFu) {
                BSNN_TSTART(t_wait_);
                // every CTA has stepped its slice of the unit's class at step tq
                if (!count_wait(S->nready + S->units[ui].cls, S->error, (tq + 1ull) * gridDim.x)) {
                    bs.ok = 0u;
                    ui = 0xFFFFFFFFu;
                }
                BSNN_TSPAN(4, t_wait_);
            }
            bs.unit[ready_slot] = ui;
            mbar_arrive(saddr(&bs.ready[ready_slot]));
            ready_slot ^= 1u;
            if (ui == 0xFFFFFFFFu) break;
            BSNN_TSTART(t_issue_);
            fence_proxy_async_global();  // x tiles written by generic stores, read by the bulk copies
            const BUnit U = S->units[ui];
            if (!issue_unit(bs, ps, U, s_cls[U.cls], tmem, smem_base, stage_bytes, n_stages, keep)) {
                atomicExch(S->error, kErrStageTimeout);
                bs.ok = 0u;
            }
            BSNN_TSPAN(5, t_issue_);
        }
        if (bs.ok == 0u) producer_quiesce(bs, ps, n_stages);
    } else if (warp < 4) {
        // the epilogue; its wait for the next unit spans the producer's wait for the unit's class,
        // so it is bounded by twice the limit
        uint32_t accum_ph = 0, ready_slot = 0, ready_ph = 0;
        for (;;) {
            // (made uniform over the warp before its warp-wide tensor-memory loads)
            if (!__all_sync(kFull, mbar_wait_for(saddr(&bs.ready[ready_slot]), (ready_ph >> ready_slot) & 1u,
                                                 2ull * s_wait_limit_ns))) {
                atomicExch(S->error, kErrStageTimeout);
                bs.ok = 0u;
                break;
            }
            ready_ph ^= 1u << ready_slot;
            const uint32_t ui = bs.unit[ready_slot];
            ready_slot ^= 1u;
            if (ui == 0xFFFFFFFFu) break;
            const BUnit U = S->units[ui];
            BSNN_TSTART(t_drain_);
            drain_unit(S, bs, U, s_cls[U.cls], tmem, accum_ph, warp, lane);
            // each epilogue warp counts its own 32 posts (no barrier across the warps, whose waits
            // may end differently after a timeout)
            if (lane == 0) red_release_add_u64(S->udone + U.cls, 1ull);
            if (tid == 0) BSNN_TSPAN(7, t_drain_);
        }
    } else if (warp >= kFlowNeuronWarp0) {
        // the neuron side
        const uint32_t me = tid - 32u * kFlowNeuronWarp0;
        bool nok = true;
        for (uint32_t k = 0; k < n_steps && nok; ++k) {
            const unsigned long long t = t0 + k;
            for (uint32_t p = 0; p < nc; ++p) {
                const uint32_t c = s_order[p];
                const uint32_t s0 = s_slice[p][0], s1 = s_slice[p][1], soff = s_slice[p][2];
                BSNN_TSTART(t_noise_);
                // the slice's Poisson counts of step t (they need no propagation: drawn while the
                // class's GEMM of the previous step may still run)
                if (S->noise_on) noise_ahead(S, P, s_cls, s_nz + soff, s0, s1, t, me, kFlowNeuronThreads);
                if (me == 0) {
                    BSNN_TSPAN(0, t_noise_);
                    BSNN_TSTART(t_wait_);
                    // the class's propagation of step t - 1 is complete (4 counts per unit)
                    s_nok = count_wait(S->udone + c, S->error, 4ull * t * S->units_of[c]) ? 1 : 0;
                    BSNN_TSPAN(1, t_wait_);
                }
                named_barrier_sync(2, kFlowNeuronThreads);
                if (s_nok == 0) {
                    nok = false;
                    break;
                }
                BSNN_TSTART(t_nrn_);
                BState X;
                if constexpr (SMEM_STATE) X = smem_state(state_raw, S->per_cta, soff, s0);
                else X = global_state(S);
                batch_neurons<SMEM_STATE>(S, P, s_cls, X, s_nz + soff, s0, s1, t, me, kFlowNeuronThreads);
                fence_proxy_async_global();
                named_barrier_sync(2, kFlowNeuronThreads);
                if (me == 0) {
                    red_release_add_u64(S->nready + c, 1ull);
                    BSNN_TSPAN(2, t_nrn_);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
#ifdef BSNN_PHASE_TIMING
    if (tid == 0)
        for (int i = 0; i < 8; ++i) S->phase_ns[blockIdx.x * 8u + i] += s_tally_[i];
#endif
    if constexpr (SMEM_STATE) {
        for (uint32_t p = 0; p < nc; ++p)
            state_copy(S, smem_state(state_raw, S->per_cta, s_slice[p][2], s_slice[p][0]), s_slice[p][0], s_slice[p][1], false);
    }
    if (warp == 0) tmem_dealloc(tmem, kBatchTmemCols);
    if (blockIdx.x == 0 && tid == 0 && ld_relaxed_s32(S->error) == kErrNone) *S->steps_done = t0 + n_steps;
}

// g of one instance's neurons: the background conductance (d - r) * scale of the background
// traces, plus, with `pending`, the propagation still pending in the partial sums (the value the
// reference holds after step_the_clock).  Reads only.  `instance` is the instance's position in the
// device's instance table.
__global__ void bsnn_batch_g_kernel(const BSim* __restrict__ S, uint32_t instance, int with_pending, float* out_ge,
                                    float* out_gi) {
    const BInst& B = S->inst[instance];
    const BClass& C = S->cls[B.cls];
    const bool pending = with_pending && *S->steps_done > 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < C.N; j += gridDim.x * blockDim.x) {
        const uint32_t n = B.nbase + j, mt = j >> 7, row = j & 127u;
        const BGroupP& G = B.g[j < C.E ? 0 : 1];
        float g[2] = {(S->ed[n] - S->er[n]) * G.bg_scale_e, (S->id[n] - S->ir[n]) * G.bg_scale_i};
        if (pending)
            for (uint32_t sd = 0; sd < 2; ++sd) {
                const float* p = S->partials + C.pbase[sd] + static_cast<size_t>(mt) * C.nkc[sd] * C.NP * 128u +
                                 static_cast<size_t>(B.row) * 128u + row;
                float dot = 0.0f;
                for (uint32_t kc = 0; kc < C.nkc[sd]; ++kc) dot += p[static_cast<size_t>(kc) * C.NP * 128u];
                g[sd] = g[sd] + dot;
            }
        out_ge[j] = g[0];
        out_gi[j] = g[1];
    }
}

}  // namespace bsnn
