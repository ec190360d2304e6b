// step_kernel.cuh -- the fused, persistent per-step kernel for sm_100a.
//
// One cooperative launch runs `n_steps` consecutive calls of System::step_the_clock
// (cpp_src/core/system.cpp:43-63) with ONE grid-wide barrier per step.  Each CTA owns a
// contiguous range of neurons; it updates them as neurons (phase A) and streams their outgoing
// weight rows as presynaptic rows (phase B):
//
//   phase A (own neurons): g = g_base + sum of the previous step's GEMV partials (fixed order)
//                           -> background Poisson shot noise      (kernel_neuron_group_evolve.cu:11-83)
//                           -> conductance-EIF Euler step, spike   (kernel_neuron_group_evolve.cu:85-130)
//                           -> stimulus events of this step        (kernel_stimulus_apply.cu:7-21)
//                           -> difference-of-exponentials traces   (kernel_connection_propagate.cu:8-46)
//                           -> plasticity trace decay/increment    (kernel_*_plasticity_update.cu)
//                           -> monitor ring buffers                (kernel_historicize_*.cu)
//   phase B (own rows):    the previous step's plasticity weight update (+ row normalisation),
//                           fused with this step's propagation GEMV (the cublasSgemv of
//                           kernel_connection_propagate.cu:79-94): each weight is read once,
//                           updated, written back and multiplied by x in the same pass; the
//                           CTA's per-column partial sums go to a parity buffer.
//   grid barrier
//
// Deferring step t's plasticity into step t+1's phase B is exact: between the two the
// reference touches the weights only to read them in step t+1's propagation, which phase B
// performs after the update.  At the end of a launch a finalize pass applies the pending
// plasticity and reduces the pending partials, so between launches the device state is the
// reference's state after step_the_clock.
#pragma once

#include <cuda_runtime.h>

#include "bsnn_device.cuh"

namespace bsnn {

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Philox4x32-10 (Salmon et al., SC'11): 10 rounds, published multipliers and Weyl constants.
__device__ __forceinline__ void philox4x32_10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0,
                                              uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Poisson count by Knuth's multiplication method over uniforms u = ((r >> 8) + 1) * 2^-24 in
// (0, 1].  Counter (neuron, step lo, step hi, channel << 16 | block), key (seed, 0); saturates at
// 255, which also bounds the loop (at most 64 Philox blocks).
__device__ __forceinline__ uint32_t poisson_knuth(float exp_neg_mean, uint32_t seed, uint32_t neuron,
                                                  unsigned long long step, uint32_t channel) {
    float p = 1.0f;
    uint32_t k = 0;
    for (uint32_t block = 0; block < 64u; ++block) {
        uint32_t c0 = neuron, c1 = static_cast<uint32_t>(step), c2 = static_cast<uint32_t>(step >> 32),
                 c3 = (channel << 16) | block;
        philox4x32_10(c0, c1, c2, c3, seed, 0u);
        const uint32_t r[4] = {c0, c1, c2, c3};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float u = __fmul_rn(__uint2float_rn((r[i] >> 8) + 1u), 5.9604644775390625e-8f);
            p = __fmul_rn(p, u);
            if (p <= exp_neg_mean) return k;
            if (++k >= 255u) return 255u;
        }
    }
    return k;
}

__device__ __forceinline__ float flush_tiny(float t) { return t < 1e-30f ? 0.0f : t; }

__device__ __forceinline__ float clamp_w(float w, float wmin, float wmax) {
    if (w < wmin) return wmin;
    if (w > wmax) return wmax;
    return w;
}

// Grid-wide barrier over the persistent CTAs: monotonically increasing 64-bit arrival counter,
// release/acquire at gpu scope.  Bounded: after kBarrierTimeoutNs (or when another CTA has
// already given up) it records kErrBarrierTimeout and returns false so the kernel can exit.
__device__ __forceinline__ bool grid_barrier(const DSim* S, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        const unsigned long long n = gridDim.x;
        const unsigned long long old = atomicAdd(S->barrier, 1ull);
        const unsigned long long target = (old / n + 1ull) * n;
        unsigned long long t_start = 0;
        uint32_t spins = 0;
        while (static_cast<long long>(ld_acquire_u64(S->barrier) - target) < 0) {
            if ((++spins & 255u) == 0u) {
                const unsigned long long now = globaltimer_ns();
                if (t_start == 0) {
                    t_start = now;
                } else if (now - t_start > kBarrierTimeoutNs) {
                    atomicExch(S->error, kErrBarrierTimeout);
                    ok = 0;
                    break;
                }
                if (ld_relaxed_s32(S->error) != kErrNone) {
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

struct SmemLayout {
    DRowMeta* meta;     // [max_rows]
    float4* row;        // [max_rows] {x, rowA, rowB, scale}
    uint32_t* rowflag;  // [max_rows] bit0: presynaptic neuron spiked at the step being applied
    float* part;        // [kMaxWarps][max_rows] per-warp row sums for the normalisation
    float* dot;         // [2][max_own]
    uint32_t* bits;     // [n_spike_monitors][max_own/32 + 2]
};

__device__ __forceinline__ int group_of(const uint32_t* s_goff, const uint32_t* s_gn, uint32_t n_groups, uint32_t j) {
    for (uint32_t g = 0; g < n_groups; ++g)
        if (j - s_goff[g] < s_gn[g]) return static_cast<int>(g);
    return -1;
}

// Phase A1 / finalize: dot[T][i] = sum over the slots listed for (T, group of neuron n0+i) of the
// parity-`par` partial sums at that neuron's column.  Warp per (neuron, target), lanes stride the
// slot list, xor-butterfly: a fixed summation order.
__device__ __forceinline__ void reduce_partials(const DSim* S, const DCta& cta, uint32_t par, const SmemLayout& sm,
                                                uint32_t max_own, const uint32_t* s_goff, const uint32_t* s_gn) {
    const uint32_t n_own = cta.n1 - cta.n0;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nwarps = blockDim.x >> 5;
    const float* part = S->partials + static_cast<size_t>(par) * S->n_slots * S->N_pad;
    for (uint32_t pr = warp; pr < 2u * n_own; pr += nwarps) {
        const uint32_t i = pr >> 1, T = pr & 1u, j = cta.n0 + i;
        const int g = group_of(s_goff, s_gn, S->n_groups, j);
        float s = 0.0f;
        if (g >= 0) {
            const uint32_t b = S->red_begin[T][g], e = S->red_end[T][g];
            const uint32_t col = S->groups[g].pcol + (j - s_goff[g]);
            for (uint32_t k = b + lane; k < e; k += 32u)
                s += __ldcg(part + static_cast<size_t>(S->red_list[k]) * S->N_pad + col);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
        if (lane == 0) sm.dot[T * max_own + i] = s;
    }
}

// Phase A2: one thread per owned neuron.
__device__ __forceinline__ void neuron_phase(const DSim* S, const DCta& cta, unsigned long long t, uint32_t clock,
                                             uint32_t par, bool has_dot, const SmemLayout& sm, uint32_t max_own,
                                             const uint32_t* s_goff, const uint32_t* s_gn, const uint32_t* s_bitbase) {
    const uint32_t i = threadIdx.x;
    if (i >= cta.n1 - cta.n0) return;
    const uint32_t j = cta.n0 + i;
    const int g = group_of(s_goff, s_gn, S->n_groups, j);
    if (g < 0) return;
    const DGroup& G = S->groups[g];
    const uint32_t loc = j - G.off;

    // Conductances seen by this step's evolve: background of the previous step plus the
    // previous step's propagation (cublasSgemv y = A x + y, kernel_connection_propagate.cu:79-94).
    float ge_used = S->ge[j], gi_used = S->gi[j];
    if (has_dot) {
        ge_used = ge_used + sm.dot[i];
        gi_used = gi_used + sm.dot[max_own + i];
    }

    // kernel_update_background_conductances (kernel_neuron_group_evolve.cu:11-83)
    float er = flush_tiny(S->bg_er[j] * G.bg_er_decay);
    float ir = flush_tiny(S->bg_ir[j] * G.bg_ir_decay);
    float ed = flush_tiny(S->bg_ed[j] * G.bg_ed_decay);
    float id = flush_tiny(S->bg_id[j] * G.bg_id_decay);
    uint32_t ne = 0, ni = 0;
    if (S->noise_mode == kNoisePhilox) {
        if (G.has_bg_e) ne = poisson_knuth(G.exp_neg_mean_e, S->seed, j, t, 0u);
        if (G.has_bg_i) ni = poisson_knuth(G.exp_neg_mean_i, S->seed, j, t, 1u);
    } else if (S->noise_mode == kNoiseReplay && t < S->replay_steps) {
        const size_t base = (static_cast<size_t>(t) * S->N + j) * 2u;
        ne = S->replay[base];
        ni = S->replay[base + 1];
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
    S->bg_er[j] = er;
    S->bg_ed[j] = ed;
    S->bg_ir[j] = ir;
    S->bg_id[j] = id;
    S->bg_ge[j] = bg_ge;
    S->bg_gi[j] = bg_gi;

    // kernel_neuron_group_evolve (kernel_neuron_group_evolve.cu:85-130)
    float istim = S->istim[j];
    uint32_t spike = 0;
    float v = S->v[j];
    uint32_t refrac = S->refrac[j];
    if (refrac > 0) {
        --refrac;
        v = G.v_reset;
    } else {
        const float linear_leak_term = -1.0f * G.g_leak * (v - G.v_rest);
        const float exponential_depolarization_term =
            G.g_leak * G.delta_t * expf((v - G.v_eff) / G.delta_t);
        const float excitatory_synaptic_term = -1.0f * ge_used * (v - G.e_exc);
        const float inhibitory_synaptic_term = -1.0f * gi_used * (v - G.e_inh);
        const float dv = (G.timestep / G.cap) * (linear_leak_term + exponential_depolarization_term +
                                                 excitatory_synaptic_term + inhibitory_synaptic_term + istim);
        const float v_next = v + dv;
        if (v_next >= G.v_th) {
            refrac = G.refractory_steps;
            spike = 1;
            v = G.v_th;
        } else {
            v = v_next;
        }
    }
    S->v[j] = v;
    S->refrac[j] = refrac;
    S->ge[j] = bg_ge;  // reset for the next propagation (kernel_neuron_group_evolve.cu:126-129)
    S->gi[j] = bg_gi;
    S->spikes[par][j] = spike;

    // Stimulus::apply / kernel_stimulus_apply (stimulus.cpp:46-60, kernel_stimulus_apply.cu:7-21):
    // events of this step land after the evolve read i_stimulus, so they act from the next step.
    if (t < S->stim_len) {
        uint32_t lo = S->stim_off[t], hi = S->stim_off[t + 1];
        while (lo < hi) {  // lower_bound of j in the step's events (sorted by neuron)
            const uint32_t mid = (lo + hi) >> 1;
            if (S->ev_neuron[mid] < j) lo = mid + 1;
            else hi = mid;
        }
        const uint32_t end = S->stim_off[t + 1];
        bool any = false;
        for (uint32_t k = lo; k < end && S->ev_neuron[k] == j; ++k) {
            istim = istim + S->ev_delta[k];
            any = true;
        }
        if (any) S->istim[j] = istim;
    }

    // Connection traces (kernel_connection_propagate.cu:8-46): decay d, decay r, +norm on spike.
    for (uint32_t k = 0; k < G.n_ts; ++k) {
        const DTraceSet& TS = S->ts[G.ts[k]];
        float d = flush_tiny(TS.d[loc] * TS.d_decay);
        float r = flush_tiny(TS.r[loc] * TS.r_decay);
        if (spike == 1) {
            r += TS.norm;
            d += TS.norm;
        }
        TS.r[loc] = r;
        TS.d[loc] = d;
        TS.x[loc] = d - r;
    }

    // Plasticity traces as presynaptic neuron: decay (the value the weight update uses), row
    // factors for that update, then the spike increment (kernel_*_plasticity_update.cu).
    for (uint32_t k = 0; k < G.n_plast_pre; ++k) {
        const DPlast& P = S->plast[G.plast_pre[k]];
        const float pre = flush_tiny(P.pre[loc] * P.pre_decay);
        float rowA, rowB;
        if (P.kind == kKindTriplet) {
            const float tpre = flush_tiny(P.tpre[loc] * P.tpre_decay);
            rowA = pre;
            rowB = P.ltd_A + (P.ltd_B * tpre);
            P.tpre[loc] = spike == 1 ? tpre + 1.0f : tpre;
        } else {
            rowA = pre;
            rowB = -1.0f * P.ltd_A;
        }
        P.rowA[par][loc] = rowA;
        P.rowB[par][loc] = rowB;
        P.pre[loc] = spike == 1 ? pre + 1.0f : pre;
    }
    // ... and as postsynaptic neuron: column factors.
    for (uint32_t k = 0; k < G.n_plast_post; ++k) {
        const DPlast& P = S->plast[G.plast_post[k]];
        const float post = flush_tiny(P.post[loc] * P.post_decay);
        float colA, colB;
        if (P.kind == kKindTriplet) {
            const float tpost = flush_tiny(P.tpost[loc] * P.tpost_decay);
            colA = P.ltp_A + (P.ltp_B * tpost);
            colB = -1.0f * post;
            P.tpost[loc] = spike == 1 ? tpost + 1.0f : tpost;
        } else if (P.kind == kKindIstdp) {
            colA = P.ltp_A;
            colB = post - P.ltd_B;
        } else {
            colA = P.ltp_A;
            colB = post;
        }
        P.colA[par][loc] = colA;
        P.colB[par][loc] = colB;
        P.pspk[par][loc] = spike;
        P.post[loc] = spike == 1 ? post + 1.0f : post;
    }

    // Monitors (kernel_historicize_spikes.cu:7-21, kernel_historicize_membrane_potentials.cu:7-21).
    for (uint32_t k = 0; k < G.n_mon; ++k) {
        const int m = G.mon[k];
        const DMon& M = S->mons[m];
        if (M.kind == kMonSpikes) {
            if (spike) {
                const uint32_t w0 = (cta.n0 > G.off ? cta.n0 - G.off : 0u) >> 5;
                atomicOr(&sm.bits[s_bitbase[m] + ((loc >> 5) - w0)], 1u << (loc & 31u));
            }
        } else {
            const int32_t col = M.sel_idx[loc];
            if (col >= 0) M.vh[static_cast<size_t>(clock % M.interval) * M.n_sel + col] = v;
        }
    }
}

// Writes this CTA's spike bits of each spike monitor into the ring slot of `clock`.  Each CTA
// clears and sets only the bits of its own neurons, so the word updates of different CTAs commute.
__device__ __forceinline__ void flush_spike_bits(const DSim* S, const DCta& cta, uint32_t clock,
                                                 const SmemLayout& sm, const uint32_t* s_bitbase) {
    for (uint32_t m = 0; m < S->n_mons; ++m) {
        const DMon& M = S->mons[m];
        if (M.kind != kMonSpikes) continue;
        const DGroup& G = S->groups[M.group];
        const uint32_t a = cta.n0 > G.off ? cta.n0 - G.off : 0u;
        const uint32_t b_end = cta.n1 - G.off < G.n ? cta.n1 - G.off : G.n;
        if (cta.n1 <= G.off || a >= b_end) continue;
        const uint32_t w0 = a >> 5, w1 = (b_end - 1) >> 5;
        for (uint32_t w = w0 + threadIdx.x; w <= w1; w += blockDim.x) {
            const uint32_t lo = w == w0 ? (a & 31u) : 0u;
            const uint32_t hi = w == w1 ? ((b_end - 1) & 31u) : 31u;
            const uint32_t mask = (hi == 31u ? 0xffffffffu : ((1u << (hi + 1u)) - 1u)) & ~((1u << lo) - 1u);
            const uint32_t bits = sm.bits[s_bitbase[m] + (w - w0)] & mask;
            uint32_t* word = M.bits + static_cast<size_t>(clock % M.interval) * M.words + w;
            const uint32_t clear = mask & ~bits;
            if (clear) atomicAnd(word, ~clear);
            if (bits) atomicOr(word, bits);
        }
    }
}

// Per-row data for phase B: x of this step, and the pending plasticity's row factors.
__device__ __forceinline__ void build_rows(const DSim* S, const DCta& cta, bool pending, uint32_t ppar,
                                           const SmemLayout& sm, bool with_x) {
    for (uint32_t r = threadIdx.x; r < cta.n_rows; r += blockDim.x) {
        const DRowMeta meta = sm.meta[r];
        const DConn& C = S->conns[meta.conn];
        float4 row = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        uint32_t flag = 0;
        if (with_x) row.x = __ldcg(S->ts[C.ts].x + meta.pl);
        if (pending && C.plast >= 0) {
            const DPlast& P = S->plast[C.plast];
            row.y = __ldcg(P.rowA[ppar] + meta.pl);
            row.z = __ldcg(P.rowB[ppar] + meta.pl);
            flag = __ldcg(S->spikes[ppar] + meta.j) == 1u ? 1u : 0u;
        }
        sm.row[r] = row;
        sm.rowflag[r] = flag;
    }
}

__device__ __forceinline__ float4 ld_col4(const float* p) { return __ldcg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ uint4 ld_col4u(const uint32_t* p) { return __ldcg(reinterpret_cast<const uint4*>(p)); }

// The reference's per-element plasticity sequence: LTP clamp (if post spiked), then LTD clamp
// (if pre spiked), skipping the diagonal of group-local indices.
__device__ __forceinline__ float plastic_update(float w, uint32_t q, uint32_t pl, uint32_t n_post, uint32_t post_spk,
                                                uint32_t pre_spk, float rowA, float colA, float colB, float rowB,
                                                float wmin, float wmax) {
    if (q >= n_post || q == pl) return w;
    if (post_spk) w = clamp_w(fmaf(rowA, colA, w), wmin, wmax);
    if (pre_spk) w = clamp_w(fmaf(colB, rowB, w), wmin, wmax);
    return w;
}

__device__ __forceinline__ int seg_of_item(const DSeg* s_seg, uint32_t n_seg, uint32_t it) {
    for (uint32_t s = 0; s < n_seg; ++s) {
        const uint32_t b = s_seg[s].item_begin;
        if (it >= b && it < b + ((s_seg[s].units + 31u) & ~31u)) return static_cast<int>(s);
    }
    return -1;
}

// Pass 1 of the triplet normalisation: each warp sums, per normalised row, the updated weights
// of its 32 units into its own slot sm.part[warp][row] (no atomics; fixed order).
__device__ __forceinline__ void norm_pass1(const DSim* S, const DCta& cta, uint32_t ppar, const SmemLayout& sm,
                                           const DSeg* s_seg, const DBlk* s_blk, uint32_t n_seg, uint32_t max_rows) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t r = threadIdx.x; r < cta.n_rows; r += blockDim.x)
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) sm.part[w * max_rows + r] = 0.0f;
    __syncthreads();
    for (uint32_t it0 = 0; it0 < cta.n_items; it0 += blockDim.x) {
        const uint32_t it = it0 + threadIdx.x;
        const int s = seg_of_item(s_seg, n_seg, it - lane);  // warp-uniform
        if (s < 0 || !s_seg[s].normalized) continue;
        const DSeg& SG = s_seg[s];
        const uint32_t u = it - SG.item_begin;
        const bool valid = u < SG.units;
        for (uint32_t bk = SG.blk_begin; bk < SG.blk_end; ++bk) {
            const DBlk& B = s_blk[bk];
            const DConn& C = S->conns[B.conn];
            if (C.plast < 0 || S->plast[C.plast].kind != kKindTriplet) continue;
            const DPlast& P = S->plast[C.plast];
            float4 cA = make_float4(0.f, 0.f, 0.f, 0.f), cB = cA;
            uint4 ps = make_uint4(0u, 0u, 0u, 0u);
            if (valid) {
                cA = ld_col4(P.colA[ppar] + 4u * u);
                cB = ld_col4(P.colB[ppar] + 4u * u);
                ps = ld_col4u(P.pspk[ppar] + 4u * u);
            }
            const float* wrow = C.w + 4u * u;
            for (uint32_t pl = B.row_begin, r = B.srow; pl < B.row_end; ++pl, ++r) {
                float sum = 0.0f;
                if (valid) {
                    const float4 rw = sm.row[r];
                    const uint32_t pre_spk = sm.rowflag[r];
                    float4 w4 = *reinterpret_cast<const float4*>(wrow + static_cast<size_t>(pl) * C.ld);
                    const uint32_t q = 4u * u;
                    w4.x = plastic_update(w4.x, q + 0u, pl, C.n_post, ps.x, pre_spk, rw.y, cA.x, cB.x, rw.z, P.wmin, P.wmax);
                    w4.y = plastic_update(w4.y, q + 1u, pl, C.n_post, ps.y, pre_spk, rw.y, cA.y, cB.y, rw.z, P.wmin, P.wmax);
                    w4.z = plastic_update(w4.z, q + 2u, pl, C.n_post, ps.z, pre_spk, rw.y, cA.z, cB.z, rw.z, P.wmin, P.wmax);
                    w4.w = plastic_update(w4.w, q + 3u, pl, C.n_post, ps.w, pre_spk, rw.y, cA.w, cB.w, rw.z, P.wmin, P.wmax);
                    sum = (w4.x + w4.y) + (w4.z + w4.w);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
                if (lane == 0) sm.part[warp * max_rows + r] += sum;
            }
        }
    }
    __syncthreads();
    // Row scale = target / current sum; rows with sum <= 0 are left unscaled (scale 1 is exact).
    for (uint32_t s = 0; s < n_seg; ++s) {
        if (!s_seg[s].normalized) continue;
        for (uint32_t bk = s_seg[s].blk_begin; bk < s_seg[s].blk_end; ++bk) {
            const DBlk& B = s_blk[bk];
            const DConn& C = S->conns[B.conn];
            if (C.plast < 0 || S->plast[C.plast].kind != kKindTriplet) continue;
            const DPlast& P = S->plast[C.plast];
            for (uint32_t pl = B.row_begin + threadIdx.x; pl < B.row_end; pl += blockDim.x) {
                const uint32_t r = B.srow + (pl - B.row_begin);
                float sum = 0.0f;
                for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) sum += sm.part[w * max_rows + r];
                const float scale = sum <= 0.0f ? 1.0f : __fdiv_rn(P.sums[pl], sum);
                sm.row[r].w = scale;
            }
        }
    }
    __syncthreads();
}

// Pass 2: update + normalise + store the pending plasticity, and (if `accumulate`) the GEMV
// partial sums of this step, written to the parity-`par` partial slots.
__device__ __forceinline__ void weight_pass(const DSim* S, const DCta& cta, bool pending, uint32_t ppar,
                                            bool accumulate, uint32_t par, const SmemLayout& sm, const DSeg* s_seg,
                                            const DBlk* s_blk, uint32_t n_seg) {
    float* part_out = S->partials + static_cast<size_t>(par) * S->n_slots * S->N_pad;
    for (uint32_t it0 = 0; it0 < cta.n_items; it0 += blockDim.x) {
        const uint32_t it = it0 + threadIdx.x;
        const int s = seg_of_item(s_seg, n_seg, it);
        if (s < 0) continue;
        const DSeg& SG = s_seg[s];
        const uint32_t u = it - SG.item_begin;
        if (u >= SG.units) continue;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        bool touched = false;
        for (uint32_t bk = SG.blk_begin; bk < SG.blk_end; ++bk) {
            const DBlk& B = s_blk[bk];
            const DConn& C = S->conns[B.conn];
            const bool plastic = pending && C.plast >= 0;
            if (!plastic && !accumulate) continue;
            touched = true;
            float* wrow = C.w + 4u * u;
            if (plastic) {
                const DPlast& P = S->plast[C.plast];
                const float4 cA = ld_col4(P.colA[ppar] + 4u * u);
                const float4 cB = ld_col4(P.colB[ppar] + 4u * u);
                const uint4 ps = ld_col4u(P.pspk[ppar] + 4u * u);
                const uint32_t q = 4u * u;
                for (uint32_t pl = B.row_begin, r = B.srow; pl < B.row_end; ++pl, ++r) {
                    const float4 rw = sm.row[r];
                    const uint32_t pre_spk = sm.rowflag[r];
                    float4* wp = reinterpret_cast<float4*>(wrow + static_cast<size_t>(pl) * C.ld);
                    float4 w4 = *wp;
                    w4.x = plastic_update(w4.x, q + 0u, pl, C.n_post, ps.x, pre_spk, rw.y, cA.x, cB.x, rw.z, P.wmin, P.wmax) * rw.w;
                    w4.y = plastic_update(w4.y, q + 1u, pl, C.n_post, ps.y, pre_spk, rw.y, cA.y, cB.y, rw.z, P.wmin, P.wmax) * rw.w;
                    w4.z = plastic_update(w4.z, q + 2u, pl, C.n_post, ps.z, pre_spk, rw.y, cA.z, cB.z, rw.z, P.wmin, P.wmax) * rw.w;
                    w4.w = plastic_update(w4.w, q + 3u, pl, C.n_post, ps.w, pre_spk, rw.y, cA.w, cB.w, rw.z, P.wmin, P.wmax) * rw.w;
                    *wp = w4;
                    if (accumulate) {
                        acc.x = fmaf(w4.x, rw.x, acc.x);
                        acc.y = fmaf(w4.y, rw.x, acc.y);
                        acc.z = fmaf(w4.z, rw.x, acc.z);
                        acc.w = fmaf(w4.w, rw.x, acc.w);
                    }
                }
            } else {
                for (uint32_t pl = B.row_begin, r = B.srow; pl < B.row_end; ++pl, ++r) {
                    const float x = sm.row[r].x;
                    const float4 w4 = *reinterpret_cast<const float4*>(wrow + static_cast<size_t>(pl) * C.ld);
                    acc.x = fmaf(w4.x, x, acc.x);
                    acc.y = fmaf(w4.y, x, acc.y);
                    acc.z = fmaf(w4.z, x, acc.z);
                    acc.w = fmaf(w4.w, x, acc.w);
                }
            }
        }
        if (accumulate && touched)
            *reinterpret_cast<float4*>(part_out + static_cast<size_t>(SG.slot) * S->N_pad + SG.pcol + 4u * u) = acc;
    }
}

__global__ void __launch_bounds__(kMaxThreads, 1) bsnn_step_kernel(const DSim* __restrict__ S, uint32_t n_steps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ DCta s_cta;
    __shared__ DSeg s_seg[kMaxSegsPerCta];
    __shared__ DBlk s_blk[kMaxBlksPerCta];
    __shared__ uint32_t s_goff[kMaxGroups], s_gn[kMaxGroups];
    __shared__ uint32_t s_bitbase[kMaxMonitors];
    __shared__ unsigned long long s_t0;
    __shared__ uint32_t s_clock0;
    __shared__ int s_ok;
    __shared__ uint32_t s_has_norm;
    __shared__ uint32_t s_blk_base, s_nblk;

    const uint32_t max_rows = S->max_rows, max_own = S->max_own;
    SmemLayout sm;
    {
        unsigned char* p = smem_raw;
        sm.row = reinterpret_cast<float4*>(p);
        p += sizeof(float4) * max_rows;
        sm.meta = reinterpret_cast<DRowMeta*>(p);
        p += sizeof(DRowMeta) * max_rows;
        sm.rowflag = reinterpret_cast<uint32_t*>(p);
        p += sizeof(uint32_t) * max_rows;
        sm.part = reinterpret_cast<float*>(p);
        p += sizeof(float) * kMaxWarps * max_rows;
        sm.dot = reinterpret_cast<float*>(p);
        p += sizeof(float) * 2 * max_own;
        sm.bits = reinterpret_cast<uint32_t*>(p);
    }

    if (threadIdx.x == 0) {
        s_cta = S->ctas[blockIdx.x];
        s_t0 = *S->steps_done;
        s_clock0 = *S->clock;
        uint32_t base = 0, has_norm = 0;
        for (uint32_t m = 0; m < S->n_mons; ++m) {
            s_bitbase[m] = base;
            if (S->mons[m].kind == kMonSpikes) base += max_own / 32u + 2u;
        }
        for (uint32_t g = 0; g < S->n_groups; ++g) {
            s_goff[g] = S->groups[g].off;
            s_gn[g] = S->groups[g].n;
        }
        // Segments index the global block list; rebase them onto this CTA's copy in s_blk.
        const uint32_t blk_base = s_cta.seg_end > s_cta.seg_begin ? S->segs[s_cta.seg_begin].blk_begin : 0u;
        uint32_t nblk = 0;
        for (uint32_t s = s_cta.seg_begin; s < s_cta.seg_end; ++s) {
            DSeg sg = S->segs[s];
            sg.blk_begin -= blk_base;
            sg.blk_end -= blk_base;
            nblk = sg.blk_end > nblk ? sg.blk_end : nblk;
            s_seg[s - s_cta.seg_begin] = sg;
            has_norm |= sg.normalized;
        }
        s_has_norm = has_norm;
        s_blk_base = blk_base;
        s_nblk = nblk;
    }
    __syncthreads();
    const DCta cta = s_cta;
    const uint32_t n_seg = cta.seg_end - cta.seg_begin;
    for (uint32_t b = threadIdx.x; b < s_nblk; b += blockDim.x) s_blk[b] = S->blks[s_blk_base + b];
    {
        const DRowMeta* rows = S->rows + S->rows_begin[blockIdx.x];
        for (uint32_t r = threadIdx.x; r < cta.n_rows; r += blockDim.x) sm.meta[r] = rows[r];
    }
    uint32_t n_bits_words = 0;
    for (uint32_t m = 0; m < S->n_mons; ++m)
        if (S->mons[m].kind == kMonSpikes) n_bits_words += max_own / 32u + 2u;
    __syncthreads();

    const unsigned long long t0 = s_t0;
    const uint32_t clock0 = s_clock0;
    bool ok = true;
    for (uint32_t k = 0; k < n_steps; ++k) {
        const unsigned long long t = t0 + k;
        const uint32_t clock = clock0 + k;
        const uint32_t par = static_cast<uint32_t>(t & 1ull), ppar = par ^ 1u;
        const bool pending = k > 0;  // the previous step's plasticity and partials are outstanding

        if (pending) reduce_partials(S, cta, ppar, sm, max_own, s_goff, s_gn);
        for (uint32_t w = threadIdx.x; w < n_bits_words; w += blockDim.x) sm.bits[w] = 0u;
        __syncthreads();
        neuron_phase(S, cta, t, clock, par, pending, sm, max_own, s_goff, s_gn, s_bitbase);
        __syncthreads();
        flush_spike_bits(S, cta, clock, sm, s_bitbase);
        build_rows(S, cta, pending, ppar, sm, true);
        __syncthreads();
        if (pending && s_has_norm) norm_pass1(S, cta, ppar, sm, s_seg, s_blk, n_seg, max_rows);
        weight_pass(S, cta, pending, ppar, true, par, sm, s_seg, s_blk, n_seg);
        if (!grid_barrier(S, &s_ok)) {
            ok = false;
            break;
        }
    }
    if (!ok) return;

    // Finalize: apply the last step's plasticity and fold its propagation into g.
    const unsigned long long t_last = t0 + n_steps - 1ull;
    const uint32_t lpar = static_cast<uint32_t>(t_last & 1ull);
    build_rows(S, cta, true, lpar, sm, false);
    __syncthreads();
    if (s_has_norm) norm_pass1(S, cta, lpar, sm, s_seg, s_blk, n_seg, max_rows);
    weight_pass(S, cta, true, lpar, false, lpar, sm, s_seg, s_blk, n_seg);
    reduce_partials(S, cta, lpar, sm, max_own, s_goff, s_gn);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < cta.n1 - cta.n0; i += blockDim.x) {
        const uint32_t j = cta.n0 + i;
        if (group_of(s_goff, s_gn, S->n_groups, j) < 0) continue;
        S->ge[j] = S->ge[j] + sm.dot[i];
        S->gi[j] = S->gi[j] + sm.dot[max_own + i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *S->steps_done = t0 + n_steps;
        *S->clock = clock0 + n_steps;
    }
}

// Sets the clock_step of the next step (bsnn_run with a first_clock_step that does not follow
// the previous call).
__global__ void bsnn_set_clock_kernel(uint32_t* clock, uint32_t value) { *clock = value; }

}  // namespace bsnn
