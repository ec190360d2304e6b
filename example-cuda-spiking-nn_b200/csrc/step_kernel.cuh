// step_kernel.cuh -- the fused, persistent per-step kernel for sm_100a.
//
// One cooperative launch runs `n_steps` consecutive calls of System::step_the_clock
// (cpp_src/core/system.cpp:43-63) with ONE grid-wide barrier per step.  Each CTA owns a
// contiguous range of neurons; it updates them as neurons (phase A) and streams their outgoing
// weight rows as presynaptic rows (phase B).  The own neurons' state stays in shared memory for
// the whole launch; global memory carries only what other CTAs read (GEMV partial sums, the
// spike bitmask, plasticity column factors) and the monitor rings.
//
//   inputs (one batch of loads): the previous step's GEMV partials of the own neurons, the
//                           network spike bitmask of the previous step, the step's stimulus range
//   phase A (own neurons): g = g_base + sum of the previous step's GEMV partials (fixed order)
//                           -> background Poisson shot noise      (kernel_neuron_group_evolve.cu:11-83)
//                           -> conductance-EIF Euler step, spike   (kernel_neuron_group_evolve.cu:85-130)
//                           -> stimulus events of this step        (kernel_stimulus_apply.cu:7-21)
//                           -> difference-of-exponentials traces   (kernel_connection_propagate.cu:8-46)
//                           -> plasticity trace decay/increment    (kernel_*_plasticity_update.cu)
//                           -> monitor ring buffers                (kernel_historicize_*.cu)
//                           while the remaining warps compute the triplet row-normalisation sums
//                           of the previous step's update
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
// plasticity, reduces the pending partials and writes the neuron state back, so between
// launches the device state is the reference's state after step_the_clock.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include "bsnn_device.cuh"

namespace bsnn {

// Every device-side wait (the grid barrier, the staging mbarriers) gives up after the launch's wait
// limit, a DSim field the host sets (2 s unless bsnn_set_device_wait_limit changed it).  Each
// kernel that waits copies it into this shared variable before its first wait.
constexpr unsigned long long kDefaultWaitLimitNs = 2000000000ull;  // 2 s
__shared__ unsigned long long s_wait_limit_ns;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kRowBatch = 4;     // rows whose weights one thread loads before using them (plastic rows)
constexpr int kStreamBatch = 4;  // same for read-only rows

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

// Knuth's method continued from Philox block `block` with the running product p and count k (the
// tail of poisson_knuth).
__device__ __forceinline__ uint32_t poisson_knuth_from(float exp_neg_mean, uint32_t seed, uint32_t neuron,
                                                       unsigned long long step, uint32_t channel, uint32_t block,
                                                       float p, uint32_t k) {
    for (; block < 64u; ++block) {
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

// Both background channels of one neuron (channel 0: excitatory, channel 1: inhibitory; a channel
// that is off counts 0): the same counts as two poisson_knuth calls.  The first Philox block of
// the two channels is computed together, two independent chains the scheduler interleaves; the
// rarer later blocks follow per channel.
__device__ __forceinline__ void poisson_knuth_pair(float em0, bool on0, float em1, bool on1, uint32_t seed,
                                                   uint32_t neuron, unsigned long long step, uint32_t& n0,
                                                   uint32_t& n1) {
    uint32_t a0 = neuron, a1 = static_cast<uint32_t>(step), a2 = static_cast<uint32_t>(step >> 32), a3 = 0u;
    uint32_t b0 = neuron, b1 = a1, b2 = a2, b3 = 1u << 16;
    philox4x32_10(a0, a1, a2, a3, seed, 0u);
    philox4x32_10(b0, b1, b2, b3, seed, 0u);
    const uint32_t ra[4] = {a0, a1, a2, a3}, rb[4] = {b0, b1, b2, b3};
    // channel c from its first block: done (count) or the running product and count after 4 uniforms
    auto first = [&](const uint32_t* r, float em, uint32_t& out) -> bool {
        float p = 1.0f;
        uint32_t k = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float u = __fmul_rn(__uint2float_rn((r[i] >> 8) + 1u), 5.9604644775390625e-8f);
            p = __fmul_rn(p, u);
            if (p <= em) {
                out = k;
                return true;
            }
            ++k;
        }
        out = __float_as_uint(p);  // the running product, continued below with k = 4
        return false;
    };
    n0 = 0u;
    n1 = 0u;
    if (on0) {
        uint32_t v;
        n0 = first(ra, em0, v) ? v : poisson_knuth_from(em0, seed, neuron, step, 0u, 1u, __uint_as_float(v), 4u);
    }
    if (on1) {
        uint32_t v;
        n1 = first(rb, em1, v) ? v : poisson_knuth_from(em1, seed, neuron, step, 1u, 1u, __uint_as_float(v), 4u);
    }
}

__device__ __forceinline__ float4 ld_col4(const float* p) { return __ldcg(reinterpret_cast<const float4*>(p)); }

__device__ __forceinline__ float flush_tiny(float t) { return t < 1e-30f ? 0.0f : t; }

__device__ __forceinline__ float clamp_w(float w, float wmin, float wmax) {
    if (w < wmin) return wmin;
    if (w > wmax) return wmax;
    return w;
}

// Barrier among `threads` threads (a multiple of 32) of the CTA on hardware barrier `id` (> 0;
// barrier 0 is __syncthreads).
__device__ __forceinline__ void named_barrier_sync(uint32_t id, uint32_t threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Grid-wide barrier over the persistent CTAs on a monotonically increasing 64-bit arrival counter.
// After the CTA-wide sync, thread 0 arrives with a gpu-scope release reduction (no return value
// to wait for) and spins with gpu-scope acquire loads until the counter reaches `target`, the
// count at which every CTA has arrived; the closing CTA-wide sync extends the acquire to the
// whole CTA.  Bounded: after s_wait_limit_ns (or when another CTA has already given up) it
// records kErrBarrierTimeout and returns false so the kernel can exit.  `arrive` false (a test
// switch only) makes this CTA wait without arriving, so that every CTA's wait runs out.
__device__ __forceinline__ bool grid_barrier(unsigned long long* barrier, int32_t* error, unsigned long long target,
                                             int* s_ok, bool arrive = true) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if (arrive) red_release_add_u64(barrier, 1ull);
        unsigned long long t_start = 0;
        uint32_t spins = 0;
        while (static_cast<long long>(ld_acquire_u64(barrier) - target) < 0) {
            if ((++spins & 255u) == 0u) {
                const unsigned long long now = globaltimer_ns();
                if (t_start == 0) {
                    t_start = now;
                } else if (now - t_start > s_wait_limit_ns) {
                    atomicExch(error, kErrBarrierTimeout);
                    ok = 0;
                    break;
                }
                if (ld_relaxed_s32(error) != kErrNone) {
                    ok = 0;
                    break;
                }
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// The same barrier in two halves, so a CTA can do work that needs nothing from other CTAs between
// its arrival and its wait: grid_arrive (after the CTA-wide sync, thread 0's release reduction)
// and grid_wait (thread 0's bounded acquire spin, then the CTA-wide sync that extends it).
__device__ __forceinline__ void grid_arrive(unsigned long long* barrier, bool arrive) {
    __syncthreads();
    if (threadIdx.x == 0 && arrive) red_release_add_u64(barrier, 1ull);
}

__device__ __forceinline__ bool grid_wait(unsigned long long* barrier, int32_t* error, unsigned long long target,
                                          int* s_ok) {
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned long long t_start = 0;
        uint32_t spins = 0;
        while (static_cast<long long>(ld_acquire_u64(barrier) - target) < 0) {
            if ((++spins & 255u) == 0u) {
                const unsigned long long now = globaltimer_ns();
                if (t_start == 0) {
                    t_start = now;
                } else if (now - t_start > s_wait_limit_ns) {
                    atomicExch(error, kErrBarrierTimeout);
                    ok = 0;
                    break;
                }
                if (ld_relaxed_s32(error) != kErrNone) {
                    ok = 0;
                    break;
                }
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// Optional phase timing (profiling builds only, -DBSNN_PHASE_TIMING): thread 0 of every CTA adds
// the SM clock cycles spent in each phase to a shared-memory tally (s_tally_[phase]) that the
// kernel adds to S->phase_ns[cta * kPhaseSlots + phase] when it ends: 3 partial-sum loads, 0 rest
// of the step inputs, 1 neuron phase beside the plasticity update and normalisation, 2 spike bits
// and row x, 4 weight pass, 5 grid barrier.  Spans of single threads inside those phases: 6 the
// neuron warp's own neuron phase, 7 the update warps' update plus normalisation sums, 8 their
// update alone, 9 thread 0's share of the weight pass, 10 the last warp's share of it, 11 thread
// 0's share of the spike-bit merge, 12 the normalisation sums alone, 13 the last warp's update,
// 14 the work done between arrival and wait (warp 1), 15 arrival to release (thread 0).
#ifdef BSNN_PHASE_TIMING
#define BSNN_TMARK(slot)                                                                   \
    do {                                                                                   \
        if (threadIdx.x == 0) {                                                            \
            const unsigned long long now_ = static_cast<unsigned long long>(clock64());    \
            s_tally_[(slot)] += now_ - t_mark_;                                            \
            t_mark_ = now_;                                                                \
        }                                                                                  \
    } while (0)
// Per-thread spans (same builds): the calling thread adds the cycles since its own start mark
// to s_tally_[slot] (one thread per slot, so no two threads add to the same slot).
#define BSNN_TSTART(var) const unsigned long long var = static_cast<unsigned long long>(clock64())
#define BSNN_TSPAN(slot, var) (s_tally_[(slot)] += static_cast<unsigned long long>(clock64()) - (var))
#else
#define BSNN_TMARK(slot) \
    do {                 \
    } while (0)
#define BSNN_TSTART(var) \
    do {                 \
    } while (0)
#define BSNN_TSPAN(slot, var) \
    do {                      \
    } while (0)
#endif


// Shared-memory copies of the launch-invariant descriptors, so every phase dereferences shared
// memory instead of chaining dependent global loads through DSim.
struct Desc {
    const DGroup* groups;
    const DTraceSet* ts;
    const DConn* conns;
    const DPlast* plast;
    const DMon* mons;
    const uint32_t* red_list;
    uint32_t n_groups, n_mons, n_plast, N;
    int32_t noise_mode;
    uint32_t seed, stim_len, replay_steps;
    uint32_t goff[kMaxGroups], gn[kMaxGroups];
    uint32_t bitbase[kMaxMonitors];
    uint32_t red_begin[2][kMaxGroups], red_end[2][kMaxGroups];
    // DSim pointers and sizes the step loop uses (read from shared memory, not through DSim)
    float* partials;
    uint32_t n_slots, N_pad, spk_words, max_own;
    uint32_t* spk_bits[2];
    const uint32_t* stim_off;
    const uint32_t* ev_neuron;
    const float* ev_delta;
    const uint8_t* replay;
    unsigned long long* barrier;
    int32_t* error;
    uint32_t stage_rows;  // rows per staging buffer (0 = streamed rows are loaded directly)
    int32_t wfmt;         // weight storage form (kFmt*)
    uint32_t q_nonneg;    // FP8 copy decoded by bit placement (non-negative weights)
    unsigned long long skip_step;  // test switch (DSim::skip_step)
    uint32_t skip_cta;
};

// Values produced and consumed by the same CTA stay in shared memory: x of the own neurons, the
// plasticity row factors (double-buffered by step parity: the neuron phase of step t writes them
// while the weight pass of step t still reads step t-1's) and the own neurons' spike bits.
struct SmemLayout {
    float* wres;        // resident weight rows, S->resident_floats floats (16-byte aligned)
    float4* row;        // [max_rows] {x, scale, rowA, rowB}
    DRowMeta* meta;     // [max_rows]
    uint32_t* rowflag;  // [max_rows] presynaptic neuron spiked at the step being applied
    float* rowtgt;      // [max_rows] triplet normalisation target of the row
    float* rowsum;      // [max_rows] running sum of each resident triplet row (see norm_rows)
    uint32_t* sbits;    // [spk_words] spike bitmask of the step whose plasticity is being applied
    uint32_t* gbits;    // [2][max_own/32 + 2] this CTA's spike bits, by step parity
    float* xown;        // [n_ts][max_own] x = d - r of the own neurons (this step)
    float2* rowfac;     // [2][n_plast][max_own] {rowA, rowB} of the own neurons, by step parity
    float* ns;          // [ns_fields][max_own] state of the own neurons (kNs* fields below)
    float* rsum;        // [max_trows][n_chunks] carried triplet row sums by 32-unit chunk
    float* red;         // [2][max_own] the previous step's propagation into the own neurons
    unsigned char* stage;  // [warps][2][stage_rows][512 B] staging buffers for streamed rows
    uint64_t* stage_bar;   // [warps][2] their mbarriers
    uint32_t* stage_phase; // [warps] parity of each buffer's next completion (bit b: buffer b)
    float* lzs;         // [max_rows] row-scaled forms: normalisation scale s of each row
    float* lzm;         // [max_rows] sum of the row's masters
    float* lzq;         // [max_rows] quantisation scale of the row's GEMV copy
    float* lzqi;        // [max_rows] its reciprocal
    float* lzf;         // [max_rows] this step's GEMV weight of the row, x s qs
    float* lzw;         // [32] per-warp partial master sums of a spiking row (row-scaled forms)
    uint32_t* bits;     // [n_spike_monitors][max_own/32 + 2]
    unsigned char* desc;  // descriptor copies (DGroup, DTraceSet, DConn, DPlast, DMon, slot lists)
};

// Fields of the shared-memory neuron state: fixed ones, then two per trace set (r, d), two per
// plasticity on the presynaptic side (pre, triplet pre), two per plasticity on the postsynaptic
// side (post, triplet post) and one per voltage monitor (the neuron's ring column, or -1).
enum : uint32_t {
    kNsV = 0, kNsGe, kNsGi, kNsIstim, kNsEr, kNsEd, kNsIr, kNsId, kNsBgGe, kNsBgGi, kNsRefrac, kNsSpike,
    kNsNoise,  // the step's background Poisson counts, excitatory | inhibitory << 16 (drawn ahead)
    kNsFixed
};
struct NsLayout {
    uint32_t ts, pre, post, mon, fields;
};
__host__ __device__ __forceinline__ NsLayout ns_layout(uint32_t n_ts, uint32_t n_pre, uint32_t n_post, uint32_t n_mon) {
    NsLayout L;
    L.ts = kNsFixed;
    L.pre = L.ts + 2u * n_ts;
    L.post = L.pre + 2u * n_pre;
    L.mon = L.post + 2u * n_post;
    L.fields = L.mon + n_mon;
    return L;
}

__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Byte layout of the dynamic shared memory; the host sizes the launch with the same function.
struct SmemSizes {
    size_t wres, row, meta, rowflag, rowtgt, rowsum, sbits, gbits, xown, rowfac, ns, rsum, redscr, stage, lz, bits, groups, ts,
        conns, plast, mons, red, total;
};
__host__ __device__ __forceinline__ SmemSizes smem_sizes(uint32_t resident_floats, uint32_t max_rows, uint32_t max_own,
                                                         uint32_t spk_words, uint32_t n_spike_mons, uint32_t n_groups,
                                                         uint32_t n_ts, uint32_t n_conns, uint32_t n_plast,
                                                         uint32_t n_mons, uint32_t n_red, uint32_t ns_fields,
                                                         uint32_t rsum_floats, uint32_t stage_warps,
                                                         uint32_t stage_rows, uint32_t lazy_rows) {
    SmemSizes z;
    z.wres = align16(sizeof(float) * static_cast<size_t>(resident_floats));
    z.row = align16(sizeof(float4) * max_rows);
    z.meta = align16(sizeof(DRowMeta) * max_rows);
    z.rowflag = align16(sizeof(uint32_t) * max_rows);
    z.rowtgt = align16(sizeof(float) * max_rows);
    z.rowsum = align16(sizeof(float) * max_rows);
    z.sbits = align16(sizeof(uint32_t) * spk_words);
    z.gbits = align16(sizeof(uint32_t) * 2 * (max_own / 32 + 2));
    z.xown = align16(sizeof(float) * n_ts * max_own);
    z.rowfac = align16(sizeof(float2) * 2 * n_plast * max_own);
    z.ns = align16(sizeof(float) * ns_fields * max_own);
    z.rsum = align16(sizeof(float) * rsum_floats);
    z.redscr = align16(sizeof(float) * 2 * max_own);
    z.stage = stage_rows ? ((static_cast<size_t>(stage_warps) * 2u * stage_rows * 512u + 127u) & ~size_t(127)) +
                               align16(static_cast<size_t>(stage_warps) * (2u * sizeof(uint64_t) + sizeof(uint32_t)))
                         : 0;
    z.lz = align16(sizeof(float) * (5u * static_cast<size_t>(lazy_rows) + (lazy_rows ? 32u : 0u)));
    z.bits = align16(sizeof(uint32_t) * n_spike_mons * (max_own / 32 + 2));
    z.groups = align16(sizeof(DGroup) * n_groups);
    z.ts = align16(sizeof(DTraceSet) * n_ts);
    z.conns = align16(sizeof(DConn) * n_conns);
    z.plast = align16(sizeof(DPlast) * n_plast);
    z.mons = align16(sizeof(DMon) * n_mons);
    z.red = align16(sizeof(uint32_t) * n_red);
    z.total = z.wres + z.row + z.meta + z.rowflag + z.rowtgt + z.rowsum + z.sbits + z.gbits + z.xown + z.rowfac + z.ns + z.rsum + z.redscr + z.stage + z.lz +
              z.bits + z.groups + z.ts + z.conns + z.plast + z.mons + z.red;
    return z;
}

__device__ __forceinline__ int group_of(const Desc& D, uint32_t j) {
    for (uint32_t g = 0; g < D.n_groups; ++g)
        if (j - D.goff[g] < D.gn[g]) return static_cast<int>(g);
    return -1;
}

// The previous step's GEMV partial sums at the own neurons' columns: red[T][i] = sum over the
// slots listed for (T, group of neuron n0+i) of that neuron's column.  One warp takes one quad of
// 4 columns (quads start at multiples of 4 from the group's first column, which is 16-byte
// aligned in the partial rows, so the first and last quad may include neighbours' columns that are
// read and dropped); its lanes take the slot entries lane, lane + 32, ...
// of the group's two lists taken as one sequence, each lane summing its entries in order, and an
// xor-butterfly adds the lanes, so the summation order is fixed.  Up to 32 * kQ entries per quad
// cost one round trip to L2.
__device__ __forceinline__ void load_partials(const DSim* S, const Desc& D, const DCta& cta, uint32_t par,
                                              const SmemLayout& sm, uint32_t max_own) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nwarps = blockDim.x >> 5;
    const float* part = D.partials + static_cast<size_t>(par) * D.n_slots * D.N_pad;
    const uint32_t npad = D.N_pad;
    constexpr int kQ = 8;
    uint32_t qbase = 0;  // quads of earlier groups of this CTA, so that warps rotate over groups
    for (uint32_t g = 0; g < D.n_groups; ++g) {
        const uint32_t goff = D.goff[g], gend = goff + D.gn[g];
        const uint32_t a = cta.n0 > goff ? cta.n0 : goff, b = cta.n1 < gend ? cta.n1 : gend;
        if (a >= b) continue;
        const uint32_t qa = goff + ((a - goff) & ~3u);  // first column of the first quad
        const uint32_t nq = (b - qa + 3u) / 4u;
        const uint32_t lb0 = D.red_begin[0][g], n0 = D.red_end[0][g] - lb0;
        const uint32_t lb1 = D.red_begin[1][g], n1 = D.red_end[1][g] - lb1;
        const uint32_t n_all = n0 + n1;
        const float* cols = part + D.groups[g].pcol + (qa - goff);
        for (uint32_t qd = (warp + nwarps - qbase % nwarps) % nwarps; qd < nq; qd += nwarps) {
            const float* col = cols + 4u * qd;
            float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
            for (uint32_t e0 = lane; e0 < n_all; e0 += 32u * kQ) {
                float4 v[kQ];
#pragma unroll
                for (int q = 0; q < kQ; ++q) {
                    const uint32_t e = e0 + 32u * q;
                    const uint32_t k = e < n0 ? lb0 + e : lb1 + (e - n0);
                    v[q] = e < n_all ? ld_col4(col + static_cast<size_t>(D.red_list[k]) * npad)
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int q = 0; q < kQ; ++q) {
                    const uint32_t e = e0 + 32u * q;
                    float4& acc = e < n0 ? s0 : s1;
                    if (e < n_all) {
                        acc.x += v[q].x;
                        acc.y += v[q].y;
                        acc.z += v[q].z;
                        acc.w += v[q].w;
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                s0.x += __shfl_xor_sync(kFull, s0.x, o);
                s0.y += __shfl_xor_sync(kFull, s0.y, o);
                s0.z += __shfl_xor_sync(kFull, s0.z, o);
                s0.w += __shfl_xor_sync(kFull, s0.w, o);
                s1.x += __shfl_xor_sync(kFull, s1.x, o);
                s1.y += __shfl_xor_sync(kFull, s1.y, o);
                s1.z += __shfl_xor_sync(kFull, s1.z, o);
                s1.w += __shfl_xor_sync(kFull, s1.w, o);
            }
            if (lane < 4u) {
                const uint32_t j = qa + 4u * qd + lane;
                if (j >= a && j < b) {
                    const float t0 = lane == 0 ? s0.x : lane == 1 ? s0.y : lane == 2 ? s0.z : s0.w;
                    const float t1 = lane == 0 ? s1.x : lane == 1 ? s1.y : lane == 2 ? s1.z : s1.w;
                    sm.red[j - cta.n0] = t0;
                    sm.red[max_own + (j - cta.n0)] = t1;
                }
            }
        }
        qbase += nq;
    }
}

// The previous step's propagation into own neuron i for target T (after load_partials).
__device__ __forceinline__ float dot_of(const SmemLayout& sm, uint32_t T, uint32_t i, uint32_t max_own,
                                        uint32_t nwarps) {
    return sm.red[T * max_own + i];
}

// Phase A: one thread per owned neuron (threads 0 .. n_own-1).  The neuron's state is read from
// and written back to the shared-memory copy; global memory receives only the plasticity column
// factors (read by other CTAs) and the voltage rings.  The reference's per-step arithmetic runs
// statement by statement.
__device__ __forceinline__ void neuron_phase(const DSim* S, const Desc& D, const DCta& cta, unsigned long long t,
                                          uint32_t clock, uint32_t par, bool has_dot, const SmemLayout& sm,
                                          uint32_t max_own, const NsLayout& L, uint32_t ev_lo, uint32_t ev_hi) {
    const uint32_t i = threadIdx.x;
    if (i >= cta.n1 - cta.n0) return;
    const uint32_t j = cta.n0 + i;
    const int g = group_of(D, j);
    if (g < 0) return;
    const DGroup& G = D.groups[g];
    const uint32_t loc = j - G.off;
    float* ns = sm.ns + i;
    const uint32_t MO = max_own;

    // ---- loads (shared memory) ----
    float ge_used = ns[kNsGe * MO], gi_used = ns[kNsGi * MO];
    const float er0 = ns[kNsEr * MO], ir0 = ns[kNsIr * MO], ed0 = ns[kNsEd * MO], id0 = ns[kNsId * MO];
    float istim = ns[kNsIstim * MO];
    float v = ns[kNsV * MO];
    uint32_t refrac = __float_as_uint(ns[kNsRefrac * MO]);
    if (has_dot) {
        // background of the previous step plus the previous step's propagation
        // (cublasSgemv y = A x + y, kernel_connection_propagate.cu:79-94)
        const uint32_t nwarps = blockDim.x >> 5;
        ge_used = ge_used + dot_of(sm, 0u, i, MO, nwarps);
        gi_used = gi_used + dot_of(sm, 1u, i, MO, nwarps);
    }

    // ---- kernel_update_background_conductances (kernel_neuron_group_evolve.cu:11-83) ----
    float er = flush_tiny(er0 * G.bg_er_decay);
    float ir = flush_tiny(ir0 * G.bg_ir_decay);
    float ed = flush_tiny(ed0 * G.bg_ed_decay);
    float id = flush_tiny(id0 * G.bg_id_decay);
    const uint32_t noise = __float_as_uint(ns[kNsNoise * MO]);
    const uint32_t ne = noise & 0xffffu, ni = noise >> 16;
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

    // ---- kernel_neuron_group_evolve (kernel_neuron_group_evolve.cu:85-130) ----
    uint32_t spike = 0;
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

    // ---- stores ----
    ns[kNsEr * MO] = er;
    ns[kNsEd * MO] = ed;
    ns[kNsIr * MO] = ir;
    ns[kNsId * MO] = id;
    ns[kNsBgGe * MO] = bg_ge;
    ns[kNsBgGi * MO] = bg_gi;
    ns[kNsV * MO] = v;
    ns[kNsRefrac * MO] = __uint_as_float(refrac);
    ns[kNsGe * MO] = bg_ge;  // reset for the next propagation (kernel_neuron_group_evolve.cu:126-129)
    ns[kNsGi * MO] = bg_gi;
    ns[kNsSpike * MO] = __uint_as_float(spike);
    if (spike) atomicOr(&sm.gbits[par * (max_own / 32u + 2u) + (j >> 5) - (cta.n0 >> 5)], 1u << (j & 31u));

    // Stimulus::apply / kernel_stimulus_apply (stimulus.cpp:46-60, kernel_stimulus_apply.cu:7-21):
    // events of this step land after the evolve read i_stimulus, so they act from the next step.
    if (ev_lo < ev_hi) {
        uint32_t lo = ev_lo, hi = ev_hi;
        while (lo < hi) {  // lower_bound of j in the step's events (sorted by neuron)
            const uint32_t mid = (lo + hi) >> 1;
            if (D.ev_neuron[mid] < j) lo = mid + 1;
            else hi = mid;
        }
        for (uint32_t k = lo; k < ev_hi && D.ev_neuron[k] == j; ++k) istim = istim + D.ev_delta[k];
        ns[kNsIstim * MO] = istim;
    }

    // Connection traces (kernel_connection_propagate.cu:8-46): decay d, decay r, +norm on spike.
#pragma unroll
    for (int k = 0; k < kMaxGroupRoles; ++k) {
        if (k >= static_cast<int>(G.n_ts)) break;
        const DTraceSet& TS = D.ts[G.ts[k]];
        float* f = ns + (L.ts + 2u * k) * MO;
        float d = flush_tiny(f[MO] * TS.d_decay);
        float r = flush_tiny(f[0] * TS.r_decay);
        if (spike == 1) {
            r += TS.norm;
            d += TS.norm;
        }
        f[0] = r;
        f[MO] = d;
        sm.xown[static_cast<uint32_t>(G.ts[k]) * max_own + i] = d - r;
    }

    // Plasticity traces as presynaptic neuron: decay (the value the weight update uses), row
    // factors for that update, then the spike increment (kernel_*_plasticity_update.cu).
#pragma unroll
    for (int k = 0; k < kMaxGroupRoles; ++k) {
        if (k >= static_cast<int>(G.n_plast_pre)) break;
        const DPlast& P = D.plast[G.plast_pre[k]];
        float* f = ns + (L.pre + 2u * k) * MO;
        const float pre = flush_tiny(f[0] * P.pre_decay);
        float rowA, rowB;
        if (P.kind == kKindTriplet) {
            const float tpre = flush_tiny(f[MO] * P.tpre_decay);
            rowA = pre;
            rowB = P.ltd_A + (P.ltd_B * tpre);
            f[MO] = spike == 1 ? tpre + 1.0f : tpre;
        } else {
            rowA = pre;
            rowB = -1.0f * P.ltd_A;
        }
        sm.rowfac[(par * D.n_plast + static_cast<uint32_t>(G.plast_pre[k])) * max_own + i] = make_float2(rowA, rowB);
        f[0] = spike == 1 ? pre + 1.0f : pre;
    }
    // ... and as postsynaptic neuron: column factors, which other CTAs read.
#pragma unroll
    for (int k = 0; k < kMaxGroupRoles; ++k) {
        if (k >= static_cast<int>(G.n_plast_post)) break;
        const DPlast& P = D.plast[G.plast_post[k]];
        float* f = ns + (L.post + 2u * k) * MO;
        const float post = flush_tiny(f[0] * P.post_decay);
        float colA, colB;
        if (P.kind == kKindTriplet) {
            const float tpost = flush_tiny(f[MO] * P.tpost_decay);
            colA = P.ltp_A + (P.ltp_B * tpost);
            colB = -1.0f * post;
            f[MO] = spike == 1 ? tpost + 1.0f : tpost;
        } else if (P.kind == kKindIstdp) {
            colA = P.ltp_A;
            colB = post - P.ltd_B;
        } else {
            colA = P.ltp_A;
            colB = post;
        }
        P.colA[par][loc] = colA;
        P.colB[par][loc] = colB;
        f[0] = spike == 1 ? post + 1.0f : post;
    }

    // Monitors (kernel_historicize_spikes.cu:7-21, kernel_historicize_membrane_potentials.cu:7-21).
    uint32_t vk = 0;  // voltage monitors seen so far (their ring columns are ns fields)
    for (uint32_t k = 0; k < G.n_mon; ++k) {
        const int m = G.mon[k];
        const DMon& M = D.mons[m];
        if (M.kind == kMonSpikes) {
            if (spike) {
                const uint32_t w0 = (cta.n0 > G.off ? cta.n0 - G.off : 0u) >> 5;
                atomicOr(&sm.bits[D.bitbase[m] + ((loc >> 5) - w0)], 1u << (loc & 31u));
            }
        } else {
            const int32_t col = __float_as_int(ns[(L.mon + vk) * MO]);
            ++vk;
            if (col >= 0) M.vh[static_cast<size_t>(clock % M.interval) * M.n_sel + col] = v;
        }
    }
}

// The background Poisson counts of step t for the own neurons (kernel_neuron_group_evolve.cu:49-56:
// one excitatory and one inhibitory count per neuron and step), into the kNsNoise field.  They
// depend only on (seed, neuron, step) -- or on the replayed counts -- so they are drawn ahead, by
// threads [first_thread, blockDim), while the CTA waits at the grid barrier before step t.
__device__ __forceinline__ void draw_noise(const Desc& D, const DCta& cta, unsigned long long t, const SmemLayout& sm,
                                           uint32_t max_own, uint32_t first_thread) {
    if (threadIdx.x < first_thread) return;
    for (uint32_t i = threadIdx.x - first_thread; i < cta.n1 - cta.n0; i += blockDim.x - first_thread) {
        const uint32_t j = cta.n0 + i;
        const int g = group_of(D, j);
        if (g < 0) continue;
        const DGroup& G = D.groups[g];
        uint32_t ne = 0, ni = 0;
        if (D.noise_mode == kNoisePhilox) {
            poisson_knuth_pair(G.exp_neg_mean_e, G.has_bg_e, G.exp_neg_mean_i, G.has_bg_i, D.seed, j, t, ne, ni);
        } else if (D.noise_mode == kNoiseReplay && t < D.replay_steps) {
            const size_t base = (static_cast<size_t>(t) * D.N + j) * 2u;
            ne = D.replay[base];
            ni = D.replay[base + 1];
        }
        sm.ns[kNsNoise * max_own + i] = __uint_as_float(ne | (ni << 16));
    }
}

// Copies the own neurons' state between global memory and the shared-memory copy (launch
// prologue: to_smem; finalize: back, with the pending propagation added to g and x = d - r).
__device__ __forceinline__ void move_neuron_state(const DSim* S, const Desc& D, const DCta& cta, const SmemLayout& sm,
                                               uint32_t max_own, const NsLayout& L, bool to_smem, uint32_t spar,
                                               bool add_dot) {
    const uint32_t MO = max_own, nwarps = blockDim.x >> 5;
    for (uint32_t i = threadIdx.x; i < cta.n1 - cta.n0; i += blockDim.x) {
        const uint32_t j = cta.n0 + i;
        const int g = group_of(D, j);
        if (g < 0) continue;
        const DGroup& G = D.groups[g];
        const uint32_t loc = j - G.off;
        float* ns = sm.ns + i;
        if (to_smem) {
            ns[kNsV * MO] = S->v[j];
            ns[kNsGe * MO] = S->ge[j];
            ns[kNsGi * MO] = S->gi[j];
            ns[kNsIstim * MO] = S->istim[j];
            ns[kNsEr * MO] = S->bg_er[j];
            ns[kNsEd * MO] = S->bg_ed[j];
            ns[kNsIr * MO] = S->bg_ir[j];
            ns[kNsId * MO] = S->bg_id[j];
            ns[kNsBgGe * MO] = S->bg_ge[j];
            ns[kNsBgGi * MO] = S->bg_gi[j];
            ns[kNsRefrac * MO] = __uint_as_float(S->refrac[j]);
            ns[kNsSpike * MO] = 0.0f;
        } else {
            S->v[j] = ns[kNsV * MO];
            S->ge[j] = add_dot ? ns[kNsGe * MO] + dot_of(sm, 0u, i, MO, nwarps) : ns[kNsGe * MO];
            S->gi[j] = add_dot ? ns[kNsGi * MO] + dot_of(sm, 1u, i, MO, nwarps) : ns[kNsGi * MO];
            S->istim[j] = ns[kNsIstim * MO];
            S->bg_er[j] = ns[kNsEr * MO];
            S->bg_ed[j] = ns[kNsEd * MO];
            S->bg_ir[j] = ns[kNsIr * MO];
            S->bg_id[j] = ns[kNsId * MO];
            S->bg_ge[j] = ns[kNsBgGe * MO];
            S->bg_gi[j] = ns[kNsBgGi * MO];
            S->refrac[j] = __float_as_uint(ns[kNsRefrac * MO]);
            S->spikes[spar][j] = __float_as_uint(ns[kNsSpike * MO]);
        }
        for (uint32_t k = 0; k < G.n_ts; ++k) {
            const DTraceSet& TS = D.ts[G.ts[k]];
            float* f = ns + (L.ts + 2u * k) * MO;
            if (to_smem) {
                f[0] = TS.r[loc];
                f[MO] = TS.d[loc];
            } else {
                TS.r[loc] = f[0];
                TS.d[loc] = f[MO];
                TS.x[loc] = f[MO] - f[0];
            }
        }
        for (uint32_t k = 0; k < G.n_plast_pre; ++k) {
            const DPlast& P = D.plast[G.plast_pre[k]];
            float* f = ns + (L.pre + 2u * k) * MO;
            if (to_smem) {
                f[0] = P.pre[loc];
                f[MO] = P.kind == kKindTriplet ? P.tpre[loc] : 0.0f;
            } else {
                P.pre[loc] = f[0];
                if (P.kind == kKindTriplet) P.tpre[loc] = f[MO];
            }
        }
        for (uint32_t k = 0; k < G.n_plast_post; ++k) {
            const DPlast& P = D.plast[G.plast_post[k]];
            float* f = ns + (L.post + 2u * k) * MO;
            if (to_smem) {
                f[0] = P.post[loc];
                f[MO] = P.kind == kKindTriplet ? P.tpost[loc] : 0.0f;
            } else {
                P.post[loc] = f[0];
                if (P.kind == kKindTriplet) P.tpost[loc] = f[MO];
            }
        }
        if (to_smem) {
            uint32_t vk = 0;
            for (uint32_t k = 0; k < G.n_mon; ++k) {
                const DMon& M = D.mons[G.mon[k]];
                if (M.kind == kMonSpikes) continue;
                ns[(L.mon + vk) * MO] = __int_as_float(M.sel_idx[loc]);
                ++vk;
            }
        }
    }
}

// Writes this CTA's spike bits of each spike monitor into the ring slot of `clock`.  Each CTA
// clears and sets only the bits of its own neurons, so the word updates of different CTAs commute.
__device__ __forceinline__ void merge_bits(uint32_t* word, uint32_t mask, uint32_t bits) {
    const uint32_t clear = mask & ~bits;
    if (clear) atomicAnd(word, ~clear);
    if (bits) atomicOr(word, bits);
}

__device__ __forceinline__ uint32_t range_mask(uint32_t w, uint32_t w0, uint32_t w1, uint32_t a, uint32_t b_end) {
    const uint32_t lo = w == w0 ? (a & 31u) : 0u;
    const uint32_t hi = w == w1 ? ((b_end - 1) & 31u) : 31u;
    return (hi == 31u ? 0xffffffffu : ((1u << (hi + 1u)) - 1u)) & ~((1u << lo) - 1u);
}

// Runs on threads [0, nthreads) of the CTA.
__device__ __forceinline__ void flush_spike_bits(const DSim* S, const Desc& D, const DCta& cta, uint32_t clock,
                                              uint32_t par, const SmemLayout& sm, uint32_t nthreads) {
    // the network-wide spike bitmask of this step (read by every CTA's next weight pass)
    if (cta.n1 > cta.n0) {
        const uint32_t w0 = cta.n0 >> 5, w1 = (cta.n1 - 1) >> 5;
        for (uint32_t w = w0 + threadIdx.x; w <= w1; w += nthreads)
            merge_bits(D.spk_bits[par] + w, range_mask(w, w0, w1, cta.n0, cta.n1),
                       sm.gbits[par * (D.max_own / 32u + 2u) + w - w0]);
    }
    for (uint32_t m = 0; m < D.n_mons; ++m) {
        const DMon& M = D.mons[m];
        if (M.kind != kMonSpikes) continue;
        const DGroup& G = D.groups[M.group];
        const uint32_t a = cta.n0 > G.off ? cta.n0 - G.off : 0u;
        const uint32_t b_end = cta.n1 - G.off < G.n ? cta.n1 - G.off : G.n;
        if (cta.n1 <= G.off || a >= b_end) continue;
        const uint32_t w0 = a >> 5, w1 = (b_end - 1) >> 5;
        for (uint32_t w = w0 + threadIdx.x; w <= w1; w += nthreads) {
            const uint32_t lo = w == w0 ? (a & 31u) : 0u;
            const uint32_t hi = w == w1 ? ((b_end - 1) & 31u) : 31u;
            const uint32_t mask = (hi == 31u ? 0xffffffffu : ((1u << (hi + 1u)) - 1u)) & ~((1u << lo) - 1u);
            const uint32_t bits = sm.bits[D.bitbase[m] + (w - w0)] & mask;
            uint32_t* word = M.bits + static_cast<size_t>(clock % M.interval) * M.words + w;
            const uint32_t clear = mask & ~bits;
            if (clear) atomicAnd(word, ~clear);
            if (bits) atomicOr(word, bits);
        }
    }
}

// Per-row data of the pending plasticity update for phase B and the normalisation pass: the row
// factors and the presynaptic spike of the step being applied (both from shared memory); the
// row scale starts at 1 and x at 0 (row = {x, scale, rowA, rowB}).
__device__ __forceinline__ void rows_pending(const Desc& D, const DCta& cta, bool pending, uint32_t ppar,
                                          const SmemLayout& sm, uint32_t max_own) {
    const uint32_t n_gbits = max_own / 32u + 2u;
    for (uint32_t r = threadIdx.x; r < cta.n_rows; r += blockDim.x) {
        const DRowMeta meta = sm.meta[r];
        const DConn& C = D.conns[meta.conn];
        const uint32_t i = meta.j - cta.n0;  // rows belong to this CTA's own neurons
        float4 row = make_float4(0.0f, D.wfmt != kFmtF32 ? sm.lzs[r] * sm.lzq[r] : 1.0f, 0.0f, 0.0f);
        uint32_t flag = 0;
        if (pending && C.plast >= 0) {
            const float2 f = sm.rowfac[(ppar * D.n_plast + static_cast<uint32_t>(C.plast)) * max_own + i];
            row.z = f.x;
            row.w = f.y;
            flag = (sm.gbits[ppar * n_gbits + (meta.j >> 5) - (cta.n0 >> 5)] >> (meta.j & 31u)) & 1u;
        }
        sm.row[r] = row;
        sm.rowflag[r] = flag;
    }
}

// x = d - r of this step into the row table (after the neuron phase).
// (Row-scaled forms: also the row's GEMV weight x s qs, with s qs from the row table.)
// Runs on threads [0, nthreads) of the CTA.
__device__ __forceinline__ void rows_x(const Desc& D, const DCta& cta, const SmemLayout& sm, uint32_t max_own,
                                       uint32_t nthreads) {
    for (uint32_t r = threadIdx.x; r < cta.n_rows; r += nthreads) {
        const DRowMeta meta = sm.meta[r];
        const DConn& C = D.conns[meta.conn];
        const float x = sm.xown[static_cast<uint32_t>(C.ts) * max_own + (meta.j - cta.n0)];
        sm.row[r].x = x;
        if (D.wfmt != kFmtF32) sm.lzf[r] = x * sm.row[r].y;
    }
}

// Stages the network-wide spike bitmask of step parity `spar` in shared memory.
__device__ __forceinline__ void stage_spike_bits(const Desc& D, uint32_t spar, const SmemLayout& sm) {
    for (uint32_t w = threadIdx.x; w < D.spk_words; w += blockDim.x) sm.sbits[w] = __ldcg(D.spk_bits[spar] + w);
}


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

// 16-byte weight accesses: shared memory (resident rows, 32-bit shared addresses) or global.
__device__ __forceinline__ float4 lds4(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ void sts4(uint32_t a, float4 v) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w));
}
__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// mbarrier and bulk asynchronous copy (global -> this CTA's shared memory, no multicast).
constexpr uint32_t kStageDead = 0x80000000u;  // staging gave up (stage_phase bit)
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0u;
}
// Bounded wait for the completion of phase `parity` of an mbarrier.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity))
        if (globaltimer_ns() - t0 > s_wait_limit_ns) return false;
    return true;
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Address of weight (row i of block B, column q), in shared memory for resident blocks.
__device__ __forceinline__ float* weight_ptr(const DBlk& B, const DConn& C, const SmemLayout& sm, uint32_t i,
                                             uint32_t q) {
    return B.resident ? sm.wres + B.sm_off + static_cast<size_t>(i) * C.ld + q
                      : C.w + static_cast<size_t>(B.row_begin + i) * C.ld + q;
}

// The pending plasticity update of step parity `ppar`, applied in place and only where a spike
// touches a weight (spikes are sparse, so this pass is event-driven):
//   column pass: every weight in the column of a postsynaptic neuron that spiked, in rows whose
//                presynaptic neuron did not spike: LTP;
//   row pass:    every weight in the row of a presynaptic neuron that spiked: LTP where the
//                postsynaptic neuron spiked, then LTD.
// The two passes touch disjoint weights, so each weight gets the reference's LTP-then-LTD
// sequence exactly once.  The column factors come from the owners' parity buffers in global
// memory, the row factors from the row table.
// Every warp enumerates the spiking neurons in the same order (lanes over the bitmask words or the
// rows, then a ballot), and all the threads share out each one: the rows of a spiking column, or
// the columns of a spiking row, kUpdUnroll columns per thread at a time with all their loads
// issued before the first update.  A row streamed from global memory thus costs a few memory
// round trips instead of one per 32 columns.  Each weight is still updated by exactly one thread.
// Runs on warps [w_first, w_first + nwarps) of the CTA.
constexpr uint32_t kUpdUnroll = 4;

__device__ __forceinline__ void apply_updates(const Desc& D, const DBlk* s_blk, uint32_t nblk, uint32_t ppar,
                                           const SmemLayout& sm, uint32_t w_first, uint32_t nwarps) {
    const uint32_t tid = threadIdx.x - 32u * w_first, nthr = 32u * nwarps, lane = tid & 31u;
    for (uint32_t bk = 0; bk < nblk; ++bk) {
        const DBlk B = s_blk[bk];
        const DConn& C = D.conns[B.conn];
        if (C.plast < 0) continue;
        const DPlast& P = D.plast[C.plast];
        const uint32_t nrows = B.row_end - B.row_begin, n_post = C.n_post, post_off = C.post_off;
        const float* colA = P.colA[ppar];
        const float* colB = P.colB[ppar];
        const bool carry_sum = B.resident && P.kind == kKindTriplet;  // keep rowsum in step (see norm_rows)
        // column pass: lanes scan the bitmask words of the postsynaptic group
        const uint32_t w0 = post_off >> 5, w1 = (post_off + n_post - 1u) >> 5;
        for (uint32_t wb = w0; wb <= w1; wb += 32u) {
            const uint32_t w = wb + lane;
            uint32_t bits = 0u;
            if (w <= w1) {
                bits = sm.sbits[w];
                if (w == w0) bits &= 0xffffffffu << (post_off & 31u);
                if (w == w1) bits &= 0xffffffffu >> (31u - ((post_off + n_post - 1u) & 31u));
            }
            uint32_t nz = __ballot_sync(kFull, bits != 0u);
            while (nz) {
                const uint32_t src = __ffs(nz) - 1u;
                nz &= nz - 1u;
                uint32_t wbits = __shfl_sync(kFull, bits, src);
                while (wbits) {
                    const uint32_t b = __ffs(wbits) - 1u;
                    wbits &= wbits - 1u;
                    const uint32_t q = 32u * (wb + src) + b - post_off;
                    const float cA = __ldcg(colA + q), cB = __ldcg(colB + q);
                    for (uint32_t i = tid; i < nrows; i += nthr) {
                        const uint32_t r = B.srow + i;
                        if (sm.rowflag[r]) continue;  // the row pass owns this weight
                        float* wp = weight_ptr(B, C, sm, i, q);
                        const float4 rw = sm.row[r];
                        const float w0 = *wp;
                        const float w1 = plastic_update(w0, q, B.row_begin + i, n_post, 1u, 0u, rw.z, cA, cB, rw.w,
                                                        P.wmin, P.wmax);
                        *wp = w1;
                        // one thread per row, columns in ascending order: a fixed summation order
                        if (carry_sum) sm.rowsum[r] += w1 - w0;
                    }
                }
            }
        }
        // row pass: lanes scan the rows
        for (uint32_t i0 = 0; i0 < nrows; i0 += 32u) {
            uint32_t spk = __ballot_sync(kFull, i0 + lane < nrows && sm.rowflag[B.srow + i0 + lane] != 0u);
            while (spk) {
                const uint32_t i = i0 + __ffs(spk) - 1u;
                spk &= spk - 1u;
                const float4 rw = sm.row[B.srow + i];
                for (uint32_t qb = tid; qb < n_post; qb += kUpdUnroll * nthr) {
                    float wv[kUpdUnroll], a[kUpdUnroll], b[kUpdUnroll];
#pragma unroll
                    for (uint32_t u = 0; u < kUpdUnroll; ++u) {
                        const uint32_t q = qb + u * nthr;
                        wv[u] = a[u] = b[u] = 0.0f;
                        if (q < n_post) {
                            wv[u] = *weight_ptr(B, C, sm, i, q);
                            a[u] = __ldcg(colA + q);
                            b[u] = __ldcg(colB + q);
                        }
                    }
#pragma unroll
                    for (uint32_t u = 0; u < kUpdUnroll; ++u) {
                        const uint32_t q = qb + u * nthr;
                        if (q < n_post) {
                            const uint32_t g = post_off + q;
                            const uint32_t post_spk = (sm.sbits[g >> 5] >> (g & 31u)) & 1u;
                            *weight_ptr(B, C, sm, i, q) = plastic_update(wv[u], q, B.row_begin + i, n_post, post_spk,
                                                                         1u, rw.z, a[u], b[u], rw.w, P.wmin, P.wmax);
                        }
                    }
                }
            }
        }
    }
}

// For triplet rows streamed from global memory the row sums are carried from one step to the next
// in 32-unit chunks, so the normalisation need not read every row again: rsum[tr][c] is the sum
// over the units u = 32c .. 32c+31 of row tr (the CTA's tr-th streamed triplet row) of
// (w.x + w.y) + (w.z + w.w), added over the lanes of a warp by an xor-butterfly.  The weight pass
// produces them for the weights it has just stored; the next step's normalisation recomputes
// only the chunks its plasticity update touched and adds the chunks of a row in a fixed order.
// (Resident rows are summed from shared memory instead: reading them again is cheaper than the
// butterflies.)
__device__ __forceinline__ float unit_sum(float4 w) { return (w.x + w.y) + (w.z + w.w); }

__device__ __forceinline__ float warp_sum(float p) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(kFull, p, o);
    return p;
}

// Sum of `lane`'s units (lane, lane+32, ...) of two resident rows at once, each as
// (x + y) + (z + w) per unit in unit order; `two` = false sums the first row only.
__device__ __forceinline__ void row_pair_sums(uint32_t s0, uint32_t s1, uint32_t units, uint32_t lane, bool two,
                                              float& sum0, float& sum1) {
    sum0 = 0.0f;
    sum1 = 0.0f;
    for (uint32_t u0 = 0; u0 < units; u0 += 128u) {
        float4 a[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t u = u0 + lane + 32u * k;
            const bool in = u < units;
            a[k] = in ? lds4(s0 + 16u * u) : make_float4(0.f, 0.f, 0.f, 0.f);
            b[k] = in && two ? lds4(s1 + 16u * u) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (u0 + lane + 32u * k >= units) continue;
            sum0 += unit_sum(a[k]);
            sum1 += unit_sum(b[k]);
        }
    }
}

// Recomputes the carried chunk sums of row i of a streamed block B for the chunks c0 .. c0+7 set in
// `need` (bit k = chunk c0 + k), eight butterflies at a time.
__device__ __forceinline__ void chunk_sums8(const DBlk& B, const DConn& C, const SmemLayout& sm, uint32_t i,
                                           uint32_t c0, uint32_t need, uint32_t lane, uint32_t n_chunks) {
    const float* row = C.w + static_cast<size_t>(B.row_begin + i) * C.ld;
    float p[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t u = 32u * (c0 + k) + lane;
        p[k] = ((need >> k) & 1u) && u < C.units ? unit_sum(ld_col4(row + 4u * u)) : 0.0f;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 8; ++k) p[k] += __shfl_xor_sync(kFull, p[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if ((need >> k) & 1u) sm.rsum[(B.trow + i) * n_chunks + c0 + k] = p[k];
    }
}

// Pass 1 of the triplet normalisation (after apply_updates), on warps [w_first, w_first + nwarps).
// Resident rows keep a running sum (rowsum): summed exactly at the start of each launch, then
// carried from step to step -- the column pass adds each weight change (one thread per row, the
// columns in ascending order), the normalisation multiplies it by the row's scale as the weight
// pass rescales the row -- and summed again (each lane its units, then an xor-butterfly) for rows
// whose presynaptic neuron spiked, where the row pass rewrote every weight, and for every row each
// kRowSumResync steps.  Between those its rounding departs from the stored row's exact sum by
// about 1e-8 relative (the reference itself sums sequentially in float, 1e-6 from exact), so the
// scale target / sum agrees with the reference's to the comparison tolerance, and the rows are not
// read again for their sums each step.
// Streamed rows: the carried chunk sums are used; the chunks the update touched are recomputed
// first (all chunks of a row whose presynaptic neuron spiked; for a spiking postsynaptic neuron,
// its chunk in every row), then the lanes add the chunks c = lane, lane + 32, ... in order and an
// xor-butterfly adds the lanes.  Lane 0 forms target / sum.
// Steps between the exact re-summations of the resident triplet rows' running sums: the
// normalisation applied at internal step t sums every row again when t is a multiple of this, at
// a fixed step whatever the launch boundaries (results do not depend on how steps are split
// into launches).
constexpr unsigned long long kRowSumResync = 1000ull;

// The exact sum of every resident triplet row (each warp two rows at a time), into rowsum: when a
// launch starts at step 0.  Between launches the sums are kept in DConn::rowsum.
__device__ __noinline__ void resident_row_sums(const Desc& D, const SmemLayout& sm, const DBlk* s_blk,
                                                  uint32_t nblk) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nwarps = blockDim.x >> 5;
    for (uint32_t bk = 0; bk < nblk; ++bk) {
        const DBlk B = s_blk[bk];
        const DConn& C = D.conns[B.conn];
        if (!B.resident || C.plast < 0 || D.plast[C.plast].kind != kKindTriplet) continue;
        const uint32_t nrows = B.row_end - B.row_begin, base = saddr(sm.wres + B.sm_off), ld = C.ld;
        for (uint32_t i = warp; i < nrows; i += 2u * nwarps) {
            const uint32_t i2 = i + nwarps;
            const bool two = i2 < nrows;
            float sum0, sum1;
            row_pair_sums(base + 4u * ld * i, base + 4u * ld * (two ? i2 : i), C.units, lane, two, sum0, sum1);
            sum0 = warp_sum(sum0);
            sum1 = warp_sum(sum1);
            if (lane == 0) {
                sm.rowsum[B.srow + i] = sum0;
                if (two) sm.rowsum[B.srow + i2] = sum1;
            }
        }
    }
}

// Copies the running sums of the resident triplet rows between shared memory and DConn::rowsum.
__device__ __forceinline__ void move_row_sums(const Desc& D, const SmemLayout& sm, const DBlk* s_blk, uint32_t nblk,
                                              bool to_smem) {
    for (uint32_t bk = 0; bk < nblk; ++bk) {
        const DBlk& B = s_blk[bk];
        const DConn& C = D.conns[B.conn];
        if (!B.resident || C.rowsum == nullptr) continue;
        for (uint32_t i = threadIdx.x; i < B.row_end - B.row_begin; i += blockDim.x) {
            if (to_smem) sm.rowsum[B.srow + i] = __ldcg(C.rowsum + B.row_begin + i);
            else C.rowsum[B.row_begin + i] = sm.rowsum[B.srow + i];
        }
    }
}

template <bool CARRY>
__device__ __forceinline__ void norm_rows(const Desc& D, const SmemLayout& sm, const DBlk* s_blk, uint32_t nblk,
                                       uint32_t w_first, uint32_t nwarps, uint32_t n_chunks, bool resync) {
    const uint32_t warp = (threadIdx.x >> 5) - w_first, lane = threadIdx.x & 31u;
    uint32_t k = 0;  // running index over the CTA's normalised rows
    for (uint32_t bk = 0; bk < nblk; ++bk) {
        const DBlk B = s_blk[bk];
        const DConn& C = D.conns[B.conn];
        if (C.plast < 0 || D.plast[C.plast].kind != kKindTriplet) continue;
        const uint32_t nrows = B.row_end - B.row_begin, units = C.units;
        const uint32_t first = (warp + nwarps - (k % nwarps)) % nwarps;
        k += nrows;
        if (!CARRY || B.resident) {
            const uint32_t base = saddr(sm.wres + B.sm_off), ld = C.ld;
            for (uint32_t i = first; i < nrows; i += nwarps) {
                const uint32_t r = B.srow + i;
                float sum = sm.rowsum[r];
                if (resync || sm.rowflag[r]) {  // every kRowSumResync steps, or after the row pass: sum again
                    float unused;
                    row_pair_sums(base + 4u * ld * i, base + 4u * ld * i, units, lane, false, sum, unused);
                    sum = warp_sum(sum);
                }
                if (lane == 0) {
                    const float scale = sum <= 0.0f ? 1.0f : __fdiv_rn(sm.rowtgt[r], sum);
                    sm.row[r].y = scale;
                    sm.rowsum[r] = sum <= 0.0f ? sum : sum * scale;  // the sum the rescaled row will have
                }
            }
            continue;
        }
        const uint32_t nch = (units + 31u) / 32u;
        // chunks holding a postsynaptic neuron that spiked (bit c % 32 of dirty<c / 32>; chunks past
        // 128 are always recomputed)
        uint32_t dirty0 = 0, dirty1 = 0, dirty2 = 0, dirty3 = 0;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const uint32_t c = lane + 32u * m;
            bool d = false;
            if (c < nch) {
                const uint32_t q0 = 128u * c, q1 = q0 + 128u < C.n_post ? q0 + 128u : C.n_post;
                const uint32_t g0 = C.post_off + q0, g1 = C.post_off + q1 - 1u;
                for (uint32_t w = g0 >> 5; w <= (g1 >> 5); ++w) {
                    uint32_t bits = sm.sbits[w];
                    if (w == (g0 >> 5)) bits &= 0xffffffffu << (g0 & 31u);
                    if (w == (g1 >> 5)) bits &= 0xffffffffu >> (31u - (g1 & 31u));
                    d |= bits != 0u;
                }
            }
            const uint32_t bal = __ballot_sync(kFull, d);
            if (m == 0) dirty0 = bal;
            else if (m == 1) dirty1 = bal;
            else if (m == 2) dirty2 = bal;
            else dirty3 = bal;
        }
        for (uint32_t i = first; i < nrows; i += nwarps) {
            const uint32_t r = B.srow + i;
            const bool all = sm.rowflag[r] != 0u;
            for (uint32_t c0 = 0; c0 < nch; c0 += 8u) {
                const uint32_t dm = c0 < 32u ? dirty0 : c0 < 64u ? dirty1 : c0 < 96u ? dirty2 : dirty3;
                uint32_t need = all || c0 >= 128u ? 0xffu : (dm >> (c0 & 31u)) & 0xffu;
                if (nch - c0 < 8u) need &= (1u << (nch - c0)) - 1u;
                if (need) chunk_sums8(B, C, sm, i, c0, need, lane, n_chunks);
            }
            __syncwarp();
            float s = 0.0f;
            for (uint32_t c = lane; c < nch; c += 32u) s += sm.rsum[(B.trow + i) * n_chunks + c];
            s = warp_sum(s);
            if (lane == 0) sm.row[r].y = s <= 0.0f ? 1.0f : __fdiv_rn(sm.rowtgt[r], s);
        }
    }
}

// Pass 2 over the rows of one block for unit u: normalise + store the updated weights (SCALE:
// rows of a triplet plasticity with an update pending), accumulate this step's GEMV partial sums,
// and (TRIP: rows of a triplet plasticity) leave the chunk sums of the stored weights in rsum.
// All 32 lanes of a warp run this together on units 32c .. 32c+31 of one segment; lanes past the
// segment's units (live = false) only take part in the chunk butterflies.
template <bool RESIDENT, bool SCALE, bool TRIP>
__device__ __forceinline__ float4 block_rows(const DBlk& B, const DConn& C, uint32_t u, bool live, const SmemLayout& sm,
                                             bool accumulate, float4 acc, uint32_t n_chunks) {
    const uint32_t nrows = B.row_end - B.row_begin, ld = C.ld;
    const uint32_t sbase = RESIDENT ? saddr(sm.wres + B.sm_off) + 16u * u : 0u;
    float* gbase = RESIDENT ? nullptr : C.w + static_cast<size_t>(B.row_begin) * ld + 4u * u;
    const float2* rowp = reinterpret_cast<const float2*>(sm.row + B.srow);  // {x, scale} of each row
    const uint32_t lane = threadIdx.x & 31u, chunk = u / 32u;
    constexpr int kB = (RESIDENT || SCALE || TRIP) ? 4 : 8;
    for (uint32_t i0 = 0; i0 < nrows; i0 += kB) {
        float4 wb[kB];
#pragma unroll
        for (int b = 0; b < kB; ++b) {
            if (i0 + b < nrows) {
                if constexpr (RESIDENT) wb[b] = lds4(sbase + 4u * ld * (i0 + b));
                else wb[b] = ld_col4(gbase + static_cast<size_t>(i0 + b) * ld);
            }
        }
        float p[kB];
#pragma unroll
        for (int b = 0; b < kB; ++b) {
            p[b] = 0.0f;
            if (i0 + b >= nrows) continue;
            const uint32_t i = i0 + b;
            const float2 rw = rowp[2u * i];
            float4 w4 = wb[b];
            if constexpr (SCALE) {
                w4.x *= rw.y;
                w4.y *= rw.y;
                w4.z *= rw.y;
                w4.w *= rw.y;
                if (live) {
                    if constexpr (RESIDENT) sts4(sbase + 4u * ld * i, w4);
                    else __stcg(reinterpret_cast<float4*>(gbase + static_cast<size_t>(i) * ld), w4);
                }
            }
            if constexpr (TRIP) p[b] = live ? unit_sum(w4) : 0.0f;
            if (accumulate) {
                acc.x = fmaf(w4.x, rw.x, acc.x);
                acc.y = fmaf(w4.y, rw.x, acc.y);
                acc.z = fmaf(w4.z, rw.x, acc.z);
                acc.w = fmaf(w4.w, rw.x, acc.w);
            }
        }
        if constexpr (TRIP) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
                for (int b = 0; b < kB; ++b) p[b] += __shfl_xor_sync(kFull, p[b], o);
            }
            if (lane == 0) {
#pragma unroll
                for (int b = 0; b < kB; ++b)
                    if (i0 + b < nrows) sm.rsum[(B.trow + i0 + b) * n_chunks + chunk] = p[b];
            }
        }
    }
    return acc;
}

// block_rows for a streamed block whose rows are staged through shared memory: the warp's 32
// units of a row (one contiguous run of up to 512 bytes) arrive by bulk asynchronous copies,
// `stage_rows` rows per buffer, two buffers per warp, so the next batch streams in while the
// current one is used.  The lanes issue the copies (lane 0, always a live lane, sets the expected
// byte count first); every lane waits on the buffer's mbarrier, with a bound: a timeout sets the
// error word and turns staging off for the warp.
template <bool SCALE, bool TRIP>
__device__ __forceinline__ void block_rows_staged(const Desc& D, const DBlk& B, const DConn& C, uint32_t u, bool live,
                                                  unsigned mask, const SmemLayout& sm, bool accumulate, float4& acc,
                                                  uint32_t n_chunks) {
    const uint32_t nrows = B.row_end - B.row_begin, ld = C.ld, R = D.stage_rows;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, chunk = u / 32u;
    uint32_t phase = sm.stage_phase[warp];
    if (nrows == 0u || (phase & kStageDead)) return;
    const uint32_t chunk_units = C.units - 32u * chunk < 32u ? C.units - 32u * chunk : 32u;
    const uint32_t row_bytes = 16u * chunk_units;
    const uint32_t buf0 = saddr(sm.stage) + warp * 2u * R * 512u;
    const uint32_t bar0 = saddr(sm.stage_bar + 2u * warp);
    const float* src0 = C.w + static_cast<size_t>(B.row_begin) * ld + 4u * 32u * chunk;
    const float2* rowp = reinterpret_cast<const float2*>(sm.row + B.srow);
    float* gbase = C.w + static_cast<size_t>(B.row_begin) * ld + 4u * u;
    const uint32_t nb = (nrows + R - 1u) / R;
    const uint32_t rank = __popc(mask & ((1u << lane) - 1u)), nlanes = __popc(mask);
    auto issue = [&](uint32_t k) {
        const uint32_t r0 = k * R, r1 = r0 + R < nrows ? r0 + R : nrows;
        const uint32_t bar = bar0 + 8u * (k & 1u), dst = buf0 + (k & 1u) * R * 512u;
        if (lane == 0) mbar_expect_tx(bar, (r1 - r0) * row_bytes);
        __syncwarp(mask);
        for (uint32_t r = r0 + rank; r < r1; r += nlanes)
            bulk_load(dst + (r - r0) * 512u, src0 + static_cast<size_t>(r) * ld, row_bytes, bar);
    };
    issue(0);
    if (nb > 1u) issue(1);
    for (uint32_t k = 0; k < nb; ++k) {
        const uint32_t b = k & 1u;
        const bool got = mbar_wait(bar0 + 8u * b, (phase >> b) & 1u);
        if (!__all_sync(mask, got)) {
            // Give up on staging for the rest of the launch: the batches in flight (this one and
            // the next) land (bounded) and later calls return at once; the host sees the error.
            if (lane == 0) atomicExch(D.error, kErrStageTimeout);
            if (!got) mbar_wait(bar0 + 8u * b, (phase >> b) & 1u);
            if (k + 1u < nb) mbar_wait(bar0 + 8u * (b ^ 1u), (phase >> (b ^ 1u)) & 1u);
            phase |= kStageDead;
            break;
        }
        phase ^= 1u << b;
        const uint32_t r0 = k * R, r1 = r0 + R < nrows ? r0 + R : nrows;
        const uint32_t buf = buf0 + b * R * 512u + 16u * lane;
        for (uint32_t i0 = r0; i0 < r1; i0 += 4u) {
            float4 wb[4];
            float p[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (i0 + q < r1) wb[q] = lds4(buf + (i0 + q - r0) * 512u);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                p[q] = 0.0f;
                if (i0 + q >= r1) continue;
                const uint32_t i = i0 + q;
                const float2 rw = rowp[2u * i];
                float4 w4 = wb[q];
                if constexpr (SCALE) {
                    w4.x *= rw.y;
                    w4.y *= rw.y;
                    w4.z *= rw.y;
                    w4.w *= rw.y;
                    if (live) __stcg(reinterpret_cast<float4*>(gbase + static_cast<size_t>(i) * ld), w4);
                }
                if constexpr (TRIP) p[q] = live ? unit_sum(w4) : 0.0f;
                if (accumulate) {
                    acc.x = fmaf(w4.x, rw.x, acc.x);
                    acc.y = fmaf(w4.y, rw.x, acc.y);
                    acc.z = fmaf(w4.z, rw.x, acc.z);
                    acc.w = fmaf(w4.w, rw.x, acc.w);
                }
            }
            if constexpr (TRIP) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) p[q] += __shfl_xor_sync(mask, p[q], o);
                }
                if (lane == 0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (i0 + q < r1) sm.rsum[(B.trow + i0 + q) * n_chunks + chunk] = p[q];
                }
            }
        }
        // every lane is done with this buffer before it is refilled
        __syncwarp(mask);
        if (k + 2u < nb) {
            fence_proxy_async_shared();
            issue(k + 2u);
        }
    }
    if (lane == 0) sm.stage_phase[warp] = phase;
    __syncwarp(mask);
}

// ---- Row-scaled weight forms (kFmtF32Rows, kFmtBf16, kFmtFp8) ----------------------------------
// A weight is kept as an FP32 master m and the normalisation scale s of its row: the weight is
// w = s m.  The update rules act on w exactly as in the reference form (LTP clamp, then LTD clamp)
// and store m = w / s.  The triplet normalisation (the reference scales the row by target / sum of
// its weights) becomes s = target / M, M being the sum of the row's masters: a row whose
// presynaptic neuron spiked has all its entries updated, and M is summed again from the whole
// row; otherwise M changes by the changes of the entries in the columns of spiking postsynaptic
// neurons.  So the normalisation costs one number per row instead of a read and a write of the
// whole matrix.  The GEMV reads a copy of the masters -- FP32, BF16, or FP8 E4M3 with a per-row
// quantisation scale qs -- and weighs row i by x_i s_i qs_i.  Updates refresh the copy's entries
// they change.

__device__ __forceinline__ float4 bf16x4_to_float4(uint2 v) {
    return make_float4(__uint_as_float(v.x << 16), __uint_as_float(v.x & 0xffff0000u), __uint_as_float(v.y << 16),
                       __uint_as_float(v.y & 0xffff0000u));
}
__device__ __forceinline__ float2 e4m3x2_to_float2(uint32_t v16) {
    const __half2_raw h = __nv_cvt_fp8x2_to_halfraw2(static_cast<__nv_fp8x2_storage_t>(v16), __NV_E4M3);
    return __half22float2(__half2(h));
}
__device__ __forceinline__ float4 e4m3x4_to_float4(uint32_t v) {
    const float2 a = e4m3x2_to_float2(v & 0xffffu), b = e4m3x2_to_float2(v >> 16);
    return make_float4(a.x, a.y, b.x, b.y);
}
// Four non-negative E4M3 codes times 2^-120, by placing each code's 7 magnitude bits at bits 26:20
// of an FP32 word: the E4M3 exponent field becomes the low 4 bits of the FP32 exponent field and
// the 3 mantissa bits its top mantissa bits, so normals map to 2^(e-127) (1 + m/8) and subnormals
// to FP32 denormals 2^-126 (m/8) -- the E4M3 values 2^(e-7) (1 + m/8) and 2^-6 (m/8) times 2^-120,
// exactly.  (Two integer operations per value instead of two conversions.)
__device__ __forceinline__ float4 e4m3x4_nonneg_scaled(uint32_t v) {
    return make_float4(__uint_as_float((v << 20) & 0x07f00000u), __uint_as_float((v << 12) & 0x07f00000u),
                       __uint_as_float((v << 4) & 0x07f00000u), __uint_as_float((v >> 4) & 0x07f00000u));
}
// One 4-column unit of the GEMV copy (EB bytes per element) from shared memory.
template <int EB, bool NN = false>
__device__ __forceinline__ float4 copy_unit_s(uint32_t a) {
    if constexpr (EB == 4) {
        return lds4(a);
    } else if constexpr (EB == 2) {
        uint2 v;
        asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
        return bf16x4_to_float4(v);
    } else {
        uint32_t v;
        asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
        if constexpr (NN) return e4m3x4_nonneg_scaled(v);
        else return e4m3x4_to_float4(v);
    }
}
// Element index of (row, column q) in a connection's tiled GEMV copy.
__host__ __device__ __forceinline__ size_t copy_index(uint32_t n_pre, uint32_t row, uint32_t q) {
    return ((static_cast<size_t>(q >> 7) * n_pre + row) << 7) + (q & 127u);
}
// Writes master m of (row, q) into the GEMV copy.
__device__ __forceinline__ void store_copy(int32_t fmt, const DConn& C, uint32_t row, uint32_t q, float m, float qinv) {
    const size_t e = copy_index(C.n_pre, row, q);
    if (fmt == kFmtBf16) reinterpret_cast<__nv_bfloat16*>(C.q)[e] = __float2bfloat16_rn(m);
    else if (fmt == kFmtFp8) reinterpret_cast<__nv_fp8_storage_t*>(C.q)[e] = __nv_cvt_float_to_fp8(m * qinv, __NV_SATFINITE, __NV_E4M3);
    else reinterpret_cast<float*>(C.q)[e] = m;
}

// The pending plasticity update in a row-scaled form, on warps [w_first, w_first + nwarps).
// A row whose presynaptic neuron did not spike gets LTP in the columns of the spiking postsynaptic
// neurons: every warp enumerates those columns in the same order, the threads take the rows, and
// M grows by each change in column order.  A row whose presynaptic neuron spiked gets LTP (where the
// postsynaptic neuron spiked) then LTD on every entry, shared out over all the threads
// (kUpdUnroll columns each at a time, loads issued first); M is summed from the new masters: each
// thread its columns in order, an xor-butterfly per warp, then the warp sums in warp order.
// Named barrier 2 (all the warps given) orders the per-warp sums.
__device__ __forceinline__ void apply_updates_rows(const Desc& D, const DBlk* s_blk, uint32_t nblk, uint32_t ppar,
                                                const SmemLayout& sm, uint32_t w_first, uint32_t nwarps) {
    const uint32_t tid = threadIdx.x - 32u * w_first, nthr = 32u * nwarps, warp = tid >> 5, lane = tid & 31u;
    const int32_t fmt = D.wfmt;
    for (uint32_t bk = 0; bk < nblk; ++bk) {
        const DBlk B = s_blk[bk];
        const DConn& C = D.conns[B.conn];
        if (C.plast < 0) continue;
        const DPlast& P = D.plast[C.plast];
        const uint32_t nrows = B.row_end - B.row_begin, n_post = C.n_post, post_off = C.post_off;
        const float* colA = P.colA[ppar];
        const float* colB = P.colB[ppar];
        const uint32_t w0 = post_off >> 5, w1 = (post_off + n_post - 1u) >> 5;
        for (uint32_t wb = w0; wb <= w1; wb += 32u) {
            const uint32_t w = wb + lane;
            uint32_t bits = 0u;
            if (w <= w1) {
                bits = sm.sbits[w];
                if (w == w0) bits &= 0xffffffffu << (post_off & 31u);
                if (w == w1) bits &= 0xffffffffu >> (31u - ((post_off + n_post - 1u) & 31u));
            }
            uint32_t nz = __ballot_sync(kFull, bits != 0u);
            while (nz) {
                const uint32_t src = __ffs(nz) - 1u;
                nz &= nz - 1u;
                uint32_t wbits = __shfl_sync(kFull, bits, src);
                while (wbits) {
                    const uint32_t b = __ffs(wbits) - 1u;
                    wbits &= wbits - 1u;
                    const uint32_t q = 32u * (wb + src) + b - post_off;
                    const float cA = __ldcg(colA + q);
                    for (uint32_t i = tid; i < nrows; i += nthr) {
                        const uint32_t r = B.srow + i, pl = B.row_begin + i;
                        if (sm.rowflag[r] != 0u || q == pl) continue;  // the row pass below owns this row
                        const float sc = sm.lzs[r];
                        float* mrow = C.w + static_cast<size_t>(pl) * C.ld;
                        const float m0 = __ldcg(mrow + q);
                        const float wv = clamp_w(fmaf(sm.row[r].z, cA, sc * m0), P.wmin, P.wmax);
                        const float m = __fdiv_rn(wv, sc);
                        __stcg(mrow + q, m);
                        store_copy(fmt, C, pl, q, m, sm.lzqi[r]);
                        sm.lzm[r] += m - m0;  // row i always belongs to this thread: a fixed order
                    }
                }
            }
        }
        for (uint32_t i0 = 0; i0 < nrows; i0 += 32u) {
            uint32_t spk = __ballot_sync(kFull, i0 + lane < nrows && sm.rowflag[B.srow + i0 + lane] != 0u);
            while (spk) {
                const uint32_t i = i0 + __ffs(spk) - 1u;
                spk &= spk - 1u;
                const uint32_t r = B.srow + i, pl = B.row_begin + i;
                const float4 rw = sm.row[r];
                const float sc = sm.lzs[r], qinv = sm.lzqi[r];
                float* mrow = C.w + static_cast<size_t>(pl) * C.ld;
                float acc = 0.0f;
                for (uint32_t qb = tid; qb < n_post; qb += kUpdUnroll * nthr) {
                    float m0[kUpdUnroll], a[kUpdUnroll], b[kUpdUnroll];
#pragma unroll
                    for (uint32_t u = 0; u < kUpdUnroll; ++u) {
                        const uint32_t q = qb + u * nthr;
                        m0[u] = a[u] = b[u] = 0.0f;
                        if (q < n_post) {
                            m0[u] = __ldcg(mrow + q);
                            a[u] = __ldcg(colA + q);
                            b[u] = __ldcg(colB + q);
                        }
                    }
#pragma unroll
                    for (uint32_t u = 0; u < kUpdUnroll; ++u) {
                        const uint32_t q = qb + u * nthr;
                        if (q >= n_post) continue;
                        float m = m0[u];
                        if (q != pl) {
                            const uint32_t g = post_off + q;
                            const uint32_t post_spk = (sm.sbits[g >> 5] >> (g & 31u)) & 1u;
                            const float w = plastic_update(sc * m0[u], q, pl, n_post, post_spk, 1u, rw.z, a[u], b[u],
                                                           rw.w, P.wmin, P.wmax);
                            m = __fdiv_rn(w, sc);
                            __stcg(mrow + q, m);
                            store_copy(fmt, C, pl, q, m, qinv);
                        }
                        acc += m;
                    }
                }
                acc = warp_sum(acc);
                if (lane == 0) sm.lzw[warp] = acc;
                named_barrier_sync(2u, nthr);
                if (tid == 0) {
                    float M = 0.0f;
                    for (uint32_t w = 0; w < nwarps; ++w) M += sm.lzw[w];
                    sm.lzm[r] = M;
                }
                named_barrier_sync(2u, nthr);  // the per-warp sums are rewritten for the next row
            }
        }
    }
}

// The triplet normalisation in a row-scaled form: s = target / M for every normalised row (the
// reference leaves a row whose sum is not positive as it is), one warp per row on warps
// [w_first, w_first + nwarps).  A scale outside [1/2, 2] is folded into the row instead: the
// masters become the weights (m = s m, copy refreshed, M summed again) and s = 1, so a master
// never exceeds twice the plastic bound (the FP8 copy's range) and a zero target zeroes the row.
// The row's s qs goes to the row table.
__device__ __forceinline__ void norm_rows_lazy(const Desc& D, const SmemLayout& sm, const DBlk* s_blk, uint32_t nblk,
                                            uint32_t w_first, uint32_t nwarps) {
    const uint32_t warp = (threadIdx.x >> 5) - w_first, lane = threadIdx.x & 31u;
    for (uint32_t bk = 0; bk < nblk; ++bk) {
        const DBlk B = s_blk[bk];
        const DConn& C = D.conns[B.conn];
        if (C.plast < 0 || D.plast[C.plast].kind != kKindTriplet) continue;
        const uint32_t nrows = B.row_end - B.row_begin;
        for (uint32_t i = warp; i < nrows; i += nwarps) {
            const uint32_t r = B.srow + i;
            const float M = sm.lzm[r];
            if (!(M > 0.0f)) continue;
            float sc = __fdiv_rn(sm.rowtgt[r], M);
            if (!(sc >= 0.5f && sc <= 2.0f)) {
                const uint32_t pl = B.row_begin + i;
                const float qinv = sm.lzqi[r];
                float* mrow = C.w + static_cast<size_t>(pl) * C.ld;
                float acc = 0.0f;
                for (uint32_t q = lane; q < C.n_post; q += 32u) {
                    const float m = sc * __ldcg(mrow + q);
                    __stcg(mrow + q, m);
                    store_copy(D.wfmt, C, pl, q, m, qinv);
                    acc += m;
                }
                acc = warp_sum(acc);
                if (lane == 0) sm.lzm[r] = acc;
                sc = 1.0f;
            }
            if (lane == 0) {
                sm.lzs[r] = sc;
                sm.row[r].y = sc * sm.lzq[r];
            }
        }
    }
}

// All blocks of segment SG for unit u; the partial sums go to the segment's slot.  `pending` = an
// update of the previous step is to be applied (normalised triplet rows are rescaled and stored).
// CARRY: the network has streamed triplet rows (a kernel instance of its own, so that networks
// without them do not pay for the extra code).
template <bool CARRY>
__device__ __forceinline__ void segment_unit(const Desc& D, const DSeg& SG, const DBlk* s_blk, uint32_t u, bool live,
                                             bool pending, bool accumulate, const SmemLayout& sm, float* part_out,
                                             uint32_t npad, uint32_t n_chunks) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    bool touched = false;
    // the lanes of this warp that run this call: all of them in a segment with carried row sums,
    // else those whose unit lies in the segment
    const uint32_t left = SG.units - 32u * (u / 32u);
    const unsigned wmask = (CARRY && SG.carried) || left >= 32u ? kFull : (1u << left) - 1u;
    for (uint32_t bk = SG.blk_begin; bk < SG.blk_end; ++bk) {
        const DBlk B = s_blk[bk];
        const DConn& C = D.conns[B.conn];
        const bool trip = C.plast >= 0 && D.plast[C.plast].kind == kKindTriplet;
        const bool scale = pending && trip;
        if (!scale && !accumulate) continue;
        touched = true;
        if (CARRY && !B.resident && D.stage_rows) {
            if (CARRY && trip && accumulate) {
                if (scale) block_rows_staged<true, true>(D, B, C, u, live, wmask, sm, true, acc, n_chunks);
                else block_rows_staged<false, true>(D, B, C, u, live, wmask, sm, true, acc, n_chunks);
            } else if (scale) {
                block_rows_staged<true, CARRY>(D, B, C, u, live, wmask, sm, accumulate, acc, n_chunks);
            } else {
                block_rows_staged<false, false>(D, B, C, u, live, wmask, sm, true, acc, n_chunks);
            }
            continue;
        }
        if (CARRY && trip && accumulate && !B.resident) {
            if (scale) {
                acc = B.resident ? block_rows<true, true, true>(B, C, u, live, sm, true, acc, n_chunks)
                                 : block_rows<false, true, true>(B, C, u, live, sm, true, acc, n_chunks);
            } else {
                acc = B.resident ? block_rows<true, false, true>(B, C, u, live, sm, true, acc, n_chunks)
                                 : block_rows<false, false, true>(B, C, u, live, sm, true, acc, n_chunks);
            }
        } else if (scale) {
            acc = B.resident ? block_rows<true, true, false>(B, C, u, live, sm, accumulate, acc, n_chunks)
                             : block_rows<false, true, CARRY>(B, C, u, live, sm, accumulate, acc, n_chunks);
        } else {
            acc = B.resident ? block_rows<true, false, false>(B, C, u, live, sm, true, acc, n_chunks)
                             : block_rows<false, false, false>(B, C, u, live, sm, true, acc, n_chunks);
        }
    }
    if (accumulate && touched && live)
        *reinterpret_cast<float4*>(part_out + static_cast<size_t>(SG.slot) * npad + SG.pcol + 4u * u) = acc;
}

// Pass 2: each thread owns work items (one 4-column unit of one segment) and walks all of the
// segment's rows; per item the partial sums go to the parity-`par` slot of this CTA.  A warp's
// 32 items always lie in one segment (segments start at multiples of 32 items).
// The row-scaled weight pass as one stream of batches per warp: the warp's tasks are its items
// (it0 + 32 w + lane for it0 = 0, blockDim, ...; one 32-unit chunk of one segment), each item's
// blocks with rows, and each block's batches of R rows.  In the tiled copy a batch is one
// contiguous run of memory, so it arrives by ONE bulk asynchronous copy into one of the warp's two
// shared-memory buffers.  A producer cursor runs up to two batches ahead of the consumer, across
// block and item boundaries, so the next item's rows are in flight while the current one finishes.
struct RowCursor {
    uint32_t it0, seg, bk, k;
    bool valid;
};

__device__ __forceinline__ bool nonempty_block(const DSeg& SG, const DBlk* s_blk, uint32_t from, uint32_t& bk) {
    for (bk = from; bk < SG.blk_end; ++bk)
        if (s_blk[bk].row_end > s_blk[bk].row_begin) return true;
    return false;
}

// Moves c to the first batch of the warp's first item at or after c.it0 that has rows.  With
// `zeros`, the items passed over (segments whose blocks have no rows) get zero partial sums.
__device__ __forceinline__ void seek_item(RowCursor& c, uint32_t n_items, const DSeg* s_seg, uint32_t n_seg,
                                          const DBlk* s_blk, bool zeros, float* part_out, uint32_t npad) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (; c.it0 < n_items; c.it0 += blockDim.x) {
        const int s = seg_of_item(s_seg, n_seg, c.it0 + 32u * warp);
        if (s < 0) continue;
        const DSeg& SG = s_seg[s];
        c.seg = static_cast<uint32_t>(s);
        c.k = 0;
        if (nonempty_block(SG, s_blk, SG.blk_begin, c.bk)) {
            c.valid = true;
            return;
        }
        const uint32_t u = c.it0 + 32u * warp + lane - SG.item_begin;
        if (zeros && u < SG.units && SG.blk_end > SG.blk_begin)
            *reinterpret_cast<float4*>(part_out + static_cast<size_t>(SG.slot) * npad + SG.pcol + 4u * u) =
                make_float4(0.f, 0.f, 0.f, 0.f);
    }
    c.valid = false;
}

__device__ __forceinline__ void advance(RowCursor& c, uint32_t R, uint32_t n_items, const DSeg* s_seg, uint32_t n_seg,
                                        const DBlk* s_blk, bool zeros, float* part_out, uint32_t npad) {
    const DSeg& SG = s_seg[c.seg];
    const DBlk& B = s_blk[c.bk];
    if ((c.k + 1u) * R < B.row_end - B.row_begin) {
        ++c.k;
        return;
    }
    c.k = 0;
    if (nonempty_block(SG, s_blk, c.bk + 1u, c.bk)) return;
    c.it0 += blockDim.x;
    seek_item(c, n_items, s_seg, n_seg, s_blk, zeros, part_out, npad);
}

template <int EB, bool NN>
__device__ __forceinline__ void weight_pass_rows_stream(const Desc& D, const DCta& cta, uint32_t par, const SmemLayout& sm,
                                                        const DSeg* s_seg, const DBlk* s_blk, uint32_t n_seg) {
    constexpr uint32_t UB = 4u * EB, SB = 32u * UB;  // bytes per unit, per row of a tile
    float* part_out = D.partials + static_cast<size_t>(par) * D.n_slots * D.N_pad;
    const uint32_t npad = D.N_pad, n_items = cta.n_items, R = D.stage_rows * (512u / SB);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t phase = sm.stage_phase[warp];
    if (phase & kStageDead) return;
    const uint32_t buf0 = saddr(sm.stage) + warp * 2u * D.stage_rows * 512u;
    const uint32_t bar0 = saddr(sm.stage_bar + 2u * warp);
    auto issue = [&](const RowCursor& c, uint32_t slot) {
        if (lane == 0) {
            const DSeg& SG = s_seg[c.seg];
            const DBlk& B = s_blk[c.bk];
            const DConn& C = D.conns[B.conn];
            const uint32_t nrows = B.row_end - B.row_begin, r0 = c.k * R, n = nrows - r0 < R ? nrows - r0 : R;
            const uint32_t chunk = (c.it0 + 32u * warp - SG.item_begin) / 32u;
            const unsigned char* src =
                static_cast<const unsigned char*>(C.q) + copy_index(C.n_pre, B.row_begin + r0, 128u * chunk) * EB;
            const uint32_t bar = bar0 + 8u * slot;
            mbar_expect_tx(bar, n * SB);
            bulk_load(buf0 + slot * R * SB, src, n * SB, bar);
        }
    };
    RowCursor cc{0u, 0u, 0u, 0u, false};
    seek_item(cc, n_items, s_seg, n_seg, s_blk, true, part_out, npad);
    RowCursor pc = cc;
    uint32_t g_issue = 0, g_use = 0;
    for (int f = 0; f < 2 && pc.valid; ++f) {
        issue(pc, g_issue & 1u);
        ++g_issue;
        advance(pc, R, n_items, s_seg, n_seg, s_blk, false, part_out, npad);
    }
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    while (cc.valid) {
        const uint32_t b = g_use & 1u;
        const bool got = mbar_wait(bar0 + 8u * b, (phase >> b) & 1u);
        if (!__all_sync(kFull, got)) {
            // give up for the launch: the batches in flight land (bounded) and the host sees the error
            if (lane == 0) atomicExch(D.error, kErrStageTimeout);
            if (!got) mbar_wait(bar0 + 8u * b, (phase >> b) & 1u);
            if (g_issue > g_use + 1u) mbar_wait(bar0 + 8u * (b ^ 1u), (phase >> (b ^ 1u)) & 1u);
            phase |= kStageDead;
            break;
        }
        phase ^= 1u << b;
        ++g_use;
        const DSeg& SG = s_seg[cc.seg];
        const DBlk B = s_blk[cc.bk];
        const uint32_t nrows = B.row_end - B.row_begin, r0 = cc.k * R, r1 = r0 + R < nrows ? r0 + R : nrows;
        const uint32_t buf = buf0 + b * R * SB + UB * lane - r0 * SB;
        const float* rowf = sm.lzf + B.srow;
        // whole groups of 8 rows (two accumulators for independent FMA chains), then the rest
        float4 acc2 = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t i0 = r0;
        for (; i0 + 8u <= r1; i0 += 8u) {
            float4 wb[8];
            float f[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                wb[q] = copy_unit_s<EB, NN>(buf + (i0 + q) * SB);
                f[q] = rowf[i0 + q];
            }
#pragma unroll
            for (int q = 0; q < 8; q += 2) {
                acc.x = fmaf(wb[q].x, f[q], acc.x);
                acc.y = fmaf(wb[q].y, f[q], acc.y);
                acc.z = fmaf(wb[q].z, f[q], acc.z);
                acc.w = fmaf(wb[q].w, f[q], acc.w);
                acc2.x = fmaf(wb[q + 1].x, f[q + 1], acc2.x);
                acc2.y = fmaf(wb[q + 1].y, f[q + 1], acc2.y);
                acc2.z = fmaf(wb[q + 1].z, f[q + 1], acc2.z);
                acc2.w = fmaf(wb[q + 1].w, f[q + 1], acc2.w);
            }
        }
        for (; i0 < r1; ++i0) {
            const float4 w = copy_unit_s<EB, NN>(buf + i0 * SB);
            const float f = rowf[i0];
            acc.x = fmaf(w.x, f, acc.x);
            acc.y = fmaf(w.y, f, acc.y);
            acc.z = fmaf(w.z, f, acc.z);
            acc.w = fmaf(w.w, f, acc.w);
        }
        acc.x += acc2.x;
        acc.y += acc2.y;
        acc.z += acc2.z;
        acc.w += acc2.w;
        __syncwarp();
        const RowCursor done = cc;
        advance(cc, R, n_items, s_seg, n_seg, s_blk, true, part_out, npad);
        if (!cc.valid || cc.it0 != done.it0) {  // the item is complete
            const uint32_t u = done.it0 + 32u * warp + lane - SG.item_begin;
            if (u < SG.units)
                *reinterpret_cast<float4*>(part_out + static_cast<size_t>(SG.slot) * npad + SG.pcol + 4u * u) = acc;
            acc = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (pc.valid) {  // refill the buffer just used
            fence_proxy_async_shared();
            issue(pc, g_issue & 1u);
            ++g_issue;
            advance(pc, R, n_items, s_seg, n_seg, s_blk, false, part_out, npad);
        }
    }
    if (lane == 0) sm.stage_phase[warp] = phase;
    __syncwarp();
}

template <bool CARRY, bool LAZY>
__device__ __forceinline__ void weight_pass(const Desc& D, const DCta& cta, bool pending, bool accumulate, uint32_t par,
                                         const SmemLayout& sm, const DSeg* s_seg, const DBlk* s_blk, uint32_t n_seg,
                                         uint32_t n_chunks) {
    if constexpr (LAZY) {  // (the host guarantees staging buffers in the row-scaled forms)
        if (!accumulate) return;
        if (D.wfmt == kFmtBf16) weight_pass_rows_stream<2, false>(D, cta, par, sm, s_seg, s_blk, n_seg);
        else if (D.wfmt == kFmtFp8 && D.q_nonneg) weight_pass_rows_stream<1, true>(D, cta, par, sm, s_seg, s_blk, n_seg);
        else if (D.wfmt == kFmtFp8) weight_pass_rows_stream<1, false>(D, cta, par, sm, s_seg, s_blk, n_seg);
        else weight_pass_rows_stream<4, false>(D, cta, par, sm, s_seg, s_blk, n_seg);
        return;
    }
    float* part_out = D.partials + static_cast<size_t>(par) * D.n_slots * D.N_pad;
    const uint32_t npad = D.N_pad;
    for (uint32_t it0 = 0; it0 < cta.n_items; it0 += blockDim.x) {
        // the staged loads keep per-warp buffer state in shared memory: the warp enters each
        // item converged, after its lane 0 has recorded that state
        if (CARRY && D.stage_rows) __syncwarp();
        const uint32_t it = it0 + threadIdx.x;
        const int s = seg_of_item(s_seg, n_seg, it);
        if (s < 0) continue;  // the whole warp
        const DSeg& SG = s_seg[s];
        const uint32_t u = it - SG.item_begin;
        const bool live = u < SG.units;
        if (!live && !(CARRY && SG.carried)) continue;  // only the chunk butterflies need every lane
        segment_unit<CARRY>(D, SG, s_blk, live ? u : SG.units - 1u, live, pending, accumulate, sm, part_out, npad, n_chunks);
    }
}

// Copies the resident rows of this CTA between global memory and shared memory.
__device__ __forceinline__ void move_resident(const Desc& D, const DBlk* s_blk, uint32_t nblk, const SmemLayout& sm,
                                           bool to_smem) {
    for (uint32_t bk = 0; bk < nblk; ++bk) {
        const DBlk& B = s_blk[bk];
        if (!B.resident) continue;
        const DConn& C = D.conns[B.conn];
        const uint32_t n4 = (B.row_end - B.row_begin) * (C.ld / 4u);
        float4* g = reinterpret_cast<float4*>(C.w + static_cast<size_t>(B.row_begin) * C.ld);
        const uint32_t sh = saddr(sm.wres + B.sm_off);
        if (to_smem)
            for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) sts4(sh + 16u * i, __ldcg(g + i));
        else
            for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) __stcg(g + i, lds4(sh + 16u * i));
    }
}

__device__ __forceinline__ void copy_words(void* dst, const void* src, size_t bytes) {
    uint32_t* d = static_cast<uint32_t*>(dst);
    const uint32_t* s = static_cast<const uint32_t*>(src);
    for (size_t k = threadIdx.x; k < bytes / 4; k += blockDim.x) d[k] = s[k];
}

template <bool CARRY, bool LAZY>
__global__ void __launch_bounds__(CARRY ? kMaxThreads : LAZY ? kMaxThreadsRows : kMaxThreadsPlain, 1)
    bsnn_step_kernel(const DSim* __restrict__ S, uint32_t n_steps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Desc s_d;
    __shared__ DCta s_cta;
    __shared__ DSeg s_seg[kMaxSegsPerCta];
    __shared__ DBlk s_blk[kMaxBlksPerCta];
    __shared__ unsigned long long s_t0, s_bar0;
    __shared__ uint32_t s_clock0;
    __shared__ int s_ok;
    __shared__ uint32_t s_has_norm;
    __shared__ uint32_t s_blk_base, s_nblk;
    __shared__ uint32_t s_ev[2];
    // Shared-memory copies of the layout and the work plan: phases re-read them from shared memory
    // instead of keeping them in registers for the whole launch.
    __shared__ SmemLayout sm;
    __shared__ NsLayout s_L;

    const uint32_t max_rows = S->max_rows, max_own = S->max_own;
    uint32_t n_spike_mons = 0;
    for (uint32_t m = 0; m < S->n_mons; ++m) n_spike_mons += S->mons[m].kind == kMonSpikes ? 1u : 0u;
    const NsLayout L0 = ns_layout(S->ns_ts, S->ns_pre, S->ns_post, S->ns_mon);
    const SmemSizes z = smem_sizes(S->resident_floats, max_rows, max_own, S->spk_words, n_spike_mons, S->n_groups,
                                   S->n_ts, S->n_conns, S->n_plast, S->n_mons, S->n_red, L0.fields,
                                   S->max_trows * S->n_chunks, S->stage_warps, S->stage_rows,
                                   LAZY ? max_rows : 0u);
    if (threadIdx.x == 0) {
        s_wait_limit_ns = S->wait_limit_ns;
        s_L = L0;
        unsigned char* p = smem_raw;
        sm.wres = reinterpret_cast<float*>(p);
        p += z.wres;
        sm.row = reinterpret_cast<float4*>(p);
        p += z.row;
        sm.meta = reinterpret_cast<DRowMeta*>(p);
        p += z.meta;
        sm.rowflag = reinterpret_cast<uint32_t*>(p);
        p += z.rowflag;
        sm.rowtgt = reinterpret_cast<float*>(p);
        p += z.rowtgt;
        sm.rowsum = reinterpret_cast<float*>(p);
        p += z.rowsum;
        sm.sbits = reinterpret_cast<uint32_t*>(p);
        p += z.sbits;
        sm.gbits = reinterpret_cast<uint32_t*>(p);
        p += z.gbits;
        sm.xown = reinterpret_cast<float*>(p);
        p += z.xown;
        sm.rowfac = reinterpret_cast<float2*>(p);
        p += z.rowfac;
        sm.ns = reinterpret_cast<float*>(p);
        p += z.ns;
        sm.rsum = reinterpret_cast<float*>(p);
        p += z.rsum;
        sm.red = reinterpret_cast<float*>(p);
        p += z.redscr;
        {
            const size_t buf = S->stage_rows ? (static_cast<size_t>(S->stage_warps) * 2u * S->stage_rows * 512u + 127u) &
                                                   ~size_t(127)
                                             : 0;
            sm.stage = p;
            sm.stage_bar = reinterpret_cast<uint64_t*>(p + buf);
            sm.stage_phase = reinterpret_cast<uint32_t*>(p + buf + static_cast<size_t>(S->stage_warps) * 2u * sizeof(uint64_t));
        }
        p += z.stage;
        sm.lzs = reinterpret_cast<float*>(p);
        sm.lzm = sm.lzs + max_rows;
        sm.lzq = sm.lzm + max_rows;
        sm.lzqi = sm.lzq + max_rows;
        sm.lzf = sm.lzqi + max_rows;
        sm.lzw = sm.lzf + max_rows;
        p += z.lz;
        sm.bits = reinterpret_cast<uint32_t*>(p);
        p += z.bits;
        sm.desc = p;
    }
    __syncthreads();
    const NsLayout& L = s_L;
    // Descriptor copies.
    {
        unsigned char* p = sm.desc;
        copy_words(p, S->groups, sizeof(DGroup) * S->n_groups);
        p += z.groups;
        copy_words(p, S->ts, sizeof(DTraceSet) * S->n_ts);
        p += z.ts;
        copy_words(p, S->conns, sizeof(DConn) * S->n_conns);
        p += z.conns;
        copy_words(p, S->plast, sizeof(DPlast) * S->n_plast);
        p += z.plast;
        copy_words(p, S->mons, sizeof(DMon) * S->n_mons);
        p += z.mons;
        copy_words(p, S->red_list, sizeof(uint32_t) * S->n_red);
    }
    if (threadIdx.x == 0) {
        unsigned char* p = sm.desc;
        s_d.groups = reinterpret_cast<const DGroup*>(p);
        p += z.groups;
        s_d.ts = reinterpret_cast<const DTraceSet*>(p);
        p += z.ts;
        s_d.conns = reinterpret_cast<const DConn*>(p);
        p += z.conns;
        s_d.plast = reinterpret_cast<const DPlast*>(p);
        p += z.plast;
        s_d.mons = reinterpret_cast<const DMon*>(p);
        p += z.mons;
        s_d.red_list = reinterpret_cast<const uint32_t*>(p);
        s_d.n_groups = S->n_groups;
        s_d.n_mons = S->n_mons;
        s_d.n_plast = S->n_plast;
        s_d.N = S->N;
        s_d.noise_mode = S->noise_mode;
        s_d.seed = S->seed;
        s_d.stim_len = S->stim_len;
        s_d.replay_steps = S->replay_steps;
        s_d.partials = S->partials;
        s_d.n_slots = S->n_slots;
        s_d.N_pad = S->N_pad;
        s_d.spk_words = S->spk_words;
        s_d.max_own = max_own;
        s_d.spk_bits[0] = S->spk_bits[0];
        s_d.spk_bits[1] = S->spk_bits[1];
        s_d.stim_off = S->stim_off;
        s_d.ev_neuron = S->ev_neuron;
        s_d.ev_delta = S->ev_delta;
        s_d.replay = S->replay;
        s_d.barrier = S->barrier;
        s_d.error = S->error;
        s_d.stage_rows = S->stage_rows;
        s_d.wfmt = S->wfmt;
        s_d.q_nonneg = S->q_nonneg;
        s_d.skip_step = S->skip_step;
        s_d.skip_cta = S->skip_cta;
        uint32_t base = 0;
        for (uint32_t m = 0; m < S->n_mons; ++m) {
            s_d.bitbase[m] = base;
            if (S->mons[m].kind == kMonSpikes) base += max_own / 32u + 2u;
        }
        for (uint32_t g = 0; g < S->n_groups; ++g) {
            s_d.goff[g] = S->groups[g].off;
            s_d.gn[g] = S->groups[g].n;
        }
        for (uint32_t T = 0; T < 2; ++T)
            for (uint32_t g = 0; g < kMaxGroups; ++g) {
                s_d.red_begin[T][g] = S->red_begin[T][g];
                s_d.red_end[T][g] = S->red_end[T][g];
            }
        s_cta = S->ctas[blockIdx.x];
        s_t0 = *S->steps_done;
        s_clock0 = *S->clock;
        // Every launch completes all of its barriers, so between launches the arrival counter is a
        // multiple of the grid size; CTAs of this launch that already arrived at its first barrier
        // (fewer than the grid size, since this CTA has not) do not change the rounded-down value.
        const unsigned long long n = gridDim.x;
        s_bar0 = ld_acquire_u64(S->barrier) / n * n;
        uint32_t has_norm = 0;
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
    const Desc& D = s_d;
    const DCta& cta = s_cta;
    const uint32_t n_seg = cta.seg_end - cta.seg_begin;
    const uint32_t nwarps = blockDim.x >> 5;
    const uint32_t n_own = cta.n1 - cta.n0;
    const uint32_t neuron_warps = (n_own + 31u) / 32u;
    const uint32_t n_chunks = S->n_chunks;
    // The normalisation pass runs beside the neuron phase on the warps the neurons leave free.
    const bool norm_beside = neuron_warps < nwarps;
    for (uint32_t b = threadIdx.x; b < s_nblk; b += blockDim.x) s_blk[b] = S->blks[s_blk_base + b];
    {
        const DRowMeta* rows = S->rows + S->rows_begin[blockIdx.x];
        for (uint32_t r = threadIdx.x; r < cta.n_rows; r += blockDim.x) sm.meta[r] = rows[r];
    }
    const uint32_t n_bits_words = n_spike_mons * (max_own / 32u + 2u);
    const uint32_t n_gbits = max_own / 32u + 2u;
    if (D.stage_rows && (threadIdx.x & 31u) == 0u) {
        const uint32_t w = threadIdx.x >> 5;
        mbar_init(saddr(sm.stage_bar + 2u * w), 1u);
        mbar_init(saddr(sm.stage_bar + 2u * w + 1u), 1u);
        sm.stage_phase[w] = 0u;
        fence_mbar_init();
    }
    __syncthreads();
    move_resident(D, s_blk, s_nblk, sm, true);
    move_neuron_state(S, D, cta, sm, max_own, L, true, 0u, false);
    // triplet normalisation targets of this CTA's rows (constant for the launch)
    for (uint32_t r = threadIdx.x; r < cta.n_rows; r += blockDim.x) {
        const DRowMeta meta = sm.meta[r];
        const DConn& C = D.conns[meta.conn];
        sm.rowtgt[r] = C.plast >= 0 && D.plast[C.plast].kind == kKindTriplet ? __ldcg(D.plast[C.plast].sums + meta.pl)
                                                                              : 0.0f;
        if constexpr (LAZY) {
            sm.lzs[r] = __ldcg(C.lz_s + meta.pl);
            sm.lzm[r] = __ldcg(C.lz_m + meta.pl);
            // (the bit-placement decoding of non-negative FP8 codes yields values times 2^-120)
            sm.lzq[r] = (C.qscale ? __ldcg(C.qscale + meta.pl) : 1.0f) * (D.q_nonneg ? 0x1p120f : 1.0f);
            sm.lzqi[r] = C.qinv ? __ldcg(C.qinv + meta.pl) : 1.0f;
        }
    }
    __syncthreads();

    const unsigned long long t0 = s_t0, bar0 = s_bar0;
    const uint32_t clock0 = s_clock0;
    bool ok = true;
    if constexpr (!LAZY) {
        if (t0 == 0ull) {
            resident_row_sums(D, sm, s_blk, s_nblk);
        } else {
            move_row_sums(D, sm, s_blk, s_nblk, true);
        }
    }
    draw_noise(D, cta, t0, sm, max_own, 0u);
    __syncthreads();
#ifdef BSNN_PHASE_TIMING
    __shared__ unsigned long long s_tally_[kPhaseSlots];
    if (threadIdx.x == 0)
        for (int i = 0; i < kPhaseSlots; ++i) s_tally_[i] = 0;
    __syncthreads();
    unsigned long long t_mark_ = static_cast<unsigned long long>(clock64());
#endif
    for (uint32_t k = 0; k < n_steps; ++k) {
        const unsigned long long t = t0 + k;
        const uint32_t clock = clock0 + k;
        const uint32_t par = static_cast<uint32_t>(t & 1ull), ppar = par ^ 1u;
        const bool pending = k > 0;  // the previous step's plasticity and partials are outstanding

        // Global inputs of the step, issued together: the spike bitmask of the previous step, the
        // stimulus range of this step and the previous step's partial sums.
        const uint32_t tid = threadIdx.x, nthr = blockDim.x, spk_words = D.spk_words;
        uint32_t sb0 = 0, sb1 = 0, ev_lo = 0, ev_hi = 0;
        if (pending) {
            if (tid < spk_words) sb0 = __ldcg(D.spk_bits[ppar] + tid);
            if (tid + nthr < spk_words) sb1 = __ldcg(D.spk_bits[ppar] + tid + nthr);
        }
        if (tid == 0 && t < D.stim_len) {
            ev_lo = __ldg(D.stim_off + t);
            ev_hi = __ldg(D.stim_off + t + 1);
        }
        if (pending) load_partials(S, D, cta, ppar, sm, max_own);
        BSNN_TMARK(3);
        if (pending) {
            if (tid < spk_words) sm.sbits[tid] = sb0;
            if (tid + nthr < spk_words) sm.sbits[tid + nthr] = sb1;
            for (uint32_t w = tid + 2u * nthr; w < spk_words; w += nthr) sm.sbits[w] = __ldcg(D.spk_bits[ppar] + w);
        }
        if (tid == 0) {
            s_ev[0] = ev_lo;
            s_ev[1] = ev_hi;
        }
        rows_pending(D, cta, pending, ppar, sm, max_own);
        for (uint32_t w = tid; w < n_bits_words; w += nthr) sm.bits[w] = 0u;
        for (uint32_t w = tid; w < n_gbits; w += nthr) sm.gbits[par * n_gbits + w] = 0u;
        __syncthreads();
        BSNN_TMARK(0);
        const bool norm_now = pending && s_has_norm;
        if (norm_beside) {
            // The neuron phase on the first warps; the plasticity update and then the normalisation
            // sums on the others (they touch no data of the neuron phase).
            if (tid < 32u * neuron_warps) {
                BSNN_TSTART(t_nrn_);
                neuron_phase(S, D, cta, t, clock, par, pending, sm, max_own, L, s_ev[0], s_ev[1]);
                if (tid == 0) BSNN_TSPAN(6, t_nrn_);
                if constexpr (!LAZY) {
                    // The neuron warps go on to publish the step's spikes and put x into the row
                    // table while the update warps still work (the normalisation writes only the
                    // rows' scales).
                    if (neuron_warps > 1u) named_barrier_sync(3u, 32u * neuron_warps);
                    else __syncwarp();
                    BSNN_TSTART(t_fl_);
                    flush_spike_bits(S, D, cta, clock, par, sm, 32u * neuron_warps);
                    if (tid == 0) BSNN_TSPAN(11, t_fl_);
                    rows_x(D, cta, sm, max_own, 32u * neuron_warps);
                }
            } else if (pending) {
                BSNN_TSTART(t_upd_);
                const uint32_t nw = nwarps - neuron_warps;
                if constexpr (LAZY) apply_updates_rows(D, s_blk, s_nblk, ppar, sm, neuron_warps, nw);
                else apply_updates(D, s_blk, s_nblk, ppar, sm, neuron_warps, nw);
                if (tid == 32u * neuron_warps) BSNN_TSPAN(8, t_upd_);
                if (tid == blockDim.x - 32u) BSNN_TSPAN(13, t_upd_);
                if (norm_now) {
                    named_barrier_sync(1u, 32u * nw);
                    BSNN_TSTART(t_nrm_);
                    if constexpr (LAZY) norm_rows_lazy(D, sm, s_blk, s_nblk, neuron_warps, nw);
                    else norm_rows<CARRY>(D, sm, s_blk, s_nblk, neuron_warps, nw, n_chunks, t % kRowSumResync == 0ull);
                    if (tid == 32u * neuron_warps) BSNN_TSPAN(12, t_nrm_);
                }
                if (tid == 32u * neuron_warps) BSNN_TSPAN(7, t_upd_);
            }
            __syncthreads();
        } else {
            if (pending) {
                if constexpr (LAZY) apply_updates_rows(D, s_blk, s_nblk, ppar, sm, 0u, nwarps);
                else apply_updates(D, s_blk, s_nblk, ppar, sm, 0u, nwarps);
                __syncthreads();
            }
            neuron_phase(S, D, cta, t, clock, par, pending, sm, max_own, L, s_ev[0], s_ev[1]);
            __syncthreads();
            if (norm_now) {
                if constexpr (LAZY) norm_rows_lazy(D, sm, s_blk, s_nblk, 0u, nwarps);
                else norm_rows<CARRY>(D, sm, s_blk, s_nblk, 0u, nwarps, n_chunks, t % kRowSumResync == 0ull);
                __syncthreads();
            }
        }
        BSNN_TMARK(1);
        if (LAZY || !norm_beside) {
            BSNN_TSTART(t_fl_);
            flush_spike_bits(S, D, cta, clock, par, sm, blockDim.x);
            if (tid == 0) BSNN_TSPAN(11, t_fl_);
            rows_x(D, cta, sm, max_own, blockDim.x);
            __syncthreads();
        }
        BSNN_TMARK(2);
        {
            BSNN_TSTART(t_wp_);
            weight_pass<CARRY, LAZY>(D, cta, pending, true, par, sm, s_seg, s_blk, n_seg, n_chunks);
            if (tid == 0) BSNN_TSPAN(9, t_wp_);
            if (tid == blockDim.x - 32u) BSNN_TSPAN(10, t_wp_);
        }
        __syncthreads();
        BSNN_TMARK(4);
        grid_arrive(D.barrier, t != D.skip_step || blockIdx.x != D.skip_cta);
        BSNN_TSTART(t_win_);
        // the next step's Poisson counts while the other CTAs finish (warp 0 waits)
        if (k + 1u < n_steps) draw_noise(D, cta, t + 1ull, sm, max_own, nwarps > 1u ? 32u : 0u);
        if (tid == 32u) BSNN_TSPAN(14, t_win_);
        if (!grid_wait(D.barrier, D.error, bar0 + (k + 1ull) * gridDim.x, &s_ok)) {
            ok = false;
            break;
        }
        if (tid == 0) BSNN_TSPAN(15, t_win_);
        BSNN_TMARK(5);
    }
#ifdef BSNN_PHASE_TIMING
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < kPhaseSlots; ++i) S->phase_ns[blockIdx.x * kPhaseSlots + i] += s_tally_[i];
#endif
    if (!ok) return;

    // Finalize: apply the last step's plasticity, write resident rows and the neuron state back,
    // and fold the last propagation into g.
    const unsigned long long t_last = t0 + n_steps - 1ull;
    const uint32_t lpar = static_cast<uint32_t>(t_last & 1ull);
    stage_spike_bits(D, lpar, sm);
    rows_pending(D, cta, true, lpar, sm, max_own);
    __syncthreads();
    if constexpr (LAZY) {
        apply_updates_rows(D, s_blk, s_nblk, lpar, sm, 0u, nwarps);
        __syncthreads();
        if (s_has_norm) {
            norm_rows_lazy(D, sm, s_blk, s_nblk, 0u, nwarps);
            __syncthreads();
        }
        for (uint32_t r = threadIdx.x; r < cta.n_rows; r += blockDim.x) {
            const DRowMeta meta = sm.meta[r];
            const DConn& C = D.conns[meta.conn];
            C.lz_s[meta.pl] = sm.lzs[r];
            C.lz_m[meta.pl] = sm.lzm[r];
        }
    } else {
        apply_updates(D, s_blk, s_nblk, lpar, sm, 0u, nwarps);
        __syncthreads();
        if (s_has_norm) {
            norm_rows<CARRY>(D, sm, s_blk, s_nblk, 0u, nwarps, n_chunks, (t_last + 1ull) % kRowSumResync == 0ull);
            __syncthreads();
        }
        weight_pass<CARRY, LAZY>(D, cta, true, false, lpar, sm, s_seg, s_blk, n_seg, n_chunks);
    }
    __syncthreads();
    move_resident(D, s_blk, s_nblk, sm, false);
    if constexpr (!LAZY) move_row_sums(D, sm, s_blk, s_nblk, false);
    load_partials(S, D, cta, lpar, sm, max_own);
    __syncthreads();
    move_neuron_state(S, D, cta, sm, max_own, L, false, lpar, true);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *S->steps_done = t0 + n_steps;
        *S->clock = clock0 + n_steps;
    }
}

// Fills the tiled GEMV copy of a connection (row-scaled forms) from its FP32 masters, with the
// conversion the weight updates use; padding columns become 0.
__global__ void bsnn_fill_copy_kernel(DConn C, int32_t fmt) {
    const size_t n = static_cast<size_t>(C.qtiles) * C.n_pre * 128u;
    for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
         e += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t k = static_cast<uint32_t>(e & 127u);
        const size_t tr = e >> 7;
        const uint32_t i = static_cast<uint32_t>(tr % C.n_pre), q = static_cast<uint32_t>(tr / C.n_pre) * 128u + k;
        const float m = q < C.n_post ? C.w[static_cast<size_t>(i) * C.ld + q] : 0.0f;
        store_copy(fmt, C, i, q, m, C.qinv ? C.qinv[i] : 1.0f);
    }
}

// The communication skeleton of bsnn_step_kernel's clock step, timed to give the step a latency
// floor: per step every CTA stores its partial-sum slots (the weight pass's stores, without the
// weights), crosses the grid barrier and gathers its own columns from every slot (load_partials,
// the same code as the step kernel), with the same grid, block and plan.  Nothing else of a step
// runs, so no step can be faster than this.  It writes only the partial-sum buffers (dead between
// launches: each launch folds the pending partials into g before it ends) and the barrier counter
// (left a multiple of the grid size, as every launch leaves it).
__global__ void __launch_bounds__(kMaxThreadsRows, 1) bsnn_exchange_floor_kernel(const DSim* __restrict__ S,
                                                                                 uint32_t n_steps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Desc s_d;
    __shared__ DCta s_cta;
    __shared__ DSeg s_seg[kMaxSegsPerCta];
    __shared__ SmemLayout sm;
    __shared__ int s_ok;
    __shared__ unsigned long long s_bar0;
    const uint32_t max_own = S->max_own;
    const size_t red_bytes = align16(sizeof(float) * 2u * max_own);
    const size_t grp_bytes = align16(sizeof(DGroup) * S->n_groups);
    if (threadIdx.x == 0) {
        s_wait_limit_ns = S->wait_limit_ns;
        sm.red = reinterpret_cast<float*>(smem_raw);
        s_d.groups = reinterpret_cast<const DGroup*>(smem_raw + red_bytes);
        s_d.red_list = reinterpret_cast<const uint32_t*>(smem_raw + red_bytes + grp_bytes);
        s_d.n_groups = S->n_groups;
        s_d.partials = S->partials;
        s_d.n_slots = S->n_slots;
        s_d.N_pad = S->N_pad;
        s_d.max_own = max_own;
        s_d.barrier = S->barrier;
        s_d.error = S->error;
        for (uint32_t g = 0; g < S->n_groups; ++g) {
            s_d.goff[g] = S->groups[g].off;
            s_d.gn[g] = S->groups[g].n;
        }
        for (uint32_t T = 0; T < 2; ++T)
            for (uint32_t g = 0; g < kMaxGroups; ++g) {
                s_d.red_begin[T][g] = S->red_begin[T][g];
                s_d.red_end[T][g] = S->red_end[T][g];
            }
        s_cta = S->ctas[blockIdx.x];
        for (uint32_t s = s_cta.seg_begin; s < s_cta.seg_end; ++s) s_seg[s - s_cta.seg_begin] = S->segs[s];
        const unsigned long long n = gridDim.x;
        s_bar0 = ld_acquire_u64(S->barrier) / n * n;
    }
    __syncthreads();
    copy_words(smem_raw + red_bytes, S->groups, sizeof(DGroup) * S->n_groups);
    copy_words(smem_raw + red_bytes + grp_bytes, S->red_list, sizeof(uint32_t) * S->n_red);
    __syncthreads();
    const Desc& D = s_d;
    const DCta& cta = s_cta;
    const uint32_t n_seg = cta.seg_end - cta.seg_begin;
    for (uint32_t k = 0; k < n_steps; ++k) {
        const uint32_t par = k & 1u;
        float* part_out = D.partials + static_cast<size_t>(par) * D.n_slots * D.N_pad;
        const float v = sm.red[threadIdx.x % (2u * max_own > 0u ? 2u * max_own : 1u)];
        for (uint32_t s = 0; s < n_seg; ++s) {
            const DSeg& SG = s_seg[s];
            float4* out = reinterpret_cast<float4*>(part_out + static_cast<size_t>(SG.slot) * D.N_pad + SG.pcol);
            for (uint32_t u = threadIdx.x; u < SG.units; u += blockDim.x) __stcg(out + u, make_float4(v, v, v, v));
        }
        if (!grid_barrier(D.barrier, D.error, s_bar0 + (k + 1ull) * gridDim.x, &s_ok)) return;
        load_partials(S, D, cta, par, sm, max_own);
        __syncthreads();
    }
}

// Sets the clock_step of the next step (bsnn_run with a first_clock_step that does not follow
// the previous call).
__global__ void bsnn_set_clock_kernel(uint32_t* clock, uint32_t value) { *clock = value; }

}  // namespace bsnn
