// bsnn_device.cuh -- device-side description of one simulated network (the "arena" layout).
//
// One DSim lives in device memory per bsnn_sim.  All per-neuron state is structure-of-arrays
// over the global neuron index (the reference's GpuSimulationState layout,
// cpp_src/gpu_core/gpu_simulation_state.cu:35-86); between launches it is canonical there, and
// during a launch each CTA keeps its own neurons' copy in shared memory.  What differs from the
// reference:
//  * weight matrices are row-major [pre][ld] with ld = num_post rounded up to 4 floats, so every
//    row starts on a 16-byte boundary and is read with 128-bit loads;
//  * values that other CTAs read inside one persistent launch (spikes, plasticity column and
//    row factors, GEMV partial sums) are double-buffered by step parity;
//  * the per-step work of every component is planned once into per-CTA work lists (DCta,
//    DSeg, DBlk) so the fused kernel needs one grid barrier per step.
#pragma once

#include <cstdint>

namespace bsnn {

constexpr int kMaxGroups = 8;
constexpr int kMaxConns = 16;
constexpr int kMaxTraceSets = 16;
constexpr int kMaxPlast = 16;
constexpr int kMaxMonitors = 16;
constexpr int kMaxGroupRoles = 4;  // trace sets / plasticities / monitors per group and role
constexpr int kMaxSegsPerCta = 2 * kMaxGroups;
constexpr int kMaxBlksPerCta = kMaxConns;
constexpr int kPhaseSlots = 16;  // per-CTA phase tallies of the step kernel (profiling builds)
// Threads per CTA: the step-kernel instance that carries row sums needs up to 255 registers per
// thread (256 threads); the others fit in 168 registers (three warps share one scheduler's
// quarter of the register file): 288 threads for the reference form, 384 for the row-scaled
// forms.
constexpr int kMaxThreads = 256;
constexpr int kMaxThreadsPlain = 288;
constexpr int kMaxThreadsRows = 384;

enum : int32_t { kTargetExc = 0, kTargetInh = 1 };
enum : int32_t { kKindTriplet = 1, kKindIstdp = 2, kKindStdp = 3 };
enum : int32_t { kMonSpikes = 0, kMonVoltage = 1 };
enum : int32_t { kNoisePhilox = 0, kNoiseOff = 1, kNoiseReplay = 2 };
enum : int32_t { kErrNone = 0, kErrBarrierTimeout = 1, kErrStageTimeout = 2 };
// Weight storage forms.  kFmtF32: the reference's arithmetic (every normalised row rescaled and
// stored each step).  The others keep an FP32 master m per weight and a per-row normalisation
// scale s (the weight is s m), so the normalisation touches one number per row; the GEMV reads a
// copy of m in FP32, BF16, or FP8 E4M3 with a per-row quantisation scale.
enum : int32_t { kFmtF32 = 0, kFmtF32Rows = 1, kFmtBf16 = 2, kFmtFp8 = 3 };

// NeuronGroupView scalars (cpp_src/neuron_groups/neuron_group_view.h:8-49) plus derived values.
struct DGroup {
    uint32_t off, n;      // global slice
    uint32_t pcol;        // first column of this group in the padded partial-sum rows
    uint32_t inhib;
    uint32_t refractory_steps;
    uint32_t has_bg_e, has_bg_i;  // mean_background_* > 0
    float timestep, g_leak, cap, delta_t, v_eff, e_exc, e_inh, v_th, v_reset, v_rest;
    float exp_neg_mean_e, exp_neg_mean_i;  // exp(-mean) for the Poisson sampler
    float bg_er_decay, bg_ed_decay, bg_ir_decay, bg_id_decay, bg_scale_e, bg_scale_i;
    uint32_t n_ts;                 // trace sets fed by this group (as presynaptic group)
    int32_t ts[kMaxGroupRoles];
    uint32_t n_plast_pre;          // plasticities whose presynaptic group is this group
    int32_t plast_pre[kMaxGroupRoles];
    uint32_t n_plast_post;         // plasticities whose postsynaptic group is this group
    int32_t plast_post[kMaxGroupRoles];
    uint32_t n_mon;                // monitors on this group
    int32_t mon[kMaxGroupRoles];
};

// Connection traces (ConnectionView r/d/summed arrays, cpp_src/connections/connection_view.h:8-31).
// Connections from the same presynaptic group with identical decays and normalisation share one
// set, since the reference computes bit-identical values for them.
struct DTraceSet {
    uint32_t group;
    float r_decay, d_decay, norm;
    float* r;  // [n_pre]
    float* d;  // [n_pre]
    float* x;  // [n_pre]  summed_postsynaptic_conductances = d - r
};

struct DConn {
    uint32_t pre_g, post_g, pre_off, n_pre, post_off, n_post;
    uint32_t ld;      // floats per stored row (multiple of 4)
    uint32_t units;   // ld / 4
    uint32_t target;  // kTargetExc or kTargetInh (from the presynaptic group's is_inhibitory)
    int32_t ts;       // trace set
    int32_t plast;    // plasticity acting on this connection or -1
    float* w;         // [n_pre][ld]
    // Row-scaled forms (kFmtF32Rows, kFmtBf16, kFmtFp8): the GEMV copy of the masters in
    // 128-column tiles, element (row i, column q) at ((q / 128) * n_pre + i) * 128 + q % 128, so
    // the rows of one tile are contiguous and a run of rows of one 32-unit chunk is one block of
    // memory; columns past n_post are 0.
    void* q;
    uint32_t qtiles;  // ceil(n_post / 128)
    float* qscale;    // [n_pre] FP8: per-row quantisation scale (value = e4m3 * qscale), else null
    float* qinv;      // [n_pre] its reciprocal
    float* lz_s;      // [n_pre] normalisation scale s of each row
    float* lz_m;      // [n_pre] sum of the row's masters
    // Reference form, triplet connections: [n_pre] running sum of each row's weights between
    // launches (rows resident in shared memory keep it in step; see norm_rows), else null.
    float* rowsum;
};

// PlasticityView (cpp_src/plasticities/plasticity_view.h:8-38) plus per-step factor buffers.
// Row factors (per presynaptic neuron, kept in the owning CTA's shared memory) and column factors
// (per postsynaptic neuron, parity buffers here) are formed once per step by the neuron that owns
// them, so that every weight update is
//   LTP: w = clamp(fma(rowA, colA, w))   if the post neuron spiked
//   LTD: w = clamp(fma(colB, rowB, w))   if the pre neuron spiked
// which is the reference's delta expression with its factors grouped the way it computes them.
struct DPlast {
    int32_t kind;
    uint32_t conn;
    float ltp_A, ltd_A, ltp_B, ltd_B;
    float pre_decay, post_decay, tpre_decay, tpost_decay;
    float wmin, wmax;
    float* pre;    // [n_pre]  pre traces (state after the step's increment)
    float* post;   // [n_post]
    float* tpre;   // [n_pre]  triplet traces (triplet rule only)
    float* tpost;  // [n_post]
    float* colA[2];     // [units*4] parity buffers (padded)
    float* colB[2];
    float* sums;        // [n_pre] normalisation targets (triplet)
};

struct DMon {
    int32_t kind;
    uint32_t group, interval;
    uint32_t words;   // spike ring: ceil(n_group / 32) words per slot
    uint32_t n_sel;   // voltage ring: selected neurons per slot
    uint32_t* bits;   // [interval][words]
    float* vh;        // [interval][n_sel]
    int32_t* sel_idx; // [n_group] slot column of a neuron or -1
};

// Per-CTA work plan.
struct DSeg {  // all rows of this CTA that add into (target, post group)
    uint32_t target, post_g, pcol, n_post, units;
    uint32_t item_begin;  // first work item (32-aligned)
    uint32_t slot;        // partial-sum slot this CTA writes for `target`
    uint32_t blk_begin, blk_end;
    uint32_t normalized;  // some block of this segment carries the triplet row normalisation
    uint32_t carried;     // some triplet block of this segment streams from global memory
};
struct DBlk {  // rows [row_begin, row_end) (presynaptic local index) of one connection
    uint32_t conn, row_begin, row_end;
    uint32_t srow;      // index of row_begin in the CTA's row table
    uint32_t resident;  // rows held in shared memory for the whole launch
    uint32_t sm_off;    // float offset of row_begin in the resident region
    uint32_t trow;      // index of row_begin among the CTA's triplet-normalised rows
};
struct DCta {
    uint32_t n0, n1;  // owned neurons (phase A) == owned presynaptic rows (phase B)
    uint32_t seg_begin, seg_end;
    uint32_t n_rows, n_items;
};

struct DRowMeta {
    uint32_t conn, pl, j;  // connection, presynaptic local row, global neuron
};

struct DSim {
    uint32_t N, N_pad;
    uint32_t n_groups, n_conns, n_ts, n_plast, n_mons;
    uint32_t n_ctas, n_slots, max_rows, max_own;
    uint32_t resident_floats;  // shared-memory floats reserved for resident weight rows (per CTA)
    // Largest per-group role counts (trace sets, plasticities as pre / post side, voltage
    // monitors): they size the per-neuron state each CTA keeps in shared memory during a launch.
    uint32_t ns_ts, ns_pre, ns_post, ns_mon;
    // Carried triplet row sums: most triplet rows of one CTA, and 32-unit chunks per row.
    uint32_t max_trows, n_chunks;
    // Streamed rows staged through shared memory by bulk asynchronous copies: rows per buffer
    // (two buffers per warp), 0 = off (no shared memory left over).
    uint32_t stage_rows;
    uint32_t stage_warps;  // warps per CTA (the staging buffers are per warp)
    int32_t wfmt;          // weight storage form (kFmt*)
    // FP8 form with no negative weight possible (every weight and every plastic weight_min >= 0):
    // the copy is decoded by bit placement, exact up to a factor 2^-120 that the row weights carry.
    uint32_t q_nonneg;
    DGroup groups[kMaxGroups];
    DTraceSet ts[kMaxTraceSets];
    DConn conns[kMaxConns];
    DPlast plast[kMaxPlast];
    DMon mons[kMaxMonitors];

    // per-neuron state [N]
    float *v, *ge, *gi, *istim;
    float *bg_ge, *bg_gi, *bg_er, *bg_ed, *bg_ir, *bg_id;
    uint32_t* refrac;
    uint32_t* spikes[2];  // parity buffers; the last step's are the canonical spikes
    uint32_t* spk_bits[2];  // parity buffers: network-wide spike bitmask of a step [spk_words]
    uint32_t spk_words;     // ceil(N / 32) + 2 (one spare word for 64-bit funnel reads)

    float* partials;  // [2][n_slots][N_pad]
    uint32_t* red_list;  // slot lists per (target, group)
    uint32_t n_red;      // entries of red_list
    uint32_t red_begin[2][kMaxGroups], red_end[2][kMaxGroups];

    const DCta* ctas;
    const DSeg* segs;
    const DBlk* blks;
    const DRowMeta* rows;  // per CTA, starting at rows_begin[cta]
    const uint32_t* rows_begin;

    // stimulus: events of internal step t are ev_*[stim_off[t] .. stim_off[t+1]), sorted by neuron
    uint32_t stim_len;
    const uint32_t* stim_off;
    const uint32_t* ev_neuron;
    const float* ev_delta;

    int32_t noise_mode;
    uint32_t seed;
    const uint8_t* replay;  // [replay_steps][N][2]
    uint32_t replay_steps;

    unsigned long long* barrier;  // monotonically increasing arrival counter
    int32_t* error;
    unsigned long long* steps_done;  // internal step counter (stimulus / noise cursor)
    uint32_t* clock;                 // clock_step of the next step
    unsigned long long* phase_ns;    // [n_ctas][kPhaseSlots] phase clock tallies (profiling builds only)
    unsigned long long wait_limit_ns;  // bound of every device-side wait of a launch
    // Test switch (bsnn_debug_skip_arrival): CTA skip_cta does not arrive at the grid barrier that
    // closes internal step skip_step, so every CTA's bounded wait runs out.  ~0 = off.
    unsigned long long skip_step;
    uint32_t skip_cta;
};

}  // namespace bsnn
