// bsnn_api.cu -- host side of libbsnn: the C-ABI of include/bsnn.h.
//
// Component calls only record host-side descriptions.  The first call that needs the device
// (a step, a read) "finalizes" the sim: it plans the per-CTA work of the fused step kernel,
// allocates ONE device arena for all state, and uploads everything, i.e. what the reference
// spreads over GpuSimulationState::initialize_device_buffers and the upload_*_view helpers
// (cpp_src/gpu_core/gpu_simulation_state.cu:35-86, 107-208).  After that, components can no
// longer be added.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/bsnn.h"
#include "bsnn_device.cuh"
#include "propagate.cuh"
#include "propagate_static.cuh"
#include "records.h"
#include "step_kernel.cuh"

using namespace bsnn;

namespace {

struct ApiError : std::runtime_error {
    bsnn_status code;
    ApiError(bsnn_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw ApiError(BSNN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

thread_local std::string g_thread_error;

uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

struct HostGroup {
    bsnn_neuron_group_params p;
};
struct HostConn {
    uint32_t pre, post;
    bsnn_connection_params p;
    std::vector<float> w;  // row-major [n_pre][n_post]
    float r_decay, d_decay, norm;
};
struct HostPlast {
    int32_t kind;
    uint32_t conn;
    bsnn_plasticity_params p;
};
struct HostMon {
    int32_t kind;
    uint32_t group, interval;
    std::vector<uint32_t> sel;
    std::string path;                        // output file (set by bsnn_set_monitor_output)
    std::shared_ptr<std::ofstream> spike_out;  // spike recorder's open file
};
struct HostWeightRec {
    uint32_t conn;
    std::string path;
};
struct HostStim {
    std::vector<uint32_t> counts, ids, offs;
    std::vector<float> deltas;
};

// Simple bump allocator over the device arena.
struct Arena {
    size_t size = 0;
    size_t take(size_t bytes) {
        const size_t off = (size + 255) & ~size_t(255);
        size = off + bytes;
        return off;
    }
};

}  // namespace

struct bsnn_sim {
    bsnn_state_desc desc{};
    uint32_t N = 0;
    std::string err;
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;

    std::vector<HostGroup> groups;
    std::vector<HostConn> conns;
    std::vector<HostPlast> plasts;
    std::vector<HostMon> mons;
    std::vector<HostWeightRec> wrecs;
    std::unique_ptr<rec::Writer> writer;  // formats and writes recorded text off the stepping thread
    std::vector<HostStim> stims;
    int32_t noise_mode = BSNN_NOISE_PHILOX;
    int32_t weight_format = BSNN_WEIGHTS_F32;
    std::vector<uint8_t> replay;
    uint32_t replay_steps = 0;

    bool finalized = false;
    bool failed = false;
    unsigned char* arena = nullptr;
    size_t arena_bytes = 0;
    size_t weight_bytes = 0;
    DSim h{};
    DSim* d_sim = nullptr;
    uint32_t grid = 0, block = 0;
    size_t smem_bytes = 0;
    const void* kernel = nullptr;  // the bsnn_step_kernel instantiation chosen for this network
    uint64_t steps_done = 0;
    uint32_t next_clock = 0;
    uint32_t steps_per_launch = 1000;
    uint64_t launches = 0;
    bool progress = false;  // bsnn_run_system prints System::run's progress line
    uint64_t wait_limit_ns = kDefaultWaitLimitNs;  // bound of every device-side wait
    uint64_t skip_step = ~0ull;                      // test switch (bsnn_debug_skip_arrival)
    uint32_t skip_cta = 0;
    bool graphs_ok = true;
    std::map<uint32_t, cudaGraphExec_t> graphs;
    std::vector<uint32_t> conn_ld;

    ~bsnn_sim() {
        writer.reset();  // finishes the queued writes
        for (auto& m : mons)
            if (m.spike_out) m.spike_out->flush();
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        if (arena) cudaFree(arena);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

template <class F>
bsnn_status guarded(bsnn_sim* sim, F&& f) {
    try {
        if (sim) {
            DeviceGuard g(sim->device);
            f();
        } else {
            f();
        }
        return BSNN_OK;
    } catch (const ApiError& e) {
        if (sim) sim->err = e.what();
        g_thread_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        if (sim) sim->err = e.what();
        g_thread_error = e.what();
        return BSNN_ERR_RUNTIME;
    }
}

void require(bool cond, bsnn_status code, const std::string& msg) {
    if (!cond) throw ApiError(code, msg);
}
// A literal message builds its std::string only when the check fails (checks run once per weight).
void require(bool cond, bsnn_status code, const char* msg) {
    if (!cond) throw ApiError(code, std::string(msg));
}

void require_building(const bsnn_sim* s) {
    require(!s->finalized, BSNN_ERR_STATE, "components cannot be added after the simulation has started");
}

float exp_neg_mean_of(float mean) { return static_cast<float>(std::exp(-static_cast<double>(mean))); }

// ------------------------------------------------------------------------------------------
// Planning: neuron ownership, per-CTA segments/blocks/rows, slot lists.
struct Plan {
    std::vector<DCta> ctas;
    std::vector<DSeg> segs;
    std::vector<DBlk> blks;
    std::vector<DRowMeta> rows;
    std::vector<uint32_t> rows_begin;
    std::vector<uint32_t> red_list;
    uint32_t red_begin[2][kMaxGroups]{}, red_end[2][kMaxGroups]{};
    uint32_t n_slots = 0, max_rows = 1, max_own = 1, max_items = 1, max_trows = 0, n_chunks = 0;
    uint64_t resident_floats = 0;
};

int group_of_host(const bsnn_sim* s, uint32_t j) {
    for (size_t g = 0; g < s->groups.size(); ++g) {
        const auto& p = s->groups[g].p;
        if (j >= p.offset && j - p.offset < p.num_neurons) return static_cast<int>(g);
    }
    return -1;
}

// Partitions the neurons into n_ctas contiguous ranges balancing `cost`; when `cap_bytes` > 0 the
// plastic rows of every range must also fit in cap_bytes of shared memory, and neurons flagged in
// `cut` must start a range (returns false if not possible).
bool greedy_partition(const std::vector<double>& cost, const std::vector<uint64_t>& res_bytes,
                      const std::vector<char>& cut, uint32_t n_ctas, double max_cost, uint64_t cap_bytes,
                      std::vector<uint32_t>& bounds) {
    const uint32_t N = static_cast<uint32_t>(cost.size());
    bounds.assign(n_ctas + 1, N);
    bounds[0] = 0;
    uint32_t c = 0;
    double acc = 0.0;
    uint64_t acc_res = 0;
    for (uint32_t j = 0; j < N; ++j) {
        if (cost[j] > max_cost || (cap_bytes > 0 && res_bytes[j] > cap_bytes)) return false;
        if ((cut[j] && j > 0 && acc > 0.0) || acc + cost[j] > max_cost ||
            (cap_bytes > 0 && acc_res + res_bytes[j] > cap_bytes)) {
            if (++c >= n_ctas) return false;
            bounds[c] = j;
            acc = 0.0;
            acc_res = 0;
        }
        acc += cost[j];
        acc_res += res_bytes[j];
    }
    for (uint32_t k = c + 1; k <= n_ctas; ++k) bounds[k] = N;
    return true;
}

// Contiguous partition of the neurons into n_ctas ranges that minimises the largest per-range
// cost (binary search on that maximum); with cap_bytes > 0 every range's plastic rows must also
// fit in cap_bytes of shared memory, and every range holds neurons of one group only (a range
// that spans two groups carries both groups' work and slows the whole grid).  Returns false if
// no such partition exists.
bool partition(const std::vector<double>& cost, const std::vector<uint64_t>& res_bytes, const std::vector<char>& cut,
               uint32_t n_ctas, uint64_t cap_bytes, std::vector<uint32_t>& bounds) {
    double total = 0.0, biggest = 0.0;
    for (double c : cost) {
        total += c;
        biggest = std::max(biggest, c);
    }
    double lo = std::max(biggest, total / n_ctas), hi = total + 1.0;
    if (!greedy_partition(cost, res_bytes, cut, n_ctas, hi, cap_bytes, bounds)) return false;
    for (int it = 0; it < 60 && hi - lo > 1e-6 * hi; ++it) {
        const double mid = 0.5 * (lo + hi);
        std::vector<uint32_t> b;
        if (greedy_partition(cost, res_bytes, cut, n_ctas, mid, cap_bytes, b)) hi = mid;
        else lo = mid;
    }
    return greedy_partition(cost, res_bytes, cut, n_ctas, hi, cap_bytes, bounds);
}

Plan build_plan(const bsnn_sim* s, uint32_t n_ctas, uint64_t cap_bytes, bool* resident_ok) {
    Plan P;
    const uint32_t N = s->N;
    // Per-neuron cost of its outgoing rows: one weight read, plus write and (normalised) re-read
    // for plastic rows.
    std::vector<double> cost(N, 1.0);
    for (uint32_t j = 0; j < N; ++j) {
        const int g = group_of_host(s, j);
        if (g < 0) continue;
        for (size_t c = 0; c < s->conns.size(); ++c) {
            const auto& C = s->conns[c];
            if (static_cast<int>(C.pre) != g) continue;
            double w = 1.0;  // (row-scaled forms only read their rows)
            for (const auto& pl : s->plasts)
                if (pl.conn == c && s->weight_format == BSNN_WEIGHTS_F32) w += pl.kind == BSNN_PLASTICITY_TRIPLET ? 2.0 : 1.0;
            cost[j] += w * round_up(s->groups[C.post].p.num_neurons, 4);
        }
    }
    // Shared-memory bytes of each neuron's plastic rows (resident candidates).
    std::vector<uint64_t> res_bytes(N, 0);
    for (uint32_t j = 0; j < N; ++j) {
        const int g = group_of_host(s, j);
        if (g < 0) continue;
        for (size_t c = 0; c < s->conns.size(); ++c) {
            const auto& C = s->conns[c];
            if (static_cast<int>(C.pre) != g) continue;
            bool plastic = false;
            for (const auto& pl : s->plasts) plastic |= pl.conn == c;
            if (plastic) res_bytes[j] += 4ull * round_up(s->groups[C.post].p.num_neurons, 4);
        }
    }
    std::vector<uint32_t> bounds;
    std::vector<char> cut(N, 0), no_cut(N, 0);
    for (const auto& g : s->groups)
        if (g.p.offset < N) cut[g.p.offset] = 1;
    bool resident = cap_bytes > 0 && (partition(cost, res_bytes, cut, n_ctas, cap_bytes, bounds) ||
                                      partition(cost, res_bytes, no_cut, n_ctas, cap_bytes, bounds));
    if (!resident && !partition(cost, res_bytes, cut, n_ctas, 0, bounds))
        partition(cost, res_bytes, no_cut, n_ctas, 0, bounds);
    if (resident_ok) *resident_ok = resident;

    // Slot bookkeeping: slot of (cta, target), and which (target, group) each CTA feeds.
    std::vector<std::vector<uint32_t>> red(2 * kMaxGroups);
    for (uint32_t c = 0; c < n_ctas; ++c) {
        DCta cta{};
        cta.n0 = bounds[c];
        cta.n1 = bounds[c + 1];
        cta.seg_begin = static_cast<uint32_t>(P.segs.size());
        P.rows_begin.push_back(static_cast<uint32_t>(P.rows.size()));
        const uint32_t row_base = static_cast<uint32_t>(P.rows.size());
        int32_t slot_of_target[2] = {-1, -1};
        uint32_t item = 0, trows = 0;
        for (uint32_t T = 0; T < 2; ++T) {
            for (uint32_t q = 0; q < s->groups.size(); ++q) {
                DSeg seg{};
                seg.target = T;
                seg.post_g = q;
                seg.blk_begin = static_cast<uint32_t>(P.blks.size());
                for (uint32_t ci = 0; ci < s->conns.size(); ++ci) {
                    const auto& C = s->conns[ci];
                    const auto& gp = s->groups[C.pre].p;
                    const uint32_t target = gp.is_inhibitory ? kTargetInh : kTargetExc;
                    if (target != T || C.post != q) continue;
                    const uint32_t a = std::max(cta.n0, gp.offset);
                    const uint32_t b = std::min(cta.n1, gp.offset + gp.num_neurons);
                    if (a >= b) continue;
                    DBlk blk{};
                    blk.conn = ci;
                    blk.row_begin = a - gp.offset;
                    blk.row_end = b - gp.offset;
                    blk.srow = static_cast<uint32_t>(P.rows.size()) - row_base;
                    for (uint32_t pl = blk.row_begin; pl < blk.row_end; ++pl)
                        P.rows.push_back(DRowMeta{ci, pl, gp.offset + pl});
                    for (const auto& pl : s->plasts)
                        if (pl.conn == ci && pl.kind == BSNN_PLASTICITY_TRIPLET) seg.normalized = 1;
                    P.blks.push_back(blk);
                }
                seg.blk_end = static_cast<uint32_t>(P.blks.size());
                if (seg.blk_end == seg.blk_begin) continue;
                const auto& gq = s->groups[q].p;
                // first column of group q in the padded partial rows (groups in index order,
                // each rounded up to 4 columns; the same layout finalize() gives DGroup::pcol)
                seg.pcol = 0;
                for (uint32_t g2 = 0; g2 < q; ++g2) seg.pcol += round_up(s->groups[g2].p.num_neurons, 4);
                seg.n_post = gq.num_neurons;
                seg.units = round_up(gq.num_neurons, 4) / 4;
                seg.item_begin = item;
                item += round_up(seg.units, 32);
                if (slot_of_target[T] < 0) slot_of_target[T] = static_cast<int32_t>(P.n_slots++);
                seg.slot = static_cast<uint32_t>(slot_of_target[T]);
                red[T * kMaxGroups + q].push_back(seg.slot);
                P.segs.push_back(seg);
            }
        }
        cta.seg_end = static_cast<uint32_t>(P.segs.size());
        cta.n_rows = static_cast<uint32_t>(P.rows.size()) - row_base;
        if (resident) {
            // plastic blocks first, then read-only blocks while they still fit under the cap
            const uint32_t b0 = cta.seg_end > cta.seg_begin ? P.segs[cta.seg_begin].blk_begin : 0u;
            const uint32_t b1 = cta.seg_end > cta.seg_begin ? P.segs[cta.seg_end - 1].blk_end : 0u;
            uint64_t used = 0;
            for (int pass = 0; pass < 2; ++pass)
                for (uint32_t bk = b0; bk < b1; ++bk) {
                    DBlk& B = P.blks[bk];
                    bool plastic = false;
                    for (const auto& pl : s->plasts) plastic |= pl.conn == B.conn;
                    if (plastic != (pass == 0)) continue;
                    const uint64_t bytes = 4ull * (B.row_end - B.row_begin) *
                                           round_up(s->groups[s->conns[B.conn].post].p.num_neurons, 4);
                    if (used + bytes > cap_bytes) continue;
                    B.resident = 1;
                    B.sm_off = static_cast<uint32_t>(used / 4);
                    used += bytes;
                }
            P.resident_floats = std::max<uint64_t>(P.resident_floats, used / 4);
        }
        // Streamed triplet blocks carry their row sums between steps (32-unit chunks per row).
        {
            const uint32_t b0 = cta.seg_end > cta.seg_begin ? P.segs[cta.seg_begin].blk_begin : 0u;
            const uint32_t b1 = cta.seg_end > cta.seg_begin ? P.segs[cta.seg_end - 1].blk_end : 0u;
            for (uint32_t bk = b0; bk < b1; ++bk) {
                DBlk& B = P.blks[bk];
                bool triplet = false;
                for (const auto& pl : s->plasts) triplet |= pl.conn == B.conn && pl.kind == BSNN_PLASTICITY_TRIPLET;
                if (!triplet || B.resident) continue;
                for (uint32_t sg = cta.seg_begin; sg < cta.seg_end; ++sg)
                    if (bk >= P.segs[sg].blk_begin && bk < P.segs[sg].blk_end) P.segs[sg].carried = 1;
                B.trow = trows;
                trows += B.row_end - B.row_begin;
                const uint32_t units = round_up(s->groups[s->conns[B.conn].post].p.num_neurons, 4) / 4;
                P.n_chunks = std::max(P.n_chunks, (units + 31) / 32);
            }
        }
        cta.n_items = item;
        require(cta.seg_end - cta.seg_begin <= static_cast<uint32_t>(kMaxSegsPerCta), BSNN_ERR_INVALID_ARGUMENT,
                "too many (target, post group) segments per CTA");
        const uint32_t nblk = cta.seg_end > cta.seg_begin
                                  ? P.segs[cta.seg_end - 1].blk_end - P.segs[cta.seg_begin].blk_begin
                                  : 0u;
        require(nblk <= static_cast<uint32_t>(kMaxBlksPerCta), BSNN_ERR_INVALID_ARGUMENT,
                "too many connection blocks per CTA");
        P.max_rows = std::max(P.max_rows, cta.n_rows);
        P.max_trows = std::max(P.max_trows, trows);
        P.max_own = std::max(P.max_own, cta.n1 - cta.n0);
        P.max_items = std::max(P.max_items, cta.n_items);
        P.ctas.push_back(cta);
    }
    for (uint32_t T = 0; T < 2; ++T)
        for (uint32_t q = 0; q < kMaxGroups; ++q) {
            P.red_begin[T][q] = static_cast<uint32_t>(P.red_list.size());
            for (uint32_t sl : red[T * kMaxGroups + q]) P.red_list.push_back(sl);
            P.red_end[T][q] = static_cast<uint32_t>(P.red_list.size());
        }
    if (P.red_list.empty()) P.red_list.push_back(0);
    if (P.rows.empty()) P.rows.push_back(DRowMeta{0, 0, 0});
    return P;
}

void launch_fill_copy(const DConn& C, int32_t fmt, cudaStream_t stream) {
    const size_t n = static_cast<size_t>(C.qtiles) * C.n_pre * 128u;
    const unsigned blocks = static_cast<unsigned>(std::min<size_t>((n + 255) / 256, 4096));
    bsnn_fill_copy_kernel<<<blocks, 256, 0, stream>>>(C, fmt);
    cuda_check(cudaGetLastError(), "fill weight copy");
}

void finalize(bsnn_sim* s) {
    if (s->finalized) return;
    require(!s->groups.empty(), BSNN_ERR_STATE, "no neuron groups were added");
    const uint32_t N = s->N;
    DSim& h = s->h;
    h = DSim{};
    h.N = N;
    h.n_groups = static_cast<uint32_t>(s->groups.size());
    h.n_conns = static_cast<uint32_t>(s->conns.size());
    h.n_plast = static_cast<uint32_t>(s->plasts.size());
    h.n_mons = static_cast<uint32_t>(s->mons.size());

    // Groups and their padded partial-sum columns.
    uint32_t pcol = 0;
    for (uint32_t g = 0; g < h.n_groups; ++g) {
        const auto& p = s->groups[g].p;
        DGroup& G = h.groups[g];
        G.off = p.offset;
        G.n = p.num_neurons;
        G.pcol = pcol;
        pcol += round_up(p.num_neurons, 4);
        G.inhib = p.is_inhibitory ? 1u : 0u;
        G.refractory_steps = p.refractory_steps;
        G.has_bg_e = p.mean_background_excitatory_spikes > 0.0f;
        G.has_bg_i = p.mean_background_inhibitory_spikes > 0.0f;
        G.timestep = p.timestep;
        G.g_leak = p.g_leak;
        G.cap = p.membrane_capacitance;
        G.delta_t = p.depolarization_slope_factor;
        G.v_eff = p.v_effective_spike_threshold;
        G.e_exc = p.v_excitatory_reversal;
        G.e_inh = p.v_inhibitory_reversal;
        G.v_th = p.v_threshold;
        G.v_reset = p.v_reset;
        G.v_rest = p.v_rest;
        G.exp_neg_mean_e = exp_neg_mean_of(p.mean_background_excitatory_spikes);
        G.exp_neg_mean_i = exp_neg_mean_of(p.mean_background_inhibitory_spikes);
        G.bg_er_decay = p.background_excitatory_postsynaptic_r_trace_decay;
        G.bg_ed_decay = p.background_excitatory_postsynaptic_d_trace_decay;
        G.bg_ir_decay = p.background_inhibitory_postsynaptic_r_trace_decay;
        G.bg_id_decay = p.background_inhibitory_postsynaptic_d_trace_decay;
        G.bg_scale_e = p.background_excitatory_scaling_factor;
        G.bg_scale_i = p.background_inhibitory_scaling_factor;
    }
    h.N_pad = std::max(pcol, 4u);

    // Trace sets (shared by connections with the same presynaptic group and trace constants).
    std::vector<int32_t> conn_ts(h.n_conns, -1);
    for (uint32_t c = 0; c < h.n_conns; ++c) {
        const auto& C = s->conns[c];
        for (uint32_t t = 0; t < h.n_ts; ++t) {
            const DTraceSet& T = h.ts[t];
            if (T.group == C.pre && T.r_decay == C.r_decay && T.d_decay == C.d_decay && T.norm == C.norm) {
                conn_ts[c] = static_cast<int32_t>(t);
                break;
            }
        }
        if (conn_ts[c] < 0) {
            require(h.n_ts < static_cast<uint32_t>(kMaxTraceSets), BSNN_ERR_INVALID_ARGUMENT, "too many trace sets");
            DTraceSet& T = h.ts[h.n_ts];
            T.group = C.pre;
            T.r_decay = C.r_decay;
            T.d_decay = C.d_decay;
            T.norm = C.norm;
            DGroup& G = h.groups[C.pre];
            require(G.n_ts < static_cast<uint32_t>(kMaxGroupRoles), BSNN_ERR_INVALID_ARGUMENT, "too many trace sets per group");
            G.ts[G.n_ts++] = static_cast<int32_t>(h.n_ts);
            conn_ts[c] = static_cast<int32_t>(h.n_ts++);
        }
    }

    // Device arena layout.
    Arena A;
    const size_t fN = sizeof(float) * N;
    size_t o_v = A.take(fN), o_ge = A.take(fN), o_gi = A.take(fN), o_is = A.take(fN);
    size_t o_bge = A.take(fN), o_bgi = A.take(fN), o_ber = A.take(fN), o_bed = A.take(fN), o_bir = A.take(fN),
           o_bid = A.take(fN);
    size_t o_ref = A.take(sizeof(uint32_t) * N);
    size_t o_spk0 = A.take(sizeof(uint32_t) * N), o_spk1 = A.take(sizeof(uint32_t) * N);
    const uint32_t spk_words = (N + 31) / 32 + 2;
    size_t o_sb0 = A.take(sizeof(uint32_t) * spk_words), o_sb1 = A.take(sizeof(uint32_t) * spk_words);
    std::vector<size_t> o_ts(h.n_ts * 3);
    for (uint32_t t = 0; t < h.n_ts; ++t) {
        const size_t n = sizeof(float) * s->groups[h.ts[t].group].p.num_neurons;
        o_ts[3 * t] = A.take(n);
        o_ts[3 * t + 1] = A.take(n);
        o_ts[3 * t + 2] = A.take(n);
    }
    std::vector<size_t> o_w(h.n_conns), o_q(h.n_conns, 0), o_rowv(h.n_conns, 0), o_rsum(h.n_conns, 0);
    const bool lazy = s->weight_format != BSNN_WEIGHTS_F32;
    s->conn_ld.assign(h.n_conns, 0);
    size_t wbytes = 0;
    for (uint32_t c = 0; c < h.n_conns; ++c) {
        const auto& C = s->conns[c];
        const uint32_t n_pre = s->groups[C.pre].p.num_neurons, n_post = s->groups[C.post].p.num_neurons;
        const uint32_t ld = round_up(n_post, 4);
        s->conn_ld[c] = ld;
        o_w[c] = A.take(sizeof(float) * static_cast<size_t>(n_pre) * ld);
        wbytes += sizeof(float) * static_cast<size_t>(n_pre) * ld;
        if (lazy) {
            const size_t eb = s->weight_format == BSNN_WEIGHTS_BF16 ? 2 : s->weight_format == BSNN_WEIGHTS_FP8_E4M3 ? 1 : 4;
            const size_t tiles = (n_post + 127) / 128;
            o_q[c] = A.take(eb * tiles * n_pre * 128);
            wbytes += eb * tiles * n_pre * 128;
            o_rowv[c] = A.take(sizeof(float) * 4 * static_cast<size_t>(n_pre));  // s, M, qs, 1/qs
        } else {
            bool triplet = false;
            for (const auto& PL : s->plasts) triplet |= PL.conn == c && PL.kind == BSNN_PLASTICITY_TRIPLET;
            if (triplet) o_rsum[c] = A.take(sizeof(float) * static_cast<size_t>(n_pre));  // running row sums
        }
    }
    struct PlOff { size_t pre, post, tpre, tpost, colA[2], colB[2], sums; };
    std::vector<PlOff> o_pl(h.n_plast);
    for (uint32_t k = 0; k < h.n_plast; ++k) {
        const auto& C = s->conns[s->plasts[k].conn];
        const uint32_t n_pre = s->groups[C.pre].p.num_neurons, n_post = s->groups[C.post].p.num_neurons;
        const size_t np = sizeof(float) * n_pre, nq = sizeof(float) * round_up(n_post, 4);
        PlOff& o = o_pl[k];
        o.pre = A.take(np); o.tpre = A.take(np); o.post = A.take(nq); o.tpost = A.take(nq);
        for (int p = 0; p < 2; ++p) {
            o.colA[p] = A.take(nq); o.colB[p] = A.take(nq);
        }
        o.sums = A.take(np);
    }
    struct MonOff { size_t bits, vh, sel; };
    std::vector<MonOff> o_mon(h.n_mons);
    for (uint32_t m = 0; m < h.n_mons; ++m) {
        const auto& M = s->mons[m];
        const uint32_t ng = s->groups[M.group].p.num_neurons;
        if (M.kind == kMonSpikes) {
            o_mon[m].bits = A.take(sizeof(uint32_t) * static_cast<size_t>(M.interval) * ((ng + 31) / 32));
        } else {
            o_mon[m].vh = A.take(sizeof(float) * static_cast<size_t>(M.interval) * M.sel.size());
            o_mon[m].sel = A.take(sizeof(int32_t) * ng);
        }
    }

    // Work plan.
    uint32_t n_ctas = static_cast<uint32_t>(s->sm_count);
    if (const char* e = std::getenv("BSNN_CTAS")) n_ctas = std::max(1, std::atoi(e));
    n_ctas = std::min<uint32_t>(n_ctas, std::max<uint32_t>(1u, (N + 3) / 4));
    // Shared memory: the largest opt-in dynamic allocation minus the kernel's static shared data.
    int optin = 0;
    cuda_check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device), "smem attr");
    cudaFuncAttributes fa{}, fa_carry{}, fa_lazy{};
    cuda_check(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(&bsnn_step_kernel<false, false>)), "func attr");
    cuda_check(cudaFuncGetAttributes(&fa_carry, reinterpret_cast<const void*>(&bsnn_step_kernel<true, false>)), "func attr");
    cuda_check(cudaFuncGetAttributes(&fa_lazy, reinterpret_cast<const void*>(&bsnn_step_kernel<false, true>)), "func attr");
    fa.sharedSizeBytes = std::max({fa.sharedSizeBytes, fa_carry.sharedSizeBytes, fa_lazy.sharedSizeBytes});
    uint32_t n_spike_mons = 0;
    for (const auto& M : s->mons) n_spike_mons += M.kind == kMonSpikes ? 1u : 0u;
    // Per-group role counts that size the shared-memory neuron state.
    {
        std::vector<uint32_t> n_pre(h.n_groups, 0), n_post(h.n_groups, 0), n_vmon(h.n_groups, 0);
        for (const auto& PL : s->plasts) {
            ++n_pre[s->conns[PL.conn].pre];
            ++n_post[s->conns[PL.conn].post];
        }
        for (const auto& M : s->mons)
            if (M.kind != kMonSpikes) ++n_vmon[M.group];
        for (uint32_t g = 0; g < h.n_groups; ++g) {
            h.ns_ts = std::max(h.ns_ts, h.groups[g].n_ts);
            h.ns_pre = std::max(h.ns_pre, n_pre[g]);
            h.ns_post = std::max(h.ns_post, n_post[g]);
            h.ns_mon = std::max(h.ns_mon, n_vmon[g]);
        }
    }
    const uint32_t ns_fields = ns_layout(h.ns_ts, h.ns_pre, h.ns_post, h.ns_mon).fields;
    auto smem_of = [&](const Plan& pl, uint32_t resident_floats, uint32_t stage_rows) {
        return smem_sizes(resident_floats, pl.max_rows, pl.max_own, spk_words, n_spike_mons, h.n_groups, h.n_ts,
                          h.n_conns, h.n_plast, h.n_mons, static_cast<uint32_t>(pl.red_list.size()), ns_fields,
                          lazy ? 0u : pl.max_trows * pl.n_chunks, h.stage_warps, stage_rows, lazy ? pl.max_rows : 0u)
            .total;
    };
    const int64_t smem_limit = static_cast<int64_t>(optin) - static_cast<int64_t>(fa.sharedSizeBytes) - 128;
    // Plastic weight rows stay resident in shared memory for a whole launch when every CTA's
    // share fits; otherwise all rows stream from global memory (L2 / HBM).
    // (The row-scaled forms always stream: their weight pass only reads.)
    bool use_resident = !lazy;
    if (const char* e = std::getenv("BSNN_RESIDENT"); e && !lazy) use_resident = std::atoi(e) != 0;
    Plan P;
    bool resident_ok = false;
    if (use_resident) {
        int64_t cap = smem_limit - 8192;
        for (int attempt = 0; attempt < 8 && cap > 16384; ++attempt) {
            P = build_plan(s, n_ctas, static_cast<uint64_t>(cap), &resident_ok);
            if (!resident_ok) break;
            const int64_t need = static_cast<int64_t>(smem_of(P, static_cast<uint32_t>(P.resident_floats), 0u));
            if (need <= smem_limit) break;
            cap -= need - smem_limit + 256;
            resident_ok = false;
        }
    }
    if (!resident_ok) P = build_plan(s, n_ctas, 0, nullptr);
    h.resident_floats = resident_ok ? static_cast<uint32_t>(P.resident_floats) : 0u;
    h.n_ctas = n_ctas;
    h.n_slots = std::max(P.n_slots, 1u);
    h.max_rows = P.max_rows;
    h.max_trows = lazy ? 0u : P.max_trows;
    h.n_chunks = P.n_chunks;
    h.max_own = P.max_own;
    h.wfmt = s->weight_format;
    h.q_nonneg = 0;
    if (s->weight_format == BSNN_WEIGHTS_FP8_E4M3 && std::getenv("BSNN_FP8_CVT") == nullptr) {
        bool nonneg = true;
        for (const auto& C : s->conns)
            for (float v : C.w) nonneg &= !(v < 0.0f);
        for (const auto& PL : s->plasts) nonneg &= !(PL.p.weight_min < 0.0f);
        h.q_nonneg = nonneg ? 1u : 0u;
    }
    // Networks with streamed triplet rows carry row sums between steps (a kernel instance of its
    // own, with a lower thread limit: it needs more registers); the row-scaled forms have an
    // instance of their own.
    const bool carry = !lazy && P.max_trows > 0;
    std::memcpy(h.red_begin, P.red_begin, sizeof(P.red_begin));
    std::memcpy(h.red_end, P.red_end, sizeof(P.red_end));
    const uint32_t max_threads = static_cast<uint32_t>(carry ? kMaxThreads : lazy ? kMaxThreadsRows : kMaxThreadsPlain);
    require(P.max_own <= max_threads, BSNN_ERR_INVALID_ARGUMENT,
            "network too large for one persistent grid (more neurons per CTA than threads)");
    // Threads per CTA: the work items (32-aligned 4-column units of each segment) spread evenly
    // over at most max_threads threads.
    const uint32_t k_items = (P.max_items + max_threads - 1) / max_threads;
    uint32_t block = round_up((P.max_items + k_items - 1) / k_items, 32);
    block = std::max(block, round_up(P.max_own, 32));
    block = std::min<uint32_t>(std::max<uint32_t>(block, 64), max_threads);
    if (const char* e = std::getenv("BSNN_BLOCK")) block = std::min<uint32_t>(max_threads, round_up(std::max(32, std::atoi(e)), 32));
    block = std::max(block, round_up(P.max_own, 32));
    s->grid = n_ctas;
    s->block = block;
    s->kernel = lazy    ? reinterpret_cast<const void*>(&bsnn_step_kernel<false, true>)
                : carry ? reinterpret_cast<const void*>(&bsnn_step_kernel<true, false>)
                        : reinterpret_cast<const void*>(&bsnn_step_kernel<false, false>);
    // In those two instances streamed rows go through per-warp double buffers in shared memory,
    // filled by bulk asynchronous copies, when the room left after the plan holds them (the most
    // rows per buffer that fit, up to 16).
    h.stage_warps = block / 32;
    {
        uint32_t want = carry || lazy ? 16u : 0u;
        if (const char* e = std::getenv("BSNN_STAGE"); e && (carry || lazy))
            want = std::min<uint32_t>(16u, static_cast<uint32_t>(std::max(0, std::atoi(e))));
        h.stage_rows = 0;
        for (uint32_t r = want; r >= 4u; r /= 2u)
            if (static_cast<int64_t>(smem_of(P, h.resident_floats, r)) <= smem_limit) {
                h.stage_rows = r;
                break;
            }
    }
    require(!lazy || h.stage_rows > 0, BSNN_ERR_INVALID_ARGUMENT,
            "row-scaled weight form: no shared memory left for the staging buffers");

    size_t o_part = A.take(sizeof(float) * 2 * static_cast<size_t>(h.n_slots) * h.N_pad);
    size_t o_red = A.take(sizeof(uint32_t) * P.red_list.size());
    size_t o_ctas = A.take(sizeof(DCta) * P.ctas.size());
    size_t o_segs = A.take(sizeof(DSeg) * std::max<size_t>(P.segs.size(), 1));
    size_t o_blks = A.take(sizeof(DBlk) * std::max<size_t>(P.blks.size(), 1));
    size_t o_rows = A.take(sizeof(DRowMeta) * P.rows.size());
    size_t o_rowsb = A.take(sizeof(uint32_t) * P.rows_begin.size());

    // Stimulus: merge all stimuli into one per-step CSR, each step's events sorted by neuron.
    uint32_t stim_len = 0;
    for (const auto& st : s->stims) stim_len = std::max<uint32_t>(stim_len, static_cast<uint32_t>(st.counts.size()));
    std::vector<uint32_t> stim_off(stim_len + 1, 0), ev_neuron;
    std::vector<float> ev_delta;
    {
        std::vector<size_t> cursor(s->stims.size(), 0);
        std::vector<std::pair<uint32_t, float>> step_events;
        for (uint32_t t = 0; t < stim_len; ++t) {
            step_events.clear();
            for (size_t k = 0; k < s->stims.size(); ++k) {
                const auto& st = s->stims[k];
                if (t >= st.counts.size()) continue;
                for (uint32_t e = 0; e < st.counts[t]; ++e) {
                    const size_t idx = cursor[k] + e;
                    step_events.emplace_back(st.ids[idx] + st.offs[idx], st.deltas[idx]);
                }
                cursor[k] += st.counts[t];
            }
            std::stable_sort(step_events.begin(), step_events.end(),
                             [](const auto& a, const auto& b) { return a.first < b.first; });
            for (const auto& ev : step_events) {
                ev_neuron.push_back(ev.first);
                ev_delta.push_back(ev.second);
            }
            stim_off[t + 1] = static_cast<uint32_t>(ev_neuron.size());
        }
    }
    size_t o_soff = A.take(sizeof(uint32_t) * stim_off.size());
    size_t o_evn = A.take(sizeof(uint32_t) * std::max<size_t>(ev_neuron.size(), 1));
    size_t o_evd = A.take(sizeof(float) * std::max<size_t>(ev_delta.size(), 1));
    size_t o_rep = A.take(std::max<size_t>(s->replay.size(), 1));
    size_t o_bar = A.take(sizeof(unsigned long long));
    size_t o_err = A.take(sizeof(int32_t));
    size_t o_sd = A.take(sizeof(unsigned long long));
    size_t o_clk = A.take(sizeof(uint32_t));
    size_t o_pns = A.take(sizeof(unsigned long long) * kPhaseSlots * std::max<uint32_t>(s->sm_count, 1));
    size_t o_sim = A.take(sizeof(DSim));

    cuda_check(cudaMalloc(&s->arena, A.size), "cudaMalloc arena");
    s->arena_bytes = A.size;
    s->weight_bytes = wbytes;
    unsigned char* base = s->arena;
    cuda_check(cudaMemsetAsync(base, 0, A.size, s->stream), "cudaMemset arena");
    cuda_check(cudaStreamSynchronize(s->stream), "arena memset sync");
    auto F = [&](size_t o) { return reinterpret_cast<float*>(base + o); };
    auto U = [&](size_t o) { return reinterpret_cast<uint32_t*>(base + o); };

    h.v = F(o_v); h.ge = F(o_ge); h.gi = F(o_gi); h.istim = F(o_is);
    h.bg_ge = F(o_bge); h.bg_gi = F(o_bgi); h.bg_er = F(o_ber); h.bg_ed = F(o_bed); h.bg_ir = F(o_bir);
    h.bg_id = F(o_bid);
    h.refrac = U(o_ref);
    h.spikes[0] = U(o_spk0);
    h.spikes[1] = U(o_spk1);
    h.spk_bits[0] = U(o_sb0);
    h.spk_bits[1] = U(o_sb1);
    h.spk_words = spk_words;
    for (uint32_t t = 0; t < h.n_ts; ++t) {
        h.ts[t].r = F(o_ts[3 * t]);
        h.ts[t].d = F(o_ts[3 * t + 1]);
        h.ts[t].x = F(o_ts[3 * t + 2]);
    }
    std::vector<float> vinit(N, 0.0f);
    for (const auto& g : s->groups)
        for (uint32_t i = 0; i < g.p.num_neurons; ++i) vinit[g.p.offset + i] = g.p.v_rest;
    cuda_check(cudaMemcpyAsync(h.v, vinit.data(), fN, cudaMemcpyHostToDevice, s->stream), "H2D v");

    for (uint32_t c = 0; c < h.n_conns; ++c) {
        const auto& C = s->conns[c];
        DConn& D = h.conns[c];
        D.pre_g = C.pre;
        D.post_g = C.post;
        D.pre_off = s->groups[C.pre].p.offset;
        D.n_pre = s->groups[C.pre].p.num_neurons;
        D.post_off = s->groups[C.post].p.offset;
        D.n_post = s->groups[C.post].p.num_neurons;
        D.ld = s->conn_ld[c];
        D.units = D.ld / 4;
        D.target = s->groups[C.pre].p.is_inhibitory ? kTargetInh : kTargetExc;
        D.ts = conn_ts[c];
        D.plast = -1;
        D.w = F(o_w[c]);
        D.rowsum = o_rsum[c] ? F(o_rsum[c]) : nullptr;  // written by the first launch (from step 0)
        if (D.ld == D.n_post) {  // no padding columns: the rows are already laid out as on the device
            cuda_check(cudaMemcpy(D.w, C.w.data(), sizeof(float) * C.w.size(), cudaMemcpyHostToDevice), "H2D w");
        } else {
            std::vector<float> padded(static_cast<size_t>(D.n_pre) * D.ld, 0.0f);
            for (uint32_t i = 0; i < D.n_pre; ++i)
                std::memcpy(&padded[static_cast<size_t>(i) * D.ld], &C.w[static_cast<size_t>(i) * D.n_post],
                            sizeof(float) * D.n_post);
            cuda_check(cudaMemcpy(D.w, padded.data(), sizeof(float) * padded.size(), cudaMemcpyHostToDevice), "H2D w");
        }
        if (lazy) {
            const bool fp8 = s->weight_format == BSNN_WEIGHTS_FP8_E4M3;
            D.q = base + o_q[c];
            D.qtiles = (D.n_post + 127) / 128;
            float* rv = F(o_rowv[c]);
            D.lz_s = rv;
            D.lz_m = rv + D.n_pre;
            D.qscale = fp8 ? rv + 2 * static_cast<size_t>(D.n_pre) : nullptr;
            D.qinv = fp8 ? rv + 3 * static_cast<size_t>(D.n_pre) : nullptr;
            // s = 1, M = the row sum, and (FP8) qs = the larger of the row's largest magnitude and
            // the plastic bound weight_max (doubled for a normalised row, whose masters may reach
            // twice the bound before the normalisation folds s back into them), over 448 (the
            // largest finite E4M3 value).
            float wmax = 0.0f;
            bool normalised = false;
            for (const auto& PL : s->plasts)
                if (PL.conn == c) {
                    wmax = std::max(wmax, std::fabs(PL.p.weight_max));
                    normalised |= PL.kind == BSNN_PLASTICITY_TRIPLET;
                }
            std::vector<float> rows(4 * static_cast<size_t>(D.n_pre), 1.0f);
            for (uint32_t i = 0; i < D.n_pre; ++i) {
                double sum = 0.0;
                float big = 0.0f;
                for (uint32_t q = 0; q < D.n_post; ++q) {
                    const float v = C.w[static_cast<size_t>(i) * D.n_post + q];
                    sum += v;
                    big = std::max(big, std::fabs(v));
                }
                rows[D.n_pre + i] = static_cast<float>(sum);
                float qs = std::max(big, wmax) * (normalised ? 2.0f : 1.0f) / 448.0f;
                if (!(qs > 0.0f) || !std::isfinite(qs)) qs = 1.0f;
                rows[2 * static_cast<size_t>(D.n_pre) + i] = qs;
                rows[3 * static_cast<size_t>(D.n_pre) + i] = 1.0f / qs;
            }
            cuda_check(cudaMemcpy(rv, rows.data(), sizeof(float) * rows.size(), cudaMemcpyHostToDevice), "H2D rows");
            launch_fill_copy(D, s->weight_format, s->stream);
        }
    }
    for (uint32_t k = 0; k < h.n_plast; ++k) {
        const auto& PL = s->plasts[k];
        DPlast& D = h.plast[k];
        const PlOff& o = o_pl[k];
        D.kind = PL.kind;
        D.conn = PL.conn;
        D.ltp_A = PL.p.ltp_A; D.ltd_A = PL.p.ltd_A; D.ltp_B = PL.p.ltp_B; D.ltd_B = PL.p.ltd_B;
        D.pre_decay = PL.p.pre_trace_decay; D.post_decay = PL.p.post_trace_decay;
        D.tpre_decay = PL.p.triplet_pre_trace_decay; D.tpost_decay = PL.p.triplet_post_trace_decay;
        D.wmin = PL.p.weight_min; D.wmax = PL.p.weight_max;
        D.pre = F(o.pre); D.post = F(o.post); D.tpre = F(o.tpre); D.tpost = F(o.tpost);
        for (int p = 0; p < 2; ++p) {
            D.colA[p] = F(o.colA[p]); D.colB[p] = F(o.colB[p]);
        }
        D.sums = F(o.sums);
        DConn& C = h.conns[PL.conn];
        C.plast = static_cast<int32_t>(k);
        DGroup& Gp = h.groups[C.pre_g];
        DGroup& Gq = h.groups[C.post_g];
        require(Gp.n_plast_pre < static_cast<uint32_t>(kMaxGroupRoles) && Gq.n_plast_post < static_cast<uint32_t>(kMaxGroupRoles),
                BSNN_ERR_INVALID_ARGUMENT, "too many plasticities per group");
        Gp.plast_pre[Gp.n_plast_pre++] = static_cast<int32_t>(k);
        Gq.plast_post[Gq.n_plast_post++] = static_cast<int32_t>(k);
        if (PL.kind == BSNN_PLASTICITY_TRIPLET) {
            // TripletPlasticity::initialize_data (cpp_src/plasticities/triplet_plasticity.cpp:21-31):
            // initial column sums (float, ascending pre), applied as row targets.  Rows in the outer
            // loop: each column still adds its entries in ascending pre order, so the sums are the
            // same floats, without a strided walk down the columns of a row-major matrix.
            const auto& W = s->conns[PL.conn].w;
            std::vector<float> sums(C.n_pre, 0.0f);
            for (uint32_t i = 0; i < C.n_pre; ++i) {
                const float* row = &W[static_cast<size_t>(i) * C.n_post];
                for (uint32_t q = 0; q < C.n_pre; ++q) sums[q] += row[q];
            }
            cuda_check(cudaMemcpy(D.sums, sums.data(), sizeof(float) * sums.size(), cudaMemcpyHostToDevice), "H2D sums");
        }
    }
    for (uint32_t m = 0; m < h.n_mons; ++m) {
        const auto& M = s->mons[m];
        DMon& D = h.mons[m];
        const uint32_t ng = s->groups[M.group].p.num_neurons;
        D.kind = M.kind;
        D.group = M.group;
        D.interval = M.interval;
        D.words = (ng + 31) / 32;
        DGroup& G = h.groups[M.group];
        require(G.n_mon < static_cast<uint32_t>(kMaxGroupRoles), BSNN_ERR_INVALID_ARGUMENT, "too many monitors per group");
        G.mon[G.n_mon++] = static_cast<int32_t>(m);
        if (M.kind == kMonSpikes) {
            D.bits = U(o_mon[m].bits);
        } else {
            D.n_sel = static_cast<uint32_t>(M.sel.size());
            D.vh = F(o_mon[m].vh);
            D.sel_idx = reinterpret_cast<int32_t*>(base + o_mon[m].sel);
            std::vector<int32_t> sel(ng, -1);
            for (size_t k = 0; k < M.sel.size(); ++k)
                if (sel[M.sel[k]] < 0) sel[M.sel[k]] = static_cast<int32_t>(k);
            cuda_check(cudaMemcpy(D.sel_idx, sel.data(), sizeof(int32_t) * ng, cudaMemcpyHostToDevice), "H2D sel");
        }
    }

    h.partials = F(o_part);
    h.red_list = U(o_red);
    h.n_red = static_cast<uint32_t>(P.red_list.size());
    h.ctas = reinterpret_cast<const DCta*>(base + o_ctas);
    h.segs = reinterpret_cast<const DSeg*>(base + o_segs);
    h.blks = reinterpret_cast<const DBlk*>(base + o_blks);
    h.rows = reinterpret_cast<const DRowMeta*>(base + o_rows);
    h.rows_begin = U(o_rowsb);
    cuda_check(cudaMemcpy(base + o_red, P.red_list.data(), sizeof(uint32_t) * P.red_list.size(), cudaMemcpyHostToDevice), "H2D plan");
    cuda_check(cudaMemcpy(base + o_ctas, P.ctas.data(), sizeof(DCta) * P.ctas.size(), cudaMemcpyHostToDevice), "H2D plan");
    if (!P.segs.empty())
        cuda_check(cudaMemcpy(base + o_segs, P.segs.data(), sizeof(DSeg) * P.segs.size(), cudaMemcpyHostToDevice), "H2D plan");
    if (!P.blks.empty())
        cuda_check(cudaMemcpy(base + o_blks, P.blks.data(), sizeof(DBlk) * P.blks.size(), cudaMemcpyHostToDevice), "H2D plan");
    cuda_check(cudaMemcpy(base + o_rows, P.rows.data(), sizeof(DRowMeta) * P.rows.size(), cudaMemcpyHostToDevice), "H2D plan");
    cuda_check(cudaMemcpy(base + o_rowsb, P.rows_begin.data(), sizeof(uint32_t) * P.rows_begin.size(), cudaMemcpyHostToDevice), "H2D plan");

    h.stim_len = stim_len;
    h.stim_off = U(o_soff);
    h.ev_neuron = U(o_evn);
    h.ev_delta = F(o_evd);
    cuda_check(cudaMemcpy(base + o_soff, stim_off.data(), sizeof(uint32_t) * stim_off.size(), cudaMemcpyHostToDevice), "H2D stim");
    if (!ev_neuron.empty()) {
        cuda_check(cudaMemcpy(base + o_evn, ev_neuron.data(), sizeof(uint32_t) * ev_neuron.size(), cudaMemcpyHostToDevice), "H2D stim");
        cuda_check(cudaMemcpy(base + o_evd, ev_delta.data(), sizeof(float) * ev_delta.size(), cudaMemcpyHostToDevice), "H2D stim");
    }
    h.noise_mode = s->noise_mode;
    h.seed = static_cast<uint32_t>(s->desc.rng_seed);
    h.replay = base + o_rep;
    h.replay_steps = s->replay_steps;
    if (!s->replay.empty())
        cuda_check(cudaMemcpy(base + o_rep, s->replay.data(), s->replay.size(), cudaMemcpyHostToDevice), "H2D replay");
    h.barrier = reinterpret_cast<unsigned long long*>(base + o_bar);
    h.error = reinterpret_cast<int32_t*>(base + o_err);
    h.steps_done = reinterpret_cast<unsigned long long*>(base + o_sd);
    h.clock = U(o_clk);
    h.phase_ns = reinterpret_cast<unsigned long long*>(base + o_pns);
    h.wait_limit_ns = s->wait_limit_ns;
    h.skip_step = s->skip_step;
    h.skip_cta = s->skip_cta;
    s->d_sim = reinterpret_cast<DSim*>(base + o_sim);
    cuda_check(cudaMemcpy(s->d_sim, &h, sizeof(DSim), cudaMemcpyHostToDevice), "H2D sim");

    // Launch configuration.
    s->smem_bytes = smem_of(P, h.resident_floats, h.stage_rows);
    cuda_check(cudaFuncSetAttribute(s->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(s->smem_bytes)),
               "cudaFuncSetAttribute smem");
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, s->kernel, static_cast<int>(s->block),
                                                             s->smem_bytes),
               "occupancy");
    require(per_sm >= 1 && static_cast<long>(per_sm) * s->sm_count >= static_cast<long>(s->grid), BSNN_ERR_RUNTIME,
            "persistent grid does not fit on the device");
    cuda_check(cudaStreamSynchronize(s->stream), "finalize sync");
    s->finalized = true;
}

void launch_direct(bsnn_sim* s, uint32_t n_steps) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(s->grid);
    cfg.blockDim = dim3(s->block);
    cfg.dynamicSmemBytes = s->smem_bytes;
    cfg.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const DSim* arg0 = s->d_sim;
    void* args[2] = {&arg0, &n_steps};
    cuda_check(cudaLaunchKernelExC(&cfg, s->kernel, args), "bsnn_step_kernel launch");
    ++s->launches;
}

void launch_chunk(bsnn_sim* s, uint32_t n_steps) {
    if (s->graphs_ok) {
        auto it = s->graphs.find(n_steps);
        if (it == s->graphs.end()) {
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            bool ok = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3(s->grid);
                cfg.blockDim = dim3(s->block);
                cfg.dynamicSmemBytes = s->smem_bytes;
                cfg.stream = s->stream;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeCooperative;
                attr[0].val.cooperative = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                const DSim* arg0 = s->d_sim;
                void* args[2] = {&arg0, &n_steps};
                const cudaError_t le = cudaLaunchKernelExC(&cfg, s->kernel, args);
                const cudaError_t ce = cudaStreamEndCapture(s->stream, &graph);
                ok = le == cudaSuccess && ce == cudaSuccess && graph != nullptr &&
                     cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
                if (graph) cudaGraphDestroy(graph);
            }
            if (!ok) {
                cudaGetLastError();  // clear the capture failure; fall back to direct launches
                s->graphs_ok = false;
                launch_direct(s, n_steps);
                return;
            }
            it = s->graphs.emplace(n_steps, exec).first;
        }
        cuda_check(cudaGraphLaunch(it->second, s->stream), "cudaGraphLaunch");
        ++s->launches;
        return;
    }
    launch_direct(s, n_steps);
}

void check_device_error(bsnn_sim* s) {
    cuda_check(cudaStreamSynchronize(s->stream), "stream synchronize");
    int32_t e = 0;
    cuda_check(cudaMemcpy(&e, s->h.error, sizeof(e), cudaMemcpyDeviceToHost), "D2H error flag");
    if (e != kErrNone) {
        s->failed = true;
        throw ApiError(BSNN_ERR_DEVICE_TIMEOUT, "device-side grid barrier timed out; simulation state is invalid");
    }
}

void run_steps(bsnn_sim* s, uint32_t first_clock, uint32_t n) {
    finalize(s);
    require(!s->failed, BSNN_ERR_STATE, "simulation failed earlier (device timeout)");
    if (n == 0) return;
    if (first_clock != s->next_clock) {
        bsnn_set_clock_kernel<<<1, 1, 0, s->stream>>>(s->h.clock, first_clock);
        cuda_check(cudaGetLastError(), "set clock");
    }
    uint32_t left = n;
    while (left > 0) {
        const uint32_t chunk = std::min(left, s->steps_per_launch);
        launch_chunk(s, chunk);
        left -= chunk;
    }
    s->steps_done += n;
    s->next_clock = first_clock + n;
}

// Field -> (device pointer, element count, element size).
struct FieldRef {
    void* ptr;
    uint32_t len;
};

FieldRef field_ref(bsnn_sim* s, int32_t field, uint32_t index) {
    const DSim& h = s->h;
    const uint32_t N = s->N;
    switch (field) {
        case BSNN_FIELD_MEMBRANE_POTENTIALS: return {h.v, N};
        case BSNN_FIELD_G_EXCITATORY: return {h.ge, N};
        case BSNN_FIELD_G_INHIBITORY: return {h.gi, N};
        case BSNN_FIELD_I_STIMULUS: return {h.istim, N};
        case BSNN_FIELD_REFRACTORY_COUNTER: return {h.refrac, N};
        case BSNN_FIELD_SPIKES: return {h.spikes[s->steps_done == 0 ? 0 : (s->steps_done - 1) & 1], N};
        case BSNN_FIELD_BG_G_EXCITATORY: return {h.bg_ge, N};
        case BSNN_FIELD_BG_G_INHIBITORY: return {h.bg_gi, N};
        case BSNN_FIELD_BG_E_R_TRACES: return {h.bg_er, N};
        case BSNN_FIELD_BG_E_D_TRACES: return {h.bg_ed, N};
        case BSNN_FIELD_BG_I_R_TRACES: return {h.bg_ir, N};
        case BSNN_FIELD_BG_I_D_TRACES: return {h.bg_id, N};
        default: break;
    }
    if (field >= BSNN_FIELD_CONN_R_TRACES && field <= BSNN_FIELD_CONN_SUMMED) {
        require(index < h.n_conns, BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        const DTraceSet& T = h.ts[h.conns[index].ts];
        const uint32_t n = h.conns[index].n_pre;
        return {field == BSNN_FIELD_CONN_R_TRACES ? T.r : field == BSNN_FIELD_CONN_D_TRACES ? T.d : T.x, n};
    }
    if (field >= BSNN_FIELD_CONN_ROW_SCALE && field <= BSNN_FIELD_CONN_ROW_QUANT_SCALE) {
        require(index < h.n_conns, BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        require(h.wfmt != kFmtF32, BSNN_ERR_INVALID_ARGUMENT, "no row scales in the BSNN_WEIGHTS_F32 form");
        const DConn& C = h.conns[index];
        if (field == BSNN_FIELD_CONN_ROW_SCALE) return {C.lz_s, C.n_pre};
        if (field == BSNN_FIELD_CONN_ROW_MASTER_SUM) return {C.lz_m, C.n_pre};
        require(C.qscale != nullptr, BSNN_ERR_INVALID_ARGUMENT, "no quantisation scales outside the FP8 form");
        return {C.qscale, C.n_pre};
    }
    if (field >= BSNN_FIELD_PLAST_PRE_TRACES && field <= BSNN_FIELD_PLAST_PRE_WEIGHT_SUMS) {
        require(index < h.n_plast, BSNN_ERR_OUT_OF_RANGE, "plasticity index out of range");
        const DPlast& P = h.plast[index];
        const DConn& C = h.conns[P.conn];
        switch (field) {
            case BSNN_FIELD_PLAST_PRE_TRACES: return {P.pre, C.n_pre};
            case BSNN_FIELD_PLAST_POST_TRACES: return {P.post, C.n_post};
            case BSNN_FIELD_PLAST_TRIPLET_PRE: return {P.tpre, C.n_pre};
            case BSNN_FIELD_PLAST_TRIPLET_POST: return {P.tpost, C.n_post};
            default: return {P.sums, P.kind == kKindTriplet ? C.n_pre : 0u};
        }
    }
    throw ApiError(BSNN_ERR_INVALID_ARGUMENT, "unknown field " + std::to_string(field));
}

}  // namespace

// ============================================================================================
namespace {

// Monitor::record(clock_step) for every recorder with an output (cpp_src/monitors/*.cpp): the
// rings are copied to host memory and flushed here; the text is written by the writer thread.
// A connection's weights as [n_pre][ld] floats: the stored matrix, or in a row-scaled form the
// masters times their rows' normalisation scales.
void download_weights(bsnn_sim* s, const DConn& C, float* out) {
    const size_t n = static_cast<size_t>(C.n_pre) * C.ld;
    cuda_check(cudaMemcpy(out, C.w, sizeof(float) * n, cudaMemcpyDeviceToHost), "D2H weights");
    if (s->h.wfmt == kFmtF32) return;
    std::vector<float> sc(C.n_pre);
    cuda_check(cudaMemcpy(sc.data(), C.lz_s, sizeof(float) * C.n_pre, cudaMemcpyDeviceToHost), "D2H row scales");
    for (uint32_t i = 0; i < C.n_pre; ++i)
        for (uint32_t q = 0; q < C.ld; ++q) out[static_cast<size_t>(i) * C.ld + q] *= sc[i];
}

void record_all(bsnn_sim* s, uint32_t clock_step) {
    finalize(s);
    check_device_error(s);
    if (!s->writer) s->writer = std::make_unique<rec::Writer>();
    for (uint32_t m = 0; m < s->mons.size(); ++m) {
        HostMon& hm = s->mons[m];
        if (hm.path.empty()) continue;
        const DMon& M = s->h.mons[m];
        const uint32_t ng = s->groups[M.group].p.num_neurons, interval = M.interval;
        if (M.kind == kMonSpikes) {
            if (clock_step < interval) continue;  // spike_recorder.cpp:41-43
            const size_t n = static_cast<size_t>(interval) * M.words;
            auto bits = std::make_shared<std::vector<uint32_t>>(n);
            cuda_check(cudaMemcpy(bits->data(), M.bits, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost), "D2H spike ring");
            cuda_check(cudaMemsetAsync(M.bits, 0, sizeof(uint32_t) * n, s->stream), "flush spike ring");
            auto out = hm.spike_out;
            const uint32_t words = M.words;
            s->writer->push([bits, out, words, ng, interval, clock_step] {
                std::string text;
                rec::spike_rows(text, bits->data(), words, ng, interval, clock_step);
                if (out && out->good()) out->write(text.data(), static_cast<std::streamsize>(text.size()));
            });
        } else {
            const size_t n = static_cast<size_t>(interval) * M.n_sel;
            auto vh = std::make_shared<std::vector<float>>(n);
            cuda_check(cudaMemcpy(vh->data(), M.vh, sizeof(float) * n, cudaMemcpyDeviceToHost), "D2H voltage ring");
            cuda_check(cudaMemsetAsync(M.vh, 0, sizeof(float) * n, s->stream), "flush voltage ring");
            // ring column of each selected neuron: its first occurrence in the selection
            std::vector<int32_t> first(ng, -1);
            auto col = std::make_shared<std::vector<uint32_t>>(hm.sel.size());
            for (size_t k = 0; k < hm.sel.size(); ++k) {
                if (first[hm.sel[k]] < 0) first[hm.sel[k]] = static_cast<int32_t>(k);
                (*col)[k] = static_cast<uint32_t>(first[hm.sel[k]]);
            }
            auto sel = std::make_shared<std::vector<uint32_t>>(hm.sel);
            const std::string path = hm.path;
            const uint32_t n_cols = M.n_sel;
            s->writer->push([vh, col, sel, path, n_cols, interval, clock_step] {
                for (uint32_t slot = 0; slot < interval; ++slot) {  // voltage_recorder.cpp:60-76
                    std::string text;
                    rec::voltage_file(text, *sel, *col, vh->data(), n_cols, slot);
                    rec::write_file(rec::step_path(path, clock_step - interval + slot + 1u), text);
                }
            });
        }
    }
    for (const auto& wr : s->wrecs) {
        if (clock_step % 100000u != 0u) continue;  // weight_recorder.cpp:26-28
        const DConn& C = s->h.conns[wr.conn];
        const size_t n = static_cast<size_t>(C.n_pre) * C.ld;
        auto w = std::make_shared<std::vector<float>>(n);
        download_weights(s, C, w->data());
        const std::string path = wr.path;
        const uint32_t n_pre = C.n_pre, n_post = C.n_post, ld = C.ld;
        s->writer->push([w, path, n_pre, n_post, ld, clock_step] {
            std::string text;
            rec::weight_file(text, w->data(), n_pre, n_post, ld);
            rec::write_file(rec::step_path(path, clock_step), text);
        });
    }
}

}  // namespace

extern "C" {

BSNN_API const char* bsnn_version(void) { return "bsnn 0.1 (sm_100a persistent step kernel)"; }

BSNN_API bsnn_status bsnn_create(const bsnn_state_desc* desc, bsnn_sim** out_sim) {
    return guarded(nullptr, [&] {
        require(desc && out_sim, BSNN_ERR_INVALID_ARGUMENT, "null argument");
        require(desc->num_excitatory_neurons + static_cast<uint64_t>(desc->num_inhibitory_neurons) < (1ull << 31),
                BSNN_ERR_INVALID_ARGUMENT, "too many neurons");
        auto s = std::make_unique<bsnn_sim>();
        s->desc = *desc;
        if (s->desc.recording_interval_steps == 0) s->desc.recording_interval_steps = 10000;
        s->N = desc->num_excitatory_neurons + desc->num_inhibitory_neurons;
        s->device = desc->device;
        int n_dev = 0;
        cuda_check(cudaGetDeviceCount(&n_dev), "cudaGetDeviceCount");
        require(desc->device >= 0 && desc->device < n_dev, BSNN_ERR_INVALID_ARGUMENT, "invalid CUDA device ordinal");
        DeviceGuard g(s->device);
        cudaDeviceProp prop{};
        cuda_check(cudaGetDeviceProperties(&prop, s->device), "cudaGetDeviceProperties");
        require(prop.cooperativeLaunch != 0, BSNN_ERR_RUNTIME, "device does not support cooperative launches");
        s->sm_count = prop.multiProcessorCount;
        cuda_check(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        *out_sim = s.release();
    });
}

BSNN_API bsnn_status bsnn_destroy(bsnn_sim* sim) {
    if (!sim) return BSNN_OK;
    {
        DeviceGuard g(sim->device);
        if (sim->stream) cudaStreamSynchronize(sim->stream);
        delete sim;
    }
    return BSNN_OK;
}

BSNN_API const char* bsnn_last_error(const bsnn_sim* sim) {
    return sim ? sim->err.c_str() : g_thread_error.c_str();
}

BSNN_API bsnn_status bsnn_get_info(const bsnn_sim* sim, bsnn_info* out) {
    if (!sim || !out) return BSNN_ERR_INVALID_ARGUMENT;
    bsnn_info i{};
    i.total_neurons = sim->N;
    i.num_groups = static_cast<uint32_t>(sim->groups.size());
    i.num_connections = static_cast<uint32_t>(sim->conns.size());
    i.num_plasticities = static_cast<uint32_t>(sim->plasts.size());
    i.num_monitors = static_cast<uint32_t>(sim->mons.size());
    i.grid_ctas = sim->grid;
    i.block_threads = sim->block;
    i.steps_per_launch = sim->steps_per_launch;
    i.steps_done = sim->steps_done;
    i.device_bytes = sim->arena_bytes;
    i.weight_bytes = sim->weight_bytes;
    i.kernel_launches = sim->launches;
    i.smem_bytes = sim->smem_bytes;
    i.resident_bytes = 4ull * sim->h.resident_floats;
    *out = i;
    return BSNN_OK;
}

BSNN_API bsnn_status bsnn_add_neuron_group(bsnn_sim* sim, const bsnn_neuron_group_params* p, uint32_t* out_group) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        require(p != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null params");
        // GpuSimulationState::require_upload_bounds (gpu_simulation_state.cu:211-219)
        require(p->offset <= sim->N && p->num_neurons <= sim->N - p->offset, BSNN_ERR_INVALID_ARGUMENT,
                "neuron_group slice is out of bounds. offset=" + std::to_string(p->offset) +
                    ", count=" + std::to_string(p->num_neurons) + ", total_neurons=" + std::to_string(sim->N));
        require(sim->groups.size() < static_cast<size_t>(kMaxGroups), BSNN_ERR_INVALID_ARGUMENT, "too many neuron groups");
        for (const auto& g : sim->groups) {
            const bool disjoint = p->offset + p->num_neurons <= g.p.offset || g.p.offset + g.p.num_neurons <= p->offset;
            require(disjoint, BSNN_ERR_INVALID_ARGUMENT, "neuron groups must not overlap");
        }
        require(p->num_neurons > 0, BSNN_ERR_INVALID_ARGUMENT, "neuron group must not be empty");
        require(p->membrane_capacitance > 0.0f, BSNN_ERR_INVALID_ARGUMENT, "membrane_capacitance must be > 0");
        require(p->mean_background_excitatory_spikes <= 80.0f && p->mean_background_inhibitory_spikes <= 80.0f,
                BSNN_ERR_INVALID_ARGUMENT, "mean background spikes per step must be <= 80");
        sim->groups.push_back(HostGroup{*p});
        if (out_group) *out_group = static_cast<uint32_t>(sim->groups.size() - 1);
    });
}

BSNN_API bsnn_status bsnn_add_connection(bsnn_sim* sim, uint32_t pre_group, uint32_t post_group, const float* weights,
                                         const bsnn_connection_params* p, uint32_t* out_connection) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        require(weights && p, BSNN_ERR_INVALID_ARGUMENT, "null weights or params");
        require(pre_group < sim->groups.size() && post_group < sim->groups.size(), BSNN_ERR_OUT_OF_RANGE,
                "group index out of range");
        // GpuSimulationState::lookup_weight_matrix_name (gpu_simulation_state.cu:231-236)
        require(p->weight_matrix_idx < 4, BSNN_ERR_OUT_OF_RANGE,
                "Invalid weight matrix index: " + std::to_string(p->weight_matrix_idx));
        require(sim->conns.size() < static_cast<size_t>(kMaxConns), BSNN_ERR_INVALID_ARGUMENT, "too many connections");
        for (const auto& c : sim->conns) {
            require(c.p.weight_matrix_idx != p->weight_matrix_idx, BSNN_ERR_INVALID_ARGUMENT,
                    "weight_matrix_idx already used by another connection");
            require(!(c.pre == pre_group && c.post == post_group), BSNN_ERR_INVALID_ARGUMENT,
                    "a connection between these groups already exists");
        }
        require(p->rise_time > 0.0f && p->decay_time > 0.0f, BSNN_ERR_INVALID_ARGUMENT, "rise_time and decay_time must be > 0");
        const uint32_t n_pre = sim->groups[pre_group].p.num_neurons, n_post = sim->groups[post_group].p.num_neurons;
        HostConn c;
        c.pre = pre_group;
        c.post = post_group;
        c.p = *p;
        const size_t n = static_cast<size_t>(n_pre) * n_post;
        c.w.assign(weights, weights + n);
        // GpuSimulationState::require_nonnegative_weights (gpu_simulation_state.cu:221-229)
        require(std::none_of(c.w.begin(), c.w.end(), [](float x) { return x < 0.0f; }), BSNN_ERR_INVALID_ARGUMENT,
                "connection weight_matrix must be non-negative to preserve inhibitory routing contract");
        // Connection::make_gpu_view (connection.cpp:46-47): decays in float on the host.
        c.r_decay = std::exp(-1.0f * p->timestep / p->rise_time);
        c.d_decay = std::exp(-1.0f * p->timestep / p->decay_time);
        c.norm = p->postsynaptic_kernel_normalization_value;
        sim->conns.push_back(std::move(c));
        if (out_connection) *out_connection = static_cast<uint32_t>(sim->conns.size() - 1);
    });
}

BSNN_API bsnn_status bsnn_add_stimulus(bsnn_sim* sim, const uint32_t* counts, uint32_t num_timesteps,
                                       const uint32_t* ids, const uint32_t* offsets, const float* deltas,
                                       uint32_t num_events) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        // GpuSimulationState::upload_stimulus_view (gpu_simulation_state.cu:172-186)
        require(num_timesteps == sim->desc.total_simulation_length && num_events == sim->desc.num_stimulus_events,
                BSNN_ERR_INVALID_ARGUMENT,
                "upload_stimulus_view host data vectors must match gpu_view.num_stimulus_events and total_simulation_length");
        require((counts || num_timesteps == 0) && ((ids && offsets && deltas) || num_events == 0),
                BSNN_ERR_INVALID_ARGUMENT, "null stimulus arrays");
        HostStim st;
        st.counts.assign(counts, counts + num_timesteps);
        st.ids.assign(ids, ids + num_events);
        st.offs.assign(offsets, offsets + num_events);
        st.deltas.assign(deltas, deltas + num_events);
        uint64_t total = 0;
        for (uint32_t c : st.counts) total += c;
        // Stimulus::apply (stimulus.cpp:50-53) would throw when reaching the overflowing step.
        require(total <= num_events, BSNN_ERR_RUNTIME, "Stimulus event indexing exceeded uploaded event buffers");
        for (uint32_t e = 0; e < num_events; ++e)
            require(static_cast<uint64_t>(st.ids[e]) + st.offs[e] < sim->N, BSNN_ERR_OUT_OF_RANGE,
                    "stimulus event neuron out of range");
        sim->stims.push_back(std::move(st));
    });
}

BSNN_API bsnn_status bsnn_add_plasticity(bsnn_sim* sim, int32_t kind, uint32_t connection,
                                         const bsnn_plasticity_params* p, uint32_t* out_plasticity) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        require(p != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null params");
        require(connection < sim->conns.size(), BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        require(kind == BSNN_PLASTICITY_TRIPLET || kind == BSNN_PLASTICITY_ISTDP || kind == BSNN_PLASTICITY_STDP,
                BSNN_ERR_INVALID_ARGUMENT, "unknown plasticity kind");
        require(sim->plasts.size() < static_cast<size_t>(kMaxPlast), BSNN_ERR_INVALID_ARGUMENT, "too many plasticities");
        require(p->plasticity_offset < std::max(sim->desc.num_plasticities, 1u), BSNN_ERR_OUT_OF_RANGE,
                "plasticity_offset exceeds num_plasticities");
        for (const auto& pl : sim->plasts)
            require(pl.conn != connection, BSNN_ERR_INVALID_ARGUMENT, "connection already has a plasticity");
        const auto& C = sim->conns[connection];
        if (kind == BSNN_PLASTICITY_TRIPLET)
            require(sim->groups[C.pre].p.num_neurons <= sim->groups[C.post].p.num_neurons, BSNN_ERR_INVALID_ARGUMENT,
                    "triplet normalisation needs num_pre <= num_post");
        // validate_plasticity_params (cpp_src/main_buryn.cpp:76-96)
        require(p->pre_trace_decay >= 0.0f && p->pre_trace_decay <= 1.0f, BSNN_ERR_RUNTIME, "pre_trace_decay must be in [0, 1]");
        require(p->post_trace_decay >= 0.0f && p->post_trace_decay <= 1.0f, BSNN_ERR_RUNTIME, "post_trace_decay must be in [0, 1]");
        if (kind == BSNN_PLASTICITY_TRIPLET) {
            require(p->triplet_pre_trace_decay >= 0.0f && p->triplet_pre_trace_decay <= 1.0f, BSNN_ERR_RUNTIME,
                    "triplet_pre_trace_decay must be in [0, 1]");
            require(p->triplet_post_trace_decay >= 0.0f && p->triplet_post_trace_decay <= 1.0f, BSNN_ERR_RUNTIME,
                    "triplet_post_trace_decay must be in [0, 1]");
        }
        require(p->weight_min <= p->weight_max, BSNN_ERR_RUNTIME, "weight_min must be <= weight_max");
        sim->plasts.push_back(HostPlast{kind, connection, *p});
        if (out_plasticity) *out_plasticity = static_cast<uint32_t>(sim->plasts.size() - 1);
    });
}

BSNN_API bsnn_status bsnn_add_spike_recorder(bsnn_sim* sim, uint32_t group, uint32_t interval, uint32_t* out_monitor) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        require(group < sim->groups.size(), BSNN_ERR_OUT_OF_RANGE, "group index out of range");
        require(sim->mons.size() < static_cast<size_t>(kMaxMonitors), BSNN_ERR_INVALID_ARGUMENT, "too many monitors");
        HostMon m;
        m.kind = kMonSpikes;
        m.group = group;
        m.interval = interval ? interval : sim->desc.recording_interval_steps;
        sim->mons.push_back(std::move(m));
        if (out_monitor) *out_monitor = static_cast<uint32_t>(sim->mons.size() - 1);
    });
}

BSNN_API bsnn_status bsnn_add_voltage_recorder(bsnn_sim* sim, uint32_t group, const uint32_t* ids, uint32_t n_ids,
                                               uint32_t interval, uint32_t* out_monitor) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        require(group < sim->groups.size(), BSNN_ERR_OUT_OF_RANGE, "group index out of range");
        require(sim->mons.size() < static_cast<size_t>(kMaxMonitors), BSNN_ERR_INVALID_ARGUMENT, "too many monitors");
        const uint32_t ng = sim->groups[group].p.num_neurons;
        HostMon m;
        m.kind = kMonVoltage;
        m.group = group;
        m.interval = interval ? interval : sim->desc.recording_interval_steps;
        // VoltageRecorder ctor (voltage_recorder.cpp:15-26)
        if (n_ids == 0) {
            m.sel.resize(ng);
            std::iota(m.sel.begin(), m.sel.end(), 0u);
        } else {
            require(ids != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null selected ids");
            for (uint32_t k = 0; k < n_ids; ++k)
                require(ids[k] < ng, BSNN_ERR_OUT_OF_RANGE,
                        "Selected neuron ID " + std::to_string(ids[k]) + " is out of range for the neuron group.");
            m.sel.assign(ids, ids + n_ids);
        }
        sim->mons.push_back(std::move(m));
        if (out_monitor) *out_monitor = static_cast<uint32_t>(sim->mons.size() - 1);
    });
}

BSNN_API bsnn_status bsnn_set_noise_mode(bsnn_sim* sim, int32_t mode) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        require(mode == BSNN_NOISE_PHILOX || mode == BSNN_NOISE_OFF || mode == BSNN_NOISE_REPLAY,
                BSNN_ERR_INVALID_ARGUMENT, "unknown noise mode");
        sim->noise_mode = mode;
    });
}

BSNN_API bsnn_status bsnn_set_weight_format(bsnn_sim* sim, int32_t format) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        require(format >= BSNN_WEIGHTS_F32 && format <= BSNN_WEIGHTS_FP8_E4M3, BSNN_ERR_INVALID_ARGUMENT,
                "unknown weight format");
        sim->weight_format = format;
    });
}

BSNN_API bsnn_status bsnn_set_noise_replay(bsnn_sim* sim, const uint8_t* counts, uint32_t n_steps) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require_building(sim);
        require(counts != nullptr || n_steps == 0, BSNN_ERR_INVALID_ARGUMENT, "null counts");
        sim->replay.assign(counts, counts + static_cast<size_t>(n_steps) * sim->N * 2);
        sim->replay_steps = n_steps;
        sim->noise_mode = BSNN_NOISE_REPLAY;
    });
}

BSNN_API bsnn_status bsnn_step(bsnn_sim* sim, uint32_t clock_step) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] { run_steps(sim, clock_step, 1); });
}

BSNN_API bsnn_status bsnn_run(bsnn_sim* sim, uint32_t first_clock_step, uint32_t num_steps) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] { run_steps(sim, first_clock_step, num_steps); });
}

BSNN_API bsnn_status bsnn_synchronize(bsnn_sim* sim) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        if (!sim->finalized) return;
        check_device_error(sim);
    });
}

BSNN_API bsnn_status bsnn_get_stream(const bsnn_sim* sim, void** out_stream) {
    if (!sim || !out_stream) return BSNN_ERR_INVALID_ARGUMENT;
    *out_stream = sim->stream;
    return BSNN_OK;
}

BSNN_API bsnn_status bsnn_set_steps_per_launch(bsnn_sim* sim, uint32_t steps) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require(steps >= 1 && steps <= 65536, BSNN_ERR_INVALID_ARGUMENT, "steps per launch must be in [1, 65536]");
        sim->steps_per_launch = steps;
    });
}

// Re-uploads the launch descriptor after a host-side change of one of its scalar fields (the next
// launch reads it; queued launches finish first).
static void upload_descriptor(bsnn_sim* sim) {
    if (!sim->finalized) return;
    sim->h.wait_limit_ns = sim->wait_limit_ns;
    sim->h.skip_step = sim->skip_step;
    sim->h.skip_cta = sim->skip_cta;
    cuda_check(cudaStreamSynchronize(sim->stream), "stream synchronize");
    cuda_check(cudaMemcpy(sim->d_sim, &sim->h, sizeof(DSim), cudaMemcpyHostToDevice), "H2D descriptor");
}

BSNN_API bsnn_status bsnn_set_device_wait_limit(bsnn_sim* sim, uint64_t nanoseconds) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require(nanoseconds >= 1000ull && nanoseconds <= 60000000000ull, BSNN_ERR_INVALID_ARGUMENT,
                "device wait limit must be in [1 us, 60 s]");
        sim->wait_limit_ns = nanoseconds;
        upload_descriptor(sim);
    });
}

BSNN_API bsnn_status bsnn_measure_exchange_floor(bsnn_sim* sim, uint32_t num_steps, float* out_us_per_step) {
    if (!sim || !out_us_per_step) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require(num_steps >= 1 && num_steps <= 1000000, BSNN_ERR_INVALID_ARGUMENT, "num_steps must be in [1, 1e6]");
        finalize(sim);
        require(!sim->failed, BSNN_ERR_STATE, "simulation failed earlier (device timeout)");
        const size_t smem = align16(sizeof(float) * 2u * sim->h.max_own) + align16(sizeof(DGroup) * sim->h.n_groups) +
                            sizeof(uint32_t) * sim->h.n_red;
        const void* fn = reinterpret_cast<const void*>(&bsnn_exchange_floor_kernel);
        cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                   "cudaFuncSetAttribute smem (exchange floor)");
        int per_sm = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, static_cast<int>(sim->block), smem),
                   "occupancy (exchange floor)");
        require(static_cast<uint64_t>(per_sm) * sim->sm_count >= sim->grid, BSNN_ERR_RUNTIME,
                "exchange-floor kernel cannot be co-resident with the step kernel's grid");
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(sim->grid);
        cfg.blockDim = dim3(sim->block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = sim->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const DSim* arg0 = sim->d_sim;
        uint32_t n = num_steps;
        void* args[2] = {&arg0, &n};
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        // a warm-up launch, then the timed one
        cudaError_t le = cudaLaunchKernelExC(&cfg, fn, args);
        if (le == cudaSuccess) le = cudaEventRecord(e0, sim->stream);
        if (le == cudaSuccess) le = cudaLaunchKernelExC(&cfg, fn, args);
        if (le == cudaSuccess) le = cudaEventRecord(e1, sim->stream);
        float ms = 0.0f;
        if (le == cudaSuccess) le = cudaEventSynchronize(e1);
        if (le == cudaSuccess) le = cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cuda_check(le, "exchange floor launch");
        check_device_error(sim);
        *out_us_per_step = 1000.0f * ms / static_cast<float>(num_steps);
    });
}

BSNN_API bsnn_status bsnn_debug_skip_arrival(bsnn_sim* sim, uint32_t cta, uint64_t step) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        require(cta < sim->grid, BSNN_ERR_OUT_OF_RANGE,
                "cta " + std::to_string(cta) + " is not in the grid of " + std::to_string(sim->grid));
        sim->skip_cta = cta;
        sim->skip_step = step;
        upload_descriptor(sim);
    });
}

// ---- checkpoint / resume ---------------------------------------------------------------------
// A checkpoint is the simulation's whole device arena (neuron state, traces, weights and their
// copies, plasticity traces, monitor rings, the step counters, the planned work lists) plus the
// host's clock cursor.  The arena's layout is a function of the components and their order, the
// weight form and the device's SM count, so a checkpoint loads into a simulation built the same
// way on the same kind of GPU: the header carries a fingerprint of that layout.  The one region
// holding device addresses, the kernel's descriptor, is rewritten from the loading simulation's
// own copy.  Text recording (files written by monitors) is not part of it.
namespace {

constexpr char kCkptMagic[8] = {'B', 'S', 'N', 'N', 'C', 'K', 'P', 'T'};
constexpr uint32_t kCkptVersion = 1;

struct CkptHeader {
    char magic[8];
    uint32_t version;
    uint32_t N;
    uint64_t arena_bytes;
    uint64_t fingerprint;
    uint64_t steps_done;
    uint32_t next_clock;
    int32_t weight_format;
};

uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

// The layout: sizes and counts of every component and of the launch plan.
uint64_t layout_fingerprint(const bsnn_sim* s) {
    uint64_t h = 1469598103934665603ull;
    const DSim& d = s->h;
    const uint32_t head[] = {d.N, d.N_pad, d.n_groups, d.n_conns, d.n_ts, d.n_plast, d.n_mons, d.n_ctas, d.n_slots,
                             d.max_rows, d.max_own, d.resident_floats, d.max_trows, d.n_chunks, d.stage_rows,
                             d.stage_warps, static_cast<uint32_t>(d.wfmt), d.spk_words, d.n_red, d.stim_len,
                             d.replay_steps, s->grid, s->block};
    h = fnv1a(h, head, sizeof(head));
    for (const auto& g : s->groups) h = fnv1a(h, &g.p.num_neurons, sizeof(g.p.num_neurons));
    for (const auto& c : s->conns) {
        const uint32_t cc[] = {c.pre, c.post};
        h = fnv1a(h, cc, sizeof(cc));
    }
    for (const auto& p : s->plasts) h = fnv1a(h, &p.kind, sizeof(p.kind));
    for (const auto& m : s->mons) {
        const uint32_t mm[] = {static_cast<uint32_t>(m.kind), m.group, m.interval, static_cast<uint32_t>(m.sel.size())};
        h = fnv1a(h, mm, sizeof(mm));
    }
    const uint64_t sizes[] = {s->arena_bytes, s->smem_bytes};
    return fnv1a(h, sizes, sizeof(sizes));
}

}  // namespace

BSNN_API bsnn_status bsnn_save_checkpoint(bsnn_sim* sim, const char* path) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require(path != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null path");
        finalize(sim);
        check_device_error(sim);
        std::vector<unsigned char> blob(sim->arena_bytes);
        cuda_check(cudaMemcpy(blob.data(), sim->arena, sim->arena_bytes, cudaMemcpyDeviceToHost), "D2H checkpoint");
        CkptHeader hd{};
        std::memcpy(hd.magic, kCkptMagic, sizeof(kCkptMagic));
        hd.version = kCkptVersion;
        hd.N = sim->N;
        hd.arena_bytes = sim->arena_bytes;
        hd.fingerprint = layout_fingerprint(sim);
        hd.steps_done = sim->steps_done;
        hd.next_clock = sim->next_clock;
        hd.weight_format = sim->weight_format;
        std::ofstream f(path, std::ios::binary | std::ios::trunc);
        require(f.good(), BSNN_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path + " for writing");
        f.write(reinterpret_cast<const char*>(&hd), sizeof(hd));
        f.write(reinterpret_cast<const char*>(blob.data()), static_cast<std::streamsize>(blob.size()));
        require(f.good(), BSNN_ERR_RUNTIME, std::string("write to ") + path + " failed");
    });
}

BSNN_API bsnn_status bsnn_load_checkpoint(bsnn_sim* sim, const char* path) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require(path != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null path");
        finalize(sim);
        require(!sim->failed, BSNN_ERR_STATE, "simulation failed earlier (device timeout)");
        std::ifstream f(path, std::ios::binary);
        require(f.good(), BSNN_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
        CkptHeader hd{};
        f.read(reinterpret_cast<char*>(&hd), sizeof(hd));
        require(f.good() && std::memcmp(hd.magic, kCkptMagic, sizeof(kCkptMagic)) == 0, BSNN_ERR_INVALID_ARGUMENT,
                std::string(path) + " is not a bsnn checkpoint");
        require(hd.version == kCkptVersion, BSNN_ERR_INVALID_ARGUMENT, "unsupported checkpoint version");
        require(hd.N == sim->N && hd.arena_bytes == sim->arena_bytes && hd.weight_format == sim->weight_format &&
                    hd.fingerprint == layout_fingerprint(sim),
                BSNN_ERR_INVALID_ARGUMENT,
                "checkpoint was written by a differently built simulation (components, weight form or GPU)");
        std::vector<unsigned char> blob(hd.arena_bytes);
        f.read(reinterpret_cast<char*>(blob.data()), static_cast<std::streamsize>(blob.size()));
        require(f.good(), BSNN_ERR_INVALID_ARGUMENT, std::string(path) + " is truncated");
        cuda_check(cudaStreamSynchronize(sim->stream), "stream synchronize");
        cuda_check(cudaMemcpy(sim->arena, blob.data(), blob.size(), cudaMemcpyHostToDevice), "H2D checkpoint");
        cuda_check(cudaMemcpy(sim->d_sim, &sim->h, sizeof(DSim), cudaMemcpyHostToDevice), "H2D descriptor");
        sim->steps_done = hd.steps_done;
        sim->next_clock = hd.next_clock;
    });
}

BSNN_API bsnn_status bsnn_read_state(bsnn_sim* sim, int32_t field, uint32_t index, uint32_t offset, uint32_t count,
                                     void* host_out) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        check_device_error(sim);
        const FieldRef f = field_ref(sim, field, index);
        require(offset <= f.len && count <= f.len - offset, BSNN_ERR_OUT_OF_RANGE, "read out of range");
        require(host_out != nullptr || count == 0, BSNN_ERR_INVALID_ARGUMENT, "null output");
        if (count)
            cuda_check(cudaMemcpy(host_out, static_cast<char*>(f.ptr) + 4ull * offset, 4ull * count, cudaMemcpyDeviceToHost),
                       "D2H state");
    });
}

BSNN_API bsnn_status bsnn_write_state(bsnn_sim* sim, int32_t field, uint32_t index, uint32_t offset, uint32_t count,
                                      const void* host_in) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        check_device_error(sim);
        require(field != BSNN_FIELD_SPIKES && field != BSNN_FIELD_PLAST_PRE_WEIGHT_SUMS &&
                    !(field >= BSNN_FIELD_CONN_ROW_SCALE && field <= BSNN_FIELD_CONN_ROW_QUANT_SCALE),
                BSNN_ERR_INVALID_ARGUMENT, "field is not writable");
        const FieldRef f = field_ref(sim, field, index);
        require(offset <= f.len && count <= f.len - offset, BSNN_ERR_OUT_OF_RANGE, "write out of range");
        require(host_in != nullptr || count == 0, BSNN_ERR_INVALID_ARGUMENT, "null input");
        if (count)
            cuda_check(cudaMemcpy(static_cast<char*>(f.ptr) + 4ull * offset, host_in, 4ull * count, cudaMemcpyHostToDevice),
                       "H2D state");
    });
}

BSNN_API bsnn_status bsnn_read_weights(bsnn_sim* sim, uint32_t connection, float* host_out) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        check_device_error(sim);
        require(connection < sim->h.n_conns, BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        require(host_out != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null output");
        const DConn& C = sim->h.conns[connection];
        if (sim->h.wfmt == kFmtF32) {
            cuda_check(cudaMemcpy2D(host_out, sizeof(float) * C.n_post, C.w, sizeof(float) * C.ld,
                                    sizeof(float) * C.n_post, C.n_pre, cudaMemcpyDeviceToHost),
                       "D2H weights");
            return;
        }
        std::vector<float> w(static_cast<size_t>(C.n_pre) * C.ld);
        download_weights(sim, C, w.data());
        for (uint32_t i = 0; i < C.n_pre; ++i)
            std::memcpy(host_out + static_cast<size_t>(i) * C.n_post, &w[static_cast<size_t>(i) * C.ld],
                        sizeof(float) * C.n_post);
    });
}

BSNN_API bsnn_status bsnn_read_weight_copy(bsnn_sim* sim, uint32_t connection, void* host_out) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        check_device_error(sim);
        require(connection < sim->h.n_conns, BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        require(host_out != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null output");
        require(sim->h.wfmt != kFmtF32, BSNN_ERR_INVALID_ARGUMENT, "no weight copy in the BSNN_WEIGHTS_F32 form");
        const DConn& C = sim->h.conns[connection];
        const size_t eb = sim->h.wfmt == kFmtBf16 ? 2 : sim->h.wfmt == kFmtFp8 ? 1 : 4;
        std::vector<unsigned char> tiles(eb * C.qtiles * C.n_pre * 128);
        cuda_check(cudaMemcpy(tiles.data(), C.q, tiles.size(), cudaMemcpyDeviceToHost), "D2H weight copy");
        unsigned char* out = static_cast<unsigned char*>(host_out);
        for (uint32_t i = 0; i < C.n_pre; ++i)
            for (uint32_t q0 = 0; q0 < C.n_post; q0 += 128)
                std::memcpy(out + eb * (static_cast<size_t>(i) * C.n_post + q0), &tiles[eb * copy_index(C.n_pre, i, q0)],
                            eb * std::min<uint32_t>(128, C.n_post - q0));
    });
}

BSNN_API bsnn_status bsnn_read_spike_bits(bsnn_sim* sim, uint32_t monitor, uint32_t* host_out, int32_t flush) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        check_device_error(sim);
        require(monitor < sim->h.n_mons && sim->h.mons[monitor].kind == kMonSpikes, BSNN_ERR_OUT_OF_RANGE,
                "not a spike recorder");
        const DMon& M = sim->h.mons[monitor];
        const size_t bytes = sizeof(uint32_t) * static_cast<size_t>(M.interval) * M.words;
        cuda_check(cudaMemcpy(host_out, M.bits, bytes, cudaMemcpyDeviceToHost), "D2H spike ring");
        if (flush) cuda_check(cudaMemsetAsync(M.bits, 0, bytes, sim->stream), "flush spike ring");
    });
}

BSNN_API bsnn_status bsnn_read_spike_history(bsnn_sim* sim, uint32_t monitor, uint32_t* host_out, int32_t flush) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        check_device_error(sim);
        require(monitor < sim->h.n_mons && sim->h.mons[monitor].kind == kMonSpikes, BSNN_ERR_OUT_OF_RANGE,
                "not a spike recorder");
        const DMon& M = sim->h.mons[monitor];
        const uint32_t ng = sim->groups[M.group].p.num_neurons;
        std::vector<uint32_t> bits(static_cast<size_t>(M.interval) * M.words);
        cuda_check(cudaMemcpy(bits.data(), M.bits, sizeof(uint32_t) * bits.size(), cudaMemcpyDeviceToHost), "D2H spike ring");
        if (flush) cuda_check(cudaMemsetAsync(M.bits, 0, sizeof(uint32_t) * bits.size(), sim->stream), "flush spike ring");
        for (uint32_t i = 0; i < ng; ++i)
            for (uint32_t slot = 0; slot < M.interval; ++slot)
                host_out[static_cast<size_t>(i) * M.interval + slot] =
                    (bits[static_cast<size_t>(slot) * M.words + (i >> 5)] >> (i & 31u)) & 1u;
    });
}

BSNN_API bsnn_status bsnn_read_voltage_history(bsnn_sim* sim, uint32_t monitor, float* host_out, int32_t flush) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        check_device_error(sim);
        require(monitor < sim->h.n_mons && sim->h.mons[monitor].kind == kMonVoltage, BSNN_ERR_OUT_OF_RANGE,
                "not a voltage recorder");
        const DMon& M = sim->h.mons[monitor];
        const auto& sel = sim->mons[monitor].sel;
        std::vector<float> vh(static_cast<size_t>(M.interval) * M.n_sel);
        cuda_check(cudaMemcpy(vh.data(), M.vh, sizeof(float) * vh.size(), cudaMemcpyDeviceToHost), "D2H voltage ring");
        if (flush) cuda_check(cudaMemsetAsync(M.vh, 0, sizeof(float) * vh.size(), sim->stream), "flush voltage ring");
        // first occurrence of each selected neuron holds its column
        std::vector<int32_t> first(sim->groups[M.group].p.num_neurons, -1);
        for (size_t k = 0; k < sel.size(); ++k)
            if (first[sel[k]] < 0) first[sel[k]] = static_cast<int32_t>(k);
        for (size_t k = 0; k < sel.size(); ++k) {
            const uint32_t col = static_cast<uint32_t>(first[sel[k]]);
            for (uint32_t slot = 0; slot < M.interval; ++slot)
                host_out[k * M.interval + slot] = vh[static_cast<size_t>(slot) * M.n_sel + col];
        }
    });
}

BSNN_API bsnn_status bsnn_get_device_pointer(const bsnn_sim* sim, int32_t field, uint32_t index, void** out) {
    if (!sim || !out) return BSNN_ERR_INVALID_ARGUMENT;
    bsnn_sim* s = const_cast<bsnn_sim*>(sim);
    return guarded(s, [&] {
        finalize(s);
        *out = field_ref(s, field, index).ptr;
    });
}

BSNN_API bsnn_status bsnn_set_monitor_output(bsnn_sim* sim, uint32_t monitor, const char* path) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require(monitor < sim->mons.size(), BSNN_ERR_OUT_OF_RANGE, "monitor index out of range");
        require(path != nullptr && *path != '\0', BSNN_ERR_INVALID_ARGUMENT, "empty output path");
        HostMon& m = sim->mons[monitor];
        const std::string p(path);
        if (m.kind == kMonSpikes) {
            // SpikeRecorder ctor: the file is truncated and gets its header now (spike_recorder.cpp:3-28)
            if (sim->writer) sim->writer->drain();
            m.spike_out = std::make_shared<std::ofstream>(p, std::ios::out | std::ios::trunc | std::ios::binary);
            if (m.spike_out->good()) *m.spike_out << "clock_step, neuron_ids\n";
        } else {
            // per-step file names are made by inserting "_step<N>" before ".txt" (voltage_recorder.cpp:62-64)
            require(p.rfind(".txt") != std::string::npos, BSNN_ERR_OUT_OF_RANGE, "output path must contain \".txt\"");
        }
        m.path = p;
    });
}

BSNN_API bsnn_status bsnn_add_weight_recorder(bsnn_sim* sim, uint32_t connection, const char* path) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        require(connection < sim->conns.size(), BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        require(path != nullptr && std::string(path).rfind(".txt") != std::string::npos, BSNN_ERR_OUT_OF_RANGE,
                "output path must contain \".txt\"");
        sim->wrecs.push_back(HostWeightRec{connection, std::string(path)});
    });
}

BSNN_API bsnn_status bsnn_record(bsnn_sim* sim, uint32_t clock_step) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] { record_all(sim, clock_step); });
}

BSNN_API bsnn_status bsnn_flush_records(bsnn_sim* sim) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        if (sim->writer) sim->writer->drain();
        for (auto& m : sim->mons)
            if (m.spike_out) m.spike_out->flush();
    });
}

BSNN_API bsnn_status bsnn_run_system(bsnn_sim* sim, uint32_t total_clock_steps) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        const uint32_t interval = sim->desc.recording_interval_steps;
        const auto start_time = std::chrono::steady_clock::now();
        uint32_t step = 0;
        while (step < total_clock_steps) {
            // record after every step that is a multiple of the interval (system.cpp:71-76)
            const uint64_t next = (static_cast<uint64_t>(step) + interval - 1u) / interval * interval;
            const uint32_t end = static_cast<uint32_t>(std::min<uint64_t>(total_clock_steps, next + 1u));
            run_steps(sim, step, end - step);
            if (end == next + 1u) {
                record_all(sim, static_cast<uint32_t>(next));
                if (sim->progress) {  // the progress line of system.cpp:78-81, after the record
                    const std::chrono::duration<float> elapsed = std::chrono::steady_clock::now() - start_time;
                    std::cout << "Completed clock step: " << next << " | elapsed: " << elapsed.count() << "s\n" << std::flush;
                }
            }
            step = end;
        }
    });
}

BSNN_API bsnn_status bsnn_set_progress_output(bsnn_sim* sim, int32_t enabled) {
    if (!sim) return BSNN_ERR_INVALID_ARGUMENT;
    sim->progress = enabled != 0;
    return BSNN_OK;
}

BSNN_API bsnn_status bsnn_memory_report(bsnn_sim* sim, char* buf, uint64_t capacity) {
    if (!sim || (!buf && capacity)) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        finalize(sim);
        const uint64_t total = sim->arena_bytes;
        char text[160];
        std::snprintf(text, sizeof(text), "Total GPU Memory Allocated: %llu bytes (%f MB)",
                      static_cast<unsigned long long>(total), static_cast<double>(total) / (1024.0 * 1024.0));
        require(capacity > std::strlen(text), BSNN_ERR_OUT_OF_RANGE,
                "memory report needs " + std::to_string(std::strlen(text) + 1) + " bytes of buffer");
        std::memcpy(buf, text, std::strlen(text) + 1);
    });
}

BSNN_API bsnn_status bsnn_connection_propagate(const bsnn_connection_view* view, void* stream) {
    return guarded(nullptr, [&] {
        const char* bad = prop::check_view(view);
        require(bad == nullptr, BSNN_ERR_INVALID_ARGUMENT, bad ? bad : "");
        int dev = 0, sms = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        const uint32_t n_post = view->post_group_num_neurons;
        const uint32_t splits = prop::choose_splits(view->pre_group_num_neurons, n_post, sms);
        auto st = static_cast<cudaStream_t>(stream);
        float* scratch = nullptr;
        cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&scratch), sizeof(float) * splits * size_t(n_post), st),
                   "cudaMallocAsync (propagate scratch)");
        const cudaError_t launched = prop::enqueue(view, splits, scratch, st);
        const cudaError_t freed = cudaFreeAsync(scratch, st);
        cuda_check(launched, "connection propagate launch");
        cuda_check(freed, "cudaFreeAsync (propagate scratch)");
    });
}

BSNN_API bsnn_status bsnn_connection_propagate_noalloc(const bsnn_connection_view* view, void* stream) {
    return guarded(nullptr, [&] {
        const char* bad = prop::check_view(view);
        require(bad == nullptr, BSNN_ERR_INVALID_ARGUMENT, bad ? bad : "");
        const uint32_t n_post = view->post_group_num_neurons;
        require(n_post <= prop::kStaticScratchFloats, BSNN_ERR_OUT_OF_RANGE,
                "post_group_num_neurons " + std::to_string(n_post) +
                    " exceeds the static propagate scratch limit of " + std::to_string(prop::kStaticScratchFloats));
        int dev = 0, sms = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        float* scratch = nullptr;
        cuda_check(prop::static_scratch(dev, &scratch), "static propagate scratch set-up (cudaGetSymbolAddress)");
        const uint32_t splits = prop::static_splits(view->pre_group_num_neurons, n_post, sms);
        cuda_check(prop::enqueue(view, splits, scratch, static_cast<cudaStream_t>(stream)),
                   "connection propagate launch");
    });
}

}  // extern "C"

#ifdef BSNN_PHASE_TIMING
// Profiling builds only (-DBSNN_PHASE_TIMING, `make libbsnn_phase.so`): SM clock cycles per phase of
// the step kernel (the slots listed beside BSNN_TMARK in step_kernel.cuh), accumulated since
// creation; out[cta * kPhaseSlots + slot] for every CTA of the grid.
extern "C" BSNN_API bsnn_status bsnn_debug_phase_ns(bsnn_sim* sim, unsigned long long* out) {
    if (!sim || !out) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(sim, [&] {
        check_device_error(sim);
        cuda_check(cudaMemcpy(out, sim->h.phase_ns, kPhaseSlots * sizeof(unsigned long long) * sim->grid,
                              cudaMemcpyDeviceToHost),
                   "D2H");
    });
}
#endif
#include "generate.cuh"

extern "C" {

// Distance-dependent weights generated on the GPU (see generate.cuh): pre_xy / post_xy hold
// (x, y) per neuron; w_out (host memory, n_pre * n_post floats, row-major) receives the matrix.
BSNN_API bsnn_status bsnn_generate_distance_weights(const float* pre_xy, uint32_t n_pre, const float* post_xy,
                                                    uint32_t n_post, const bsnn_weight_generation_params* params,
                                                    uint64_t seed, int32_t device, float* w_out) {
    return guarded(nullptr, [&] {
        require(pre_xy && post_xy && params && w_out, BSNN_ERR_INVALID_ARGUMENT, "null argument");
        require(n_pre > 0 && n_post > 0, BSNN_ERR_INVALID_ARGUMENT, "neuron groups must not be empty");
        require(params->spread_scale > 0.0f, BSNN_ERR_INVALID_ARGUMENT, "spread_scale must be > 0");
        require(params->max_weight_value >= 0.0f, BSNN_ERR_INVALID_ARGUMENT,
                "max_weight_value must be >= 0 (the reference rejects negative weights)");
        int nd = 0;
        cuda_check(cudaGetDeviceCount(&nd), "cudaGetDeviceCount");
        require(device >= 0 && device < nd, BSNN_ERR_INVALID_ARGUMENT, "device ordinal out of range");
        DeviceGuard g(device);
        const uint64_t n = static_cast<uint64_t>(n_pre) * n_post;
        GenParams P{};
        P.max_weight_value = params->max_weight_value;
        P.max_distance = params->max_distance;
        P.spread_scale = params->spread_scale;
        P.probability_multiplier = params->probability_multiplier;
        P.lx = params->x_location_length;
        P.ly = params->y_location_length;
        P.value_dropoff = params->weight_value_normal_dropoff ? 1u : 0u;
        P.normal_probability = params->probabilistic_normal_not_uniform ? 1u : 0u;
        P.no_diagonal = params->no_diagonal_connections ? 1u : 0u;
        P.uniform_values = params->uniform_values ? 1u : 0u;
        P.seed_lo = static_cast<uint32_t>(seed);
        P.seed_hi = static_cast<uint32_t>(seed >> 32);
        cudaStream_t st = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
        unsigned char* buf = nullptr;
        const size_t xy = 8ull * (n_pre + n_post);
        const cudaError_t me = cudaMallocAsync(reinterpret_cast<void**>(&buf), xy + 4ull * n + 256, st);
        if (me != cudaSuccess) {
            cudaStreamDestroy(st);
            cuda_check(me, "cudaMallocAsync generation buffer");
        }
        float* dpre = reinterpret_cast<float*>(buf);
        float* dpost = dpre + 2ull * n_pre;
        float* dw = reinterpret_cast<float*>(buf + ((xy + 255) & ~size_t(255)));
        cudaError_t e = cudaMemcpyAsync(dpre, pre_xy, 8ull * n_pre, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dpost, post_xy, 8ull * n_post, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            const uint64_t blocks = (n + 255) / 256;
            bsnn_generate_weights_kernel<<<static_cast<uint32_t>(blocks), 256, 0, st>>>(dpre, n_pre, dpost, n_post, P, dw);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(w_out, dw, 4ull * n, cudaMemcpyDeviceToHost, st);
        cudaFreeAsync(buf, st);
        const cudaError_t se = cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        cuda_check(e, "weight generation");
        cuda_check(se, "weight generation sync");
    });
}

}  // extern "C"

#include "batch_api.cuh"
#include "adjoint_api.cuh"
