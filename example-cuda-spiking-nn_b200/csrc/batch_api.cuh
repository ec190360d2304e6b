// batch_api.cuh -- host side of the batched form (bsnn_batch_* in include/bsnn.h); included at
// the end of bsnn_api.cu, whose helpers (cuda_check, require, ApiError, Arena) it uses.
//
// A batch is built from size classes (one shared weight set each, stored as BF16 W^T tiles in
// the tensor cores' canonical layout) and instances (per-instance neuron-group parameters,
// seed and stimulus).  The first call that needs the device plans the GEMM work units (a K chunk
// of one 128-post tile of one class and presynaptic side, sorted longest first), places the
// operand ring, instance table and neuron state in shared memory, allocates one arena and
// uploads.  bsnn_batch_run replays a captured CUDA graph of the cooperative launch per chunk of
// steps.  bsnn_batch_autotune times candidate unit sizes and ring depths on the device before
// the first step and keeps the fastest.
#pragma once

#include "batch_kernel.cuh"

struct bsnn_batch {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::string err;

    struct HClass {
        uint32_t E, I;
        std::vector<uint16_t> A[2];  // tiled W^T, BF16 bits
        float r_decay[2], d_decay[2], norm[2];
        std::vector<uint32_t> instances;
    };
    struct HInst {
        uint32_t cls;
        bsnn_neuron_group_params g[2];
        uint32_t seed;
        std::vector<uint32_t> counts;
        std::vector<uint32_t> neurons;
        std::vector<float> deltas;
    };
    std::vector<HClass> classes;
    std::vector<HInst> insts;
    bool noise_on = true;

    bool finalized = false, failed = false;
    uint64_t wait_limit_ns = kDefaultWaitLimitNs;  // bound of every device-side wait
    unsigned char* arena = nullptr;
    size_t arena_bytes = 0;
    BSim h{};
    BSim* d_sim = nullptr;
    std::vector<uint32_t> pos;    // instance id -> position in the class-sorted order (the device's
                                  // instance table is in this order)
    std::vector<uint32_t> nbase;  // per instance id: first neuron (neurons are numbered class by class)
    uint32_t grid = 0;
    size_t smem = 0;
    uint64_t steps_done = 0, launches = 0;
    uint32_t steps_per_launch = 1000;
    std::map<uint32_t, cudaGraphExec_t> graphs;
    float* scratch = nullptr;  // [2][max N] for reads of g with the pending propagation
    const void* kernel = nullptr;  // the flow or phased kernel, state in shared memory or not
    int32_t form = BSNN_BATCH_FORM_PHASED;
    uint32_t tune_kc = 0;          // K tiles per GEMM unit (0: the default rule)
    uint32_t tune_stages = 0;      // operand stages (0: the placement's choice)
    uint32_t kc = 0;               // the unit size in use

    ~bsnn_batch() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        if (arena) cudaFree(arena);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

template <class F>
bsnn_status guarded_batch(bsnn_batch* b, F&& f) {
    try {
        int prev = -1;
        if (b) {
            cudaGetDevice(&prev);
            cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
        }
        f();
        if (b && prev >= 0) cudaSetDevice(prev);
        return BSNN_OK;
    } catch (const ApiError& e) {
        if (b) b->err = e.what();
        g_thread_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        if (b) b->err = e.what();
        g_thread_error = e.what();
        return BSNN_ERR_RUNTIME;
    }
}

uint16_t host_bf16(float v) {  // round to nearest even (finite values)
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return static_cast<uint16_t>(u >> 16);
}

BGroupP batch_group(const bsnn_neuron_group_params& p) {
    BGroupP G{};
    G.refractory_steps = p.refractory_steps;
    G.has_bg_e = p.mean_background_excitatory_spikes > 0.0f;
    G.has_bg_i = p.mean_background_inhibitory_spikes > 0.0f;
    G.dt_c = p.timestep / p.membrane_capacitance;  // the quotient the reference forms every step
    G.g_leak = p.g_leak;
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
    return G;
}

void batch_finalize(bsnn_batch* b) {
    if (b->finalized) return;
    require(!b->classes.empty() && !b->insts.empty(), BSNN_ERR_STATE, "a batch needs at least one class and one instance");
    BSim& h = b->h;
    h = BSim{};
    h.n_classes = static_cast<uint32_t>(b->classes.size());
    h.n_inst = static_cast<uint32_t>(b->insts.size());
    h.noise_on = b->noise_on ? 1 : 0;

    // Instances in class order: the instance's row in its class's B operand is its rank there, and
    // neurons are numbered class by class (a class's neurons are contiguous).
    std::vector<uint32_t> row(h.n_inst), by_pos;
    b->nbase.assign(h.n_inst, 0);
    b->pos.assign(h.n_inst, 0);
    uint32_t n_neurons = 0;
    std::vector<uint32_t> cls_nbase(h.n_classes), cls_nlen(h.n_classes);
    for (uint32_t c = 0; c < h.n_classes; ++c) {
        const auto& HC = b->classes[c];
        cls_nbase[c] = n_neurons;
        for (uint32_t r = 0; r < HC.instances.size(); ++r) {
            const uint32_t i = HC.instances[r];
            row[i] = r;
            b->pos[i] = static_cast<uint32_t>(by_pos.size());
            by_pos.push_back(i);
            b->nbase[i] = n_neurons;
            n_neurons += HC.E + HC.I;
        }
        cls_nlen[c] = n_neurons - cls_nbase[c];
    }
    h.n_neurons = n_neurons;

    // Work units: K chunks of at most kc tiles, kc chosen so the largest unit is about the
    // average work per CTA.
    const uint32_t n_ctas = static_cast<uint32_t>(b->sm_count);
    uint64_t total_tiles = 0;
    for (const auto& HC : b->classes) {
        const uint32_t MT = (HC.E + HC.I + 127) / 128;
        total_tiles += static_cast<uint64_t>(MT) * ((HC.E + 63) / 64 + (HC.I + 63) / 64);
    }
    const uint32_t kc = b->tune_kc ? b->tune_kc
                                   : std::max<uint32_t>(4u, static_cast<uint32_t>((total_tiles + n_ctas - 1) / n_ctas));
    b->kc = kc;
    std::vector<BUnit> units;
    size_t part_floats = 0;
    for (uint32_t c = 0; c < h.n_classes; ++c) {
        const auto& HC = b->classes[c];
        BClass& C = h.cls[c];
        C.E = HC.E;
        C.I = HC.I;
        C.N = HC.E + HC.I;
        C.n_inst = static_cast<uint32_t>(HC.instances.size());
        C.NP = std::max<uint32_t>(8u, round_up(C.n_inst, 8));
        require(C.NP <= 128, BSNN_ERR_INVALID_ARGUMENT, "at most 128 instances per size class");
        C.nbase = cls_nbase[c];
        C.nlen = cls_nlen[c];
        C.MT = (C.N + 127) / 128;
        for (int sd = 0; sd < 2; ++sd) {
            const uint32_t K = sd == 0 ? C.E : C.I;
            C.KT[sd] = (K + 63) / 64;
            C.nkc[sd] = (C.KT[sd] + kc - 1) / kc;
            C.pbase[sd] = part_floats;
            C.r_decay[sd] = HC.r_decay[sd];
            C.d_decay[sd] = HC.d_decay[sd];
            C.norm[sd] = HC.norm[sd];
            for (uint32_t mt = 0; mt < C.MT; ++mt)
                for (uint32_t q = 0; q < C.nkc[sd]; ++q) {
                    BUnit U{};
                    U.cls = c;
                    U.side = static_cast<uint32_t>(sd);
                    U.mt = mt;
                    U.k0 = q * kc;
                    U.k1 = std::min(C.KT[sd], (q + 1) * kc);
                    U.part = part_floats;
                    part_floats += static_cast<size_t>(C.NP) * 128u;
                    units.push_back(U);
                }
        }
    }
    h.n_units = static_cast<uint32_t>(units.size());
    // Class processing order of the flow form: the classes with the most GEMM work first (their
    // chains are the longest).
    std::vector<double> cls_work(h.n_classes, 0.0);
    for (const BUnit& U : units) cls_work[U.cls] += static_cast<double>(U.k1 - U.k0);
    std::vector<uint32_t> cls_order(h.n_classes);
    std::iota(cls_order.begin(), cls_order.end(), 0u);
    std::stable_sort(cls_order.begin(), cls_order.end(), [&](uint32_t a, uint32_t c) { return cls_work[a] > cls_work[c]; });
    std::vector<uint32_t> cls_rank(h.n_classes);
    for (uint32_t p = 0; p < h.n_classes; ++p) {
        h.order[p] = cls_order[p];
        cls_rank[cls_order[p]] = p;
    }
    for (const BUnit& U : units) ++h.units_of[U.cls];
    const bool flow = b->form == BSNN_BATCH_FORM_FLOW;
    // The dispenser's order: longest first (phased form), or by class processing order and longest
    // first within a class (flow form: a step's units are taken in the order its classes become
    // ready).
    std::vector<uint32_t> order(units.size());
    std::iota(order.begin(), order.end(), 0u);
    auto cost = [&](uint32_t u) { return static_cast<double>(units[u].k1 - units[u].k0) + 2.0; };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) {
        if (flow && units[a].cls != units[c].cls) return cls_rank[units[a].cls] < cls_rank[units[c].cls];
        return cost(a) > cost(c);
    });
    std::vector<BUnit> units_sorted;
    units_sorted.reserve(units.size());
    for (uint32_t u : order) units_sorted.push_back(units[u]);

    // Stimulus: one CSR over all instances, events of a step sorted by neuron.
    uint32_t stim_len = 0;
    for (const auto& I : b->insts) stim_len = std::max<uint32_t>(stim_len, static_cast<uint32_t>(I.counts.size()));
    std::vector<std::vector<std::pair<uint32_t, float>>> per_step(stim_len);
    for (uint32_t i = 0; i < h.n_inst; ++i) {
        const auto& I = b->insts[i];
        size_t e = 0;
        for (uint32_t t = 0; t < I.counts.size(); ++t)
            for (uint32_t k = 0; k < I.counts[t]; ++k, ++e) per_step[t].emplace_back(b->nbase[i] + I.neurons[e], I.deltas[e]);
    }
    std::vector<uint32_t> stim_off(stim_len + 1, 0), ev_neuron;
    std::vector<float> ev_delta;
    for (uint32_t t = 0; t < stim_len; ++t) {
        std::stable_sort(per_step[t].begin(), per_step[t].end(),
                         [](const auto& a, const auto& c) { return a.first < c.first; });
        for (const auto& ev : per_step[t]) {
            ev_neuron.push_back(ev.first);
            ev_delta.push_back(ev.second);
        }
        stim_off[t + 1] = static_cast<uint32_t>(ev_neuron.size());
    }

    // Arena.
    Arena A;
    const size_t fN = sizeof(float) * n_neurons;
    size_t o_state[8];
    for (auto& o : o_state) o = A.take(fN);
    const size_t o_ref = A.take(sizeof(uint32_t) * n_neurons), o_spk = A.take(sizeof(uint32_t) * n_neurons);
    const size_t o_cnt = A.take(sizeof(unsigned long long) * 2 * h.n_inst);
    const size_t o_pns = A.take(sizeof(unsigned long long) * 8 * n_ctas);
    const size_t o_inst = A.take(sizeof(BInst) * h.n_inst);
    const size_t o_units = A.take(sizeof(BUnit) * units_sorted.size());
    const size_t o_ctr = A.take(sizeof(unsigned long long));
    const size_t o_nready = A.take(sizeof(unsigned long long) * kBatchMaxClasses);
    const size_t o_udone = A.take(sizeof(unsigned long long) * kBatchMaxClasses);
    const size_t o_part = A.take(sizeof(float) * std::max<size_t>(part_floats, 1));
    size_t o_a[kBatchMaxClasses][2], o_x[kBatchMaxClasses][2];
    for (uint32_t c = 0; c < h.n_classes; ++c)
        for (int sd = 0; sd < 2; ++sd) {
            const BClass& C = h.cls[c];
            o_a[c][sd] = A.take(static_cast<size_t>(C.MT) * C.KT[sd] * kATileBytes);
            o_x[c][sd] = A.take(static_cast<size_t>(C.KT[sd]) * 2u * C.NP * 64u * 2u);
        }
    const size_t o_soff = A.take(sizeof(uint32_t) * stim_off.size());
    const size_t o_evn = A.take(sizeof(uint32_t) * std::max<size_t>(ev_neuron.size(), 1));
    const size_t o_evd = A.take(sizeof(float) * std::max<size_t>(ev_delta.size(), 1));
    const size_t o_bar = A.take(sizeof(unsigned long long)), o_err = A.take(sizeof(int32_t));
    const size_t o_sd = A.take(sizeof(unsigned long long));
    uint32_t max_n = 0;
    for (const auto& HC : b->classes) max_n = std::max(max_n, HC.E + HC.I);
    const size_t o_scr = A.take(sizeof(float) * 2 * max_n);
    const size_t o_sim = A.take(sizeof(BSim));
    cuda_check(cudaMalloc(&b->arena, A.size), "cudaMalloc batch arena");
    b->arena_bytes = A.size;
    unsigned char* base = b->arena;
    cuda_check(cudaMemset(base, 0, A.size), "cudaMemset batch arena");
    auto F = [&](size_t o) { return reinterpret_cast<float*>(base + o); };
    float** fields[8] = {&h.v, &h.istim, &h.er, &h.ed, &h.ir, &h.id, &h.tr, &h.td};
    for (int k = 0; k < 8; ++k) *fields[k] = F(o_state[k]);
    h.refrac = reinterpret_cast<uint32_t*>(base + o_ref);
    h.spikes = reinterpret_cast<uint32_t*>(base + o_spk);
    h.spike_counts = reinterpret_cast<unsigned long long*>(base + o_cnt);
    h.partials = F(o_part);
    h.barrier = reinterpret_cast<unsigned long long*>(base + o_bar);
    h.error = reinterpret_cast<int32_t*>(base + o_err);
    h.wait_limit_ns = b->wait_limit_ns;
    h.steps_done = reinterpret_cast<unsigned long long*>(base + o_sd);
    b->scratch = F(o_scr);

    // neuron -> instance, instance table, initial voltages and refractory counters

    std::vector<BInst> inst(h.n_inst);  // in position order
    std::vector<float> v0(n_neurons);
    for (uint32_t i = 0; i < h.n_inst; ++i) {
        const auto& I = b->insts[i];
        const auto& HC = b->classes[I.cls];
        BInst& BI = inst[b->pos[i]];
        BI.id = i;
        BI.cls = I.cls;
        BI.row = row[i];
        BI.nbase = b->nbase[i];
        BI.seed = I.seed;
        BI.g[0] = batch_group(I.g[0]);
        BI.g[1] = batch_group(I.g[1]);
        for (uint32_t j = 0; j < HC.E + HC.I; ++j)
            v0[b->nbase[i] + j] = I.g[j < HC.E ? 0 : 1].v_rest;  // NeuronGroup::initialize_data
    }
    h.phase_ns = reinterpret_cast<unsigned long long*>(base + o_pns);
    h.inst = reinterpret_cast<const BInst*>(base + o_inst);
    h.units = reinterpret_cast<const BUnit*>(base + o_units);
    h.unit_ctr = reinterpret_cast<unsigned long long*>(base + o_ctr);
    h.nready = reinterpret_cast<unsigned long long*>(base + o_nready);
    h.udone = reinterpret_cast<unsigned long long*>(base + o_udone);
    cuda_check(cudaMemcpy(base + o_inst, inst.data(), sizeof(BInst) * inst.size(), cudaMemcpyHostToDevice), "H2D");
    cuda_check(cudaMemcpy(h.v, v0.data(), fN, cudaMemcpyHostToDevice), "H2D v");
    cuda_check(cudaMemcpy(base + o_units, units_sorted.data(), sizeof(BUnit) * units_sorted.size(),
                          cudaMemcpyHostToDevice),
               "H2D units");
    for (uint32_t c = 0; c < h.n_classes; ++c)
        for (int sd = 0; sd < 2; ++sd) {
            h.cls[c].A[sd] = reinterpret_cast<const uint16_t*>(base + o_a[c][sd]);
            h.cls[c].X[sd] = reinterpret_cast<uint16_t*>(base + o_x[c][sd]);
            const auto& tiles = b->classes[c].A[sd];
            cuda_check(cudaMemcpy(base + o_a[c][sd], tiles.data(), sizeof(uint16_t) * tiles.size(), cudaMemcpyHostToDevice),
                       "H2D weight tiles");
        }
    h.stim_len = stim_len;
    h.stim_off = reinterpret_cast<const uint32_t*>(base + o_soff);
    h.ev_neuron = reinterpret_cast<const uint32_t*>(base + o_evn);
    h.ev_delta = reinterpret_cast<const float*>(base + o_evd);
    cuda_check(cudaMemcpy(base + o_soff, stim_off.data(), sizeof(uint32_t) * stim_off.size(), cudaMemcpyHostToDevice), "H2D");
    if (!ev_neuron.empty()) {
        cuda_check(cudaMemcpy(base + o_evn, ev_neuron.data(), sizeof(uint32_t) * ev_neuron.size(), cudaMemcpyHostToDevice), "H2D");
        cuda_check(cudaMemcpy(base + o_evd, ev_delta.data(), sizeof(float) * ev_delta.size(), cudaMemcpyHostToDevice), "H2D");
    }
    b->d_sim = reinterpret_cast<BSim*>(base + o_sim);
    b->grid = n_ctas;
    // Shared memory: the operand ring, then optionally the instance table and the CTA's neuron
    // state.  Keeping the state resident matters most (phase A then touches global memory only
    // for the partial sums and x), then at least three stages, then the table.
    uint32_t max_b = 0;
    for (uint32_t c = 0; c < h.n_classes; ++c) max_b = std::max(max_b, 2u * h.cls[c].NP * 128u);
    h.stage_bytes = (kATileBytes + max_b + 1023u) & ~1023u;
    // Neurons per CTA: a contiguous range (phased form), or a slice of every class (flow form).
    h.per_cta = (n_neurons + n_ctas - 1) / n_ctas;
    if (flow) {
        h.per_cta = 0;
        for (uint32_t c = 0; c < h.n_classes; ++c) h.per_cta += (cls_nlen[c] + n_ctas - 1) / n_ctas;
    }
    int optin = 0;
    cuda_check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device), "smem attr");
    const size_t avail = static_cast<size_t>(optin) - 4096;  // the kernel's static shared memory
    const size_t table_bytes = sizeof(BInst) * h.n_inst;
    const size_t state_bytes = (static_cast<size_t>(h.per_cta) * (9u * 4u + 1u) + 15u) & ~size_t(15);
    const size_t noise_bytes = sizeof(uint16_t) * h.per_cta;  // the next step's Poisson counts
    const char* env_state = std::getenv("BSNN_BATCH_STATE");    // "global": keep the state in global memory
    const char* env_stages = std::getenv("BSNN_BATCH_STAGES");  // 2 .. kBatchStages
    const bool allow_smem_state = !(env_state && std::string(env_state) == "global");
    const uint32_t forced_stages =
        b->tune_stages ? b->tune_stages : env_stages ? static_cast<uint32_t>(std::atoi(env_stages)) : 0u;
    struct Choice { uint32_t state, stages, table; };
    // Preference without a forced depth: the state resident with 4 or 3 stages, then fewer stages,
    // then the state in global memory with 4 or 3 stages.  A forced depth (the autotuner tries
    // every depth up to kBatchStages) takes the first placement that fits it: deep rings leave no
    // room for the state, so they trade phase A's state traffic for more operand tiles in flight.
    std::vector<Choice> choices = {{1, 4, 1}, {1, 3, 1}, {1, 4, 0}, {1, 3, 0}, {1, 2, 1}, {1, 2, 0},
                                   {0, 4, 1}, {0, 3, 1}, {0, 4, 0}, {0, 3, 0}, {0, 2, 1}, {0, 2, 0}};
    for (uint32_t st = kBatchStages; st > 4; --st)
        for (uint32_t state = 2; state-- > 0;)
            for (uint32_t table = 2; table-- > 0;) choices.push_back({state, st, table});
    bool placed = false;
    for (const Choice& ch : choices) {
        if (ch.state && !allow_smem_state) continue;
        if (forced_stages && ch.stages != forced_stages) continue;
        const size_t ring = static_cast<size_t>(ch.stages) * h.stage_bytes;
        const size_t noise_off = (ring + (ch.table ? table_bytes : 0) + 15u) & ~size_t(15);
        const size_t state_off = (noise_off + noise_bytes + 15u) & ~size_t(15);
        const size_t need = state_off + (ch.state ? state_bytes : 0);
        if (need > avail) continue;
        h.n_stages = ch.stages;
        h.inst_in_smem = ch.table;
        h.state_in_smem = ch.state;
        h.state_off = static_cast<uint32_t>(state_off);
        h.noise_off = static_cast<uint32_t>(noise_off);
        b->smem = need;
        placed = true;
        break;
    }
    require(placed, BSNN_ERR_INVALID_ARGUMENT, "batch too large: the operand stages do not fit in shared memory");
    // The phased form waits per size class instead of at grid barriers (BSNN_BATCH_CLASSWAIT=0: grid
    // barriers); ctas_of[c] counts the CTAs whose neuron range holds neurons of class c.
    const char* env_cw = std::getenv("BSNN_BATCH_CLASSWAIT");
    h.classwait = !flow && !(env_cw && std::string(env_cw) == "0");
    for (uint32_t c = 0; c < h.n_classes; ++c) {
        h.ctas_of[c] = 0;
        for (uint32_t cta = 0; cta < n_ctas; ++cta) {
            const uint64_t a = static_cast<uint64_t>(cta) * h.per_cta, e = std::min<uint64_t>(a + h.per_cta, n_neurons);
            if (a < e && a < cls_nbase[c] + cls_nlen[c] && cls_nbase[c] < e) ++h.ctas_of[c];
        }
    }
    cuda_check(cudaMemcpy(b->d_sim, &h, sizeof(BSim), cudaMemcpyHostToDevice), "H2D batch sim");
    if (flow)
        b->kernel = h.state_in_smem ? reinterpret_cast<const void*>(&bsnn_batch_flow_kernel<true>)
                                    : reinterpret_cast<const void*>(&bsnn_batch_flow_kernel<false>);
    else
        b->kernel = h.state_in_smem ? reinterpret_cast<const void*>(&bsnn_batch_kernel<true>)
                                    : reinterpret_cast<const void*>(&bsnn_batch_kernel<false>);
    // the limit is per function and shared by every batch in the process: allow the most any
    // batch may use, so one batch's smaller setting never invalidates another's launches
    cuda_check(cudaFuncSetAttribute(b->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(avail)),
               "batch smem");
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->kernel,
                                                             kBatchThreads, b->smem),
               "batch occupancy");
    require(per_sm >= 1, BSNN_ERR_RUNTIME, "batch kernel does not fit on an SM");
    b->finalized = true;
}

}  // namespace

namespace {

void batch_check_error(bsnn_batch* b) {
    cuda_check(cudaStreamSynchronize(b->stream), "batch stream synchronize");
    int32_t e = 0;
    cuda_check(cudaMemcpy(&e, b->h.error, sizeof(e), cudaMemcpyDeviceToHost), "D2H batch error flag");
    if (e != kErrNone) {
        b->failed = true;
        throw ApiError(BSNN_ERR_DEVICE_TIMEOUT, "batch kernel: a device-side wait timed out; the batch state is invalid");
    }
}

// Releases the device side (graphs, arena): the next call that needs it plans and uploads anew,
// from step 0.
void batch_teardown(bsnn_batch* b) {
    cuda_check(cudaStreamSynchronize(b->stream), "batch stream synchronize");
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    if (b->arena) cudaFree(b->arena);
    b->arena = nullptr;
    b->arena_bytes = 0;
    b->d_sim = nullptr;
    b->finalized = false;
    b->steps_done = 0;
}

void batch_launch(bsnn_batch* b, uint32_t n_steps) {
    auto it = b->graphs.find(n_steps);
    if (it == b->graphs.end()) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cuda_check(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "batch capture");
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(b->grid);
        cfg.blockDim = dim3(kBatchThreads);
        cfg.dynamicSmemBytes = b->smem;
        cfg.stream = b->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const BSim* arg0 = b->d_sim;
        void* args[2] = {&arg0, &n_steps};
        const cudaError_t le = cudaLaunchKernelExC(&cfg, b->kernel, args);
        const cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
        cuda_check(le, "batch launch (capture)");
        cuda_check(ce, "batch end capture");
        cuda_check(cudaGraphInstantiate(&exec, graph, 0), "batch graph instantiate");
        cudaGraphDestroy(graph);
        it = b->graphs.emplace(n_steps, exec).first;
    }
    cuda_check(cudaGraphLaunch(it->second, b->stream), "batch graph launch");
    ++b->launches;
}

}  // namespace

extern "C" {

BSNN_API bsnn_status bsnn_batch_create(int32_t device, bsnn_batch** out) {
    if (!out) return BSNN_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    return guarded_batch(nullptr, [&] {
        int n = 0;
        cuda_check(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
        require(device >= 0 && device < n, BSNN_ERR_INVALID_ARGUMENT, "device ordinal out of range");
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        auto b = std::make_unique<bsnn_batch>();
        b->device = device;
        cuda_check(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device), "SM count");
        int major = 0;
        cuda_check(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "compute capability");
        require(major == 10, BSNN_ERR_RUNTIME, "the batched form needs an sm_100 GPU (tcgen05 tensor cores)");
        cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        *out = b.release();
    });
}

BSNN_API bsnn_status bsnn_batch_destroy(bsnn_batch* b) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    delete b;
    return BSNN_OK;
}

BSNN_API const char* bsnn_batch_last_error(const bsnn_batch* b) { return b ? b->err.c_str() : g_thread_error.c_str(); }

BSNN_API bsnn_status bsnn_batch_add_class(bsnn_batch* b, uint32_t num_e, uint32_t num_i, const float* w_ee,
                                          const float* w_ei, const float* w_ie, const float* w_ii,
                                          const bsnn_connection_params* excitatory_pre,
                                          const bsnn_connection_params* inhibitory_pre, uint32_t* out_class) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        require(!b->finalized, BSNN_ERR_STATE, "classes cannot be added after the batch has started");
        require(b->classes.size() < kBatchMaxClasses, BSNN_ERR_INVALID_ARGUMENT, "too many size classes");
        require(num_e > 0 && num_i > 0, BSNN_ERR_INVALID_ARGUMENT, "a class needs excitatory and inhibitory neurons");
        require(w_ee && w_ei && w_ie && w_ii && excitatory_pre && inhibitory_pre, BSNN_ERR_INVALID_ARGUMENT, "null argument");
        bsnn_batch::HClass C;
        C.E = num_e;
        C.I = num_i;
        const uint32_t N = num_e + num_i, MT = (N + 127) / 128;
        const bsnn_connection_params* cp[2] = {excitatory_pre, inhibitory_pre};
        for (int sd = 0; sd < 2; ++sd) {
            const uint32_t K = sd == 0 ? num_e : num_i, KT = (K + 63) / 64;
            // W_side[pre][post] = [W_x->E | W_x->I]; A = W_side^T, tiled (mt, kt), core-matrix layout
            const float* wl = sd == 0 ? w_ee : w_ie;  // posts 0 .. E-1
            const float* wr = sd == 0 ? w_ei : w_ii;  // posts E .. N-1
            std::vector<uint16_t>& A = C.A[sd];
            A.assign(static_cast<size_t>(MT) * KT * 128u * 64u, 0);
            for (uint32_t pre = 0; pre < K; ++pre)
                for (uint32_t post = 0; post < N; ++post) {
                    const float w = post < num_e ? wl[static_cast<size_t>(pre) * num_e + post]
                                                 : wr[static_cast<size_t>(pre) * num_i + (post - num_e)];
                    require(!(w < 0.0f), BSNN_ERR_INVALID_ARGUMENT, "weights must be non-negative");
                    const size_t tile = static_cast<size_t>(post >> 7) * KT + (pre >> 6);
                    A[tile * 128u * 64u + core_offset(128u, post & 127u, pre & 63u)] = host_bf16(w);
                }
            C.r_decay[sd] = std::exp(-1.0f * cp[sd]->timestep / cp[sd]->rise_time);
            C.d_decay[sd] = std::exp(-1.0f * cp[sd]->timestep / cp[sd]->decay_time);
            C.norm[sd] = cp[sd]->postsynaptic_kernel_normalization_value;
        }
        b->classes.push_back(std::move(C));
        if (out_class) *out_class = static_cast<uint32_t>(b->classes.size() - 1);
    });
}

BSNN_API bsnn_status bsnn_batch_add_instance(bsnn_batch* b, uint32_t class_index, const bsnn_neuron_group_params* e_group,
                                             const bsnn_neuron_group_params* i_group, int32_t rng_seed,
                                             const uint32_t* stim_counts, uint32_t stim_steps, const uint32_t* stim_neurons,
                                             const float* stim_deltas, uint32_t num_events, uint32_t* out_instance) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        require(!b->finalized, BSNN_ERR_STATE, "instances cannot be added after the batch has started");
        require(class_index < b->classes.size(), BSNN_ERR_OUT_OF_RANGE, "class index out of range");
        require(e_group && i_group, BSNN_ERR_INVALID_ARGUMENT, "null group parameters");
        auto& HC = b->classes[class_index];
        require(e_group->num_neurons == HC.E && i_group->num_neurons == HC.I, BSNN_ERR_INVALID_ARGUMENT,
                "group sizes must match the class");
        require((stim_counts || stim_steps == 0) && ((stim_neurons && stim_deltas) || num_events == 0),
                BSNN_ERR_INVALID_ARGUMENT, "null stimulus arrays");
        bsnn_batch::HInst I;
        I.cls = class_index;
        I.g[0] = *e_group;
        I.g[1] = *i_group;
        I.seed = static_cast<uint32_t>(rng_seed);
        I.counts.assign(stim_counts, stim_counts + stim_steps);
        uint64_t total = 0;
        for (uint32_t c : I.counts) total += c;
        require(total == num_events, BSNN_ERR_INVALID_ARGUMENT, "stimulus counts must add up to num_events");
        I.neurons.assign(stim_neurons, stim_neurons + num_events);
        I.deltas.assign(stim_deltas, stim_deltas + num_events);
        for (uint32_t nrn : I.neurons) require(nrn < HC.E + HC.I, BSNN_ERR_OUT_OF_RANGE, "stimulus neuron out of range");
        b->insts.push_back(std::move(I));
        const uint32_t id = static_cast<uint32_t>(b->insts.size() - 1);
        HC.instances.push_back(id);
        if (out_instance) *out_instance = id;
    });
}

BSNN_API bsnn_status bsnn_batch_set_noise(bsnn_batch* b, int32_t on) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        require(!b->finalized, BSNN_ERR_STATE, "set the noise before the first step");
        b->noise_on = on != 0;
    });
}

BSNN_API bsnn_status bsnn_batch_set_form(bsnn_batch* b, int32_t form) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        require(form == BSNN_BATCH_FORM_FLOW || form == BSNN_BATCH_FORM_PHASED, BSNN_ERR_INVALID_ARGUMENT,
                "unknown batch form");
        require(b->steps_done == 0, BSNN_ERR_STATE, "the form is set before the first step");
        if (form != b->form) {
            batch_teardown(b);
            b->form = form;
        }
    });
}

BSNN_API bsnn_status bsnn_batch_set_steps_per_launch(bsnn_batch* b, uint32_t steps) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        require(steps > 0, BSNN_ERR_INVALID_ARGUMENT, "steps per launch must be > 0");
        b->steps_per_launch = steps;
    });
}

BSNN_API bsnn_status bsnn_batch_set_device_wait_limit(bsnn_batch* b, uint64_t nanoseconds) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        require(nanoseconds >= 1000ull && nanoseconds <= 60000000000ull, BSNN_ERR_INVALID_ARGUMENT,
                "device wait limit must be in [1 us, 60 s]");
        b->wait_limit_ns = nanoseconds;
        if (b->finalized) {
            b->h.wait_limit_ns = nanoseconds;
            cuda_check(cudaStreamSynchronize(b->stream), "stream synchronize");
            cuda_check(cudaMemcpy(b->d_sim, &b->h, sizeof(BSim), cudaMemcpyHostToDevice), "H2D batch sim");
        }
    });
}

BSNN_API bsnn_status bsnn_batch_run(bsnn_batch* b, uint32_t num_steps) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        batch_finalize(b);
        require(!b->failed, BSNN_ERR_STATE, "the batch failed earlier (device timeout)");
        uint32_t left = num_steps;
        while (left > 0) {
            const uint32_t n = std::min(left, b->steps_per_launch);
            batch_launch(b, n);
            left -= n;
        }
        b->steps_done += num_steps;
    });
}

BSNN_API bsnn_status bsnn_batch_synchronize(bsnn_batch* b) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        if (b->finalized) batch_check_error(b);
    });
}

BSNN_API bsnn_status bsnn_batch_get_stream(const bsnn_batch* b, void** out) {
    if (!b || !out) return BSNN_ERR_INVALID_ARGUMENT;
    *out = b->stream;
    return BSNN_OK;
}

// Fields as in bsnn_read_state: membrane potentials, g (with the pending propagation), I_stim,
// refractory counters, spikes, background conductances and traces, and the neuron's connection
// traces r, d and x = d - r.  `host_out` holds the instance's E + I neurons.
BSNN_API bsnn_status bsnn_batch_read_state(bsnn_batch* b, uint32_t instance, int32_t field, void* host_out) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        batch_finalize(b);
        batch_check_error(b);
        require(instance < b->insts.size(), BSNN_ERR_OUT_OF_RANGE, "instance index out of range");
        require(host_out != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null output");
        const auto& HC = b->classes[b->insts[instance].cls];
        const uint32_t n = HC.E + HC.I;
        const size_t off = b->nbase[instance];
        const BSim& h = b->h;
        auto copy = [&](const void* src) {
            cuda_check(cudaMemcpy(host_out, static_cast<const char*>(src) + 4 * off, 4ull * n, cudaMemcpyDeviceToHost), "D2H");
        };
        switch (field) {
            case BSNN_FIELD_MEMBRANE_POTENTIALS: copy(h.v); return;
            case BSNN_FIELD_I_STIMULUS: copy(h.istim); return;
            case BSNN_FIELD_REFRACTORY_COUNTER: copy(h.refrac); return;
            case BSNN_FIELD_SPIKES: copy(h.spikes); return;

            case BSNN_FIELD_BG_E_R_TRACES: copy(h.er); return;
            case BSNN_FIELD_BG_E_D_TRACES: copy(h.ed); return;
            case BSNN_FIELD_BG_I_R_TRACES: copy(h.ir); return;
            case BSNN_FIELD_BG_I_D_TRACES: copy(h.id); return;
            case BSNN_FIELD_CONN_R_TRACES: copy(h.tr); return;
            case BSNN_FIELD_CONN_D_TRACES: copy(h.td); return;
            case BSNN_FIELD_CONN_SUMMED: {
                std::vector<float> r(n), d(n);
                cuda_check(cudaMemcpy(r.data(), h.tr + off, 4ull * n, cudaMemcpyDeviceToHost), "D2H");
                cuda_check(cudaMemcpy(d.data(), h.td + off, 4ull * n, cudaMemcpyDeviceToHost), "D2H");
                float* o = static_cast<float*>(host_out);
                for (uint32_t k = 0; k < n; ++k) o[k] = d[k] - r[k];
                return;
            }
            case BSNN_FIELD_G_EXCITATORY:
            case BSNN_FIELD_G_INHIBITORY:
            case BSNN_FIELD_BG_G_EXCITATORY:
            case BSNN_FIELD_BG_G_INHIBITORY: {
                const bool with_pending = field == BSNN_FIELD_G_EXCITATORY || field == BSNN_FIELD_G_INHIBITORY;
                const bool exc = field == BSNN_FIELD_G_EXCITATORY || field == BSNN_FIELD_BG_G_EXCITATORY;
                bsnn_batch_g_kernel<<<(n + 255) / 256, 256, 0, b->stream>>>(b->d_sim, b->pos[instance], with_pending ? 1 : 0,
                                                                            b->scratch, b->scratch + n);
                cuda_check(cudaGetLastError(), "batch g read");
                cuda_check(cudaMemcpyAsync(host_out, b->scratch + (exc ? 0 : n), 4ull * n, cudaMemcpyDeviceToHost,
                                           b->stream),
                           "D2H g");
                cuda_check(cudaStreamSynchronize(b->stream), "sync");
                return;
            }
            default: throw ApiError(BSNN_ERR_INVALID_ARGUMENT, "unknown field " + std::to_string(field));
        }
    });
}

// Spike counts since creation, [instance][0 = E, 1 = I].
BSNN_API bsnn_status bsnn_batch_read_spike_counts(bsnn_batch* b, uint64_t* host_out) {
    if (!b || !host_out) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        batch_finalize(b);
        batch_check_error(b);
        cuda_check(cudaMemcpy(host_out, b->h.spike_counts, sizeof(uint64_t) * 2 * b->insts.size(), cudaMemcpyDeviceToHost),
                   "D2H spike counts");
    });
}

// Times candidate GEMM unit sizes (K tiles per unit, around the default rule) with the placement's
// ring depth, then ring depths of 2 to 8 stages for the best unit size, each over
// `trial_steps` clock steps after a warm-up, and keeps the fastest.  Only before the first step:
// the batch is left at step 0 with the chosen shapes.  The unit size sets how many K chunks a
// neuron's partial sums add up, so it is part of the batch's arithmetic (results stay
// deterministic for a given choice); the ring depth is not.
BSNN_API bsnn_status bsnn_batch_autotune(bsnn_batch* b, uint32_t trial_steps, bsnn_batch_tuning* out) {
    if (!b) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        require(b->steps_done == 0, BSNN_ERR_STATE, "autotune runs before the first step");
        require(trial_steps > 0, BSNN_ERR_INVALID_ARGUMENT, "trial_steps must be > 0");
        batch_teardown(b);
        b->tune_kc = 0;
        b->tune_stages = 0;
        batch_finalize(b);
        const uint32_t kc0 = b->kc;
        uint32_t kt_max = 1;
        for (uint32_t c = 0; c < b->h.n_classes; ++c) kt_max = std::max(kt_max, std::max(b->h.cls[c].KT[0], b->h.cls[c].KT[1]));
        cudaEvent_t e0, e1;
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        uint32_t tried = 0;
        // one trial: a fresh device side with (kc, stages), a warm-up launch, then a timed one
        auto trial = [&](uint32_t kc, uint32_t stages) -> double {
            batch_teardown(b);
            b->tune_kc = kc;
            b->tune_stages = stages;
            try {
                batch_finalize(b);
            } catch (const ApiError&) {
                return -1.0;  // this ring depth does not fit
            }
            const uint32_t warm = std::max<uint32_t>(8u, trial_steps / 4u);
            batch_launch(b, warm);
            cuda_check(cudaEventRecord(e0, b->stream), "event record");
            batch_launch(b, trial_steps);
            cuda_check(cudaEventRecord(e1, b->stream), "event record");
            cuda_check(cudaEventSynchronize(e1), "event sync");
            batch_check_error(b);
            float ms = 0.0f;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
            ++tried;
            return 1e3 * ms / trial_steps;
        };
        std::vector<uint32_t> kcs = {kc0, std::max(1u, kc0 / 2), std::max(1u, (kc0 * 3) / 4), (kc0 * 3) / 2, kc0 * 2, kt_max};
        std::sort(kcs.begin(), kcs.end());
        kcs.erase(std::unique(kcs.begin(), kcs.end()), kcs.end());
        const double t_default = trial(kc0, 0);
        double best = t_default;
        uint32_t best_kc = kc0, best_st = 0;
        for (uint32_t kc : kcs) {
            if (kc == kc0 || kc > kt_max) continue;
            const double us = trial(kc, 0);
            if (us > 0.0 && us < best) {
                best = us;
                best_kc = kc;
            }
        }
        for (uint32_t st = 2; st <= kBatchStages; ++st) {
            const double us = trial(best_kc, st);
            if (us > 0.0 && us < best) {
                best = us;
                best_st = st;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        batch_teardown(b);
        b->tune_kc = best_kc;
        b->tune_stages = best_st;
        batch_finalize(b);
        if (out) {
            bsnn_batch_tuning r{};
            r.k_tiles_per_unit = best_kc;
            r.operand_stages = b->h.n_stages;
            r.candidates = tried;
            r.us_per_step = static_cast<float>(best);
            r.default_us_per_step = static_cast<float>(t_default);
            *out = r;
        }
    });
}

// Applies shapes found by an earlier autotune (k_tiles_per_unit and operand_stages; 0 keeps the
// default rule), before the first step.
BSNN_API bsnn_status bsnn_batch_set_tuning(bsnn_batch* b, const bsnn_batch_tuning* t) {
    if (!b || !t) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        require(b->steps_done == 0, BSNN_ERR_STATE, "shapes are set before the first step");
        require(t->operand_stages == 0 || (t->operand_stages >= 2 && t->operand_stages <= kBatchStages),
                BSNN_ERR_INVALID_ARGUMENT, "operand_stages must be 0 or 2..8");
        batch_teardown(b);
        b->tune_kc = t->k_tiles_per_unit;
        b->tune_stages = t->operand_stages;
    });
}

BSNN_API bsnn_status bsnn_batch_get_info(bsnn_batch* b, bsnn_batch_info* out) {
    if (!b || !out) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        batch_finalize(b);
        bsnn_batch_info i{};
        i.num_classes = b->h.n_classes;
        i.num_instances = b->h.n_inst;
        i.num_neurons = b->h.n_neurons;
        i.num_units = b->h.n_units;
        i.grid_ctas = b->grid;
        i.block_threads = kBatchThreads;
        i.steps_done = b->steps_done;
        i.device_bytes = b->arena_bytes;
        uint64_t wb = 0;
        for (const auto& C : b->classes) wb += 2ull * (C.A[0].size() + C.A[1].size());
        i.weight_bytes = wb;
        i.kernel_launches = b->launches;
        i.smem_bytes = b->smem;
        i.state_in_smem = b->h.state_in_smem;
        i.operand_stages = b->h.n_stages;
        i.form = b->form;
        *out = i;
    });
}

#ifdef BSNN_PHASE_TIMING
// Profiling builds: per-CTA clock tallies of the batch kernel's phases [grid][8].
BSNN_API bsnn_status bsnn_batch_debug_phase_ns(bsnn_batch* b, unsigned long long* out) {
    if (!b || !out) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_batch(b, [&] {
        batch_finalize(b);
        cuda_check(cudaMemcpy(out, b->h.phase_ns, 8 * sizeof(unsigned long long) * b->grid, cudaMemcpyDeviceToHost), "D2H");
    });
}
#endif

}  // extern "C"
