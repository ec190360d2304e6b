// adjoint_api.cuh -- host side of the differentiation form (bsnn_adjoint_* in include/bsnn.h);
// included at the end of bsnn_api.cu.
//
// bsnn_adjoint_forward runs the network for num_steps, checkpointing the state every
// checkpoint_interval steps, and evaluates
//     L = rate_weight / T * sum_t (rho_t - rho*_t)^2 + voltage_weight / T * sum_t (vbar_{t+1} - v*_t)^2
// with rho_t = a rho_{t-1} + (1 - a) n_E(t) / (N_E dt), a = exp(-dt / rate_tau) (the smoothed
// excitatory population rate) and vbar the mean excitatory membrane potential after the step.
// bsnn_adjoint_backward replays each segment from its checkpoint and propagates the adjoints back
// (adjoint_kernel.cuh), returning dL/dW_EE and dL/dg_leak (one g_leak shared by both groups).  The
// forward pass runs its last segment the way the backward pass replays it (from the restored
// checkpoint, keeping the tape), so the backward pass starts on that tape without a replay; with
// one segment (checkpoint interval >= num_steps) nothing is recomputed.
#pragma once

#include "adjoint_kernel.cuh"

struct bsnn_adjoint {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    bsnn_adjoint_desc d{};
    ADev h{};
    unsigned char* arena = nullptr;
    // device buffers
    float *WE = nullptr, *WI = nullptr, *part = nullptr, *x_cur = nullptr;
    float *tv = nullptr, *tu = nullptr, *tge = nullptr, *tgi = nullptr, *tx = nullptr, *lge_all = nullptr;
    uint8_t *ts = nullptr, *tref = nullptr;
    float *lam_v = nullptr, *lam_d = nullptr, *lam_r = nullptr, *lam_x = nullptr;
    float* lam_gi = nullptr;      // [2][ld] lambda_gi by step parity
    // the persistent backward kernel: CTAs, neurons per CTA at most, shared memory, grid barrier
    uint32_t bwd_grid = 0, bwd_max_own = 0, bwd_res = 0;  // CTAs, own neurons at most, rows of W in smem
    size_t bwd_smem = 0;
    unsigned long long* barrier = nullptr;
    int32_t* error = nullptr;
    float *c_s = nullptr, *c_v = nullptr;  // [T] loss sensitivities, uploaded before the backward pass
    float* dW = nullptr;
    double* gl_acc = nullptr;     // [bwd_grid] per-CTA g_leak shares
    double* vsum = nullptr;       // [T][nb] per-block sums of the E voltages after each step
    uint32_t* counts = nullptr;   // [T] E spikes per step
    std::vector<uint32_t> stim_off;  // [stimulus steps + 1] host copy of the stimulus offsets
    float* ckpt = nullptr;        // [n_ckpt][kAdjCkptArrays][N]
    uint32_t n_ckpt = 0, nb = 0;
    uint32_t ld = 0;              // row length of W_E, W_I and the lambda_g rows: N rounded up to 4
    // one captured graph per checkpoint segment for each pass (captured on first use, dropped when
    // g_leak changes, since the group parameters are kernel arguments)
    std::vector<cudaGraphExec_t> fwd_graphs, bwd_graphs;
    cudaGraphExec_t replay_graph = nullptr;    // the last segment's replay, when its tape is stale
    bool tape_last = false;                    // the tape holds the last segment of the last forward pass
    std::vector<size_t> fwd_nodes, bwd_nodes;  // kernels per graph
    size_t replay_nodes = 0;
    uint64_t launches = 0;                     // kernels run (graph nodes included)
    // forward results
    std::vector<double> rho, vbar;
    std::vector<float> rate_target, v_target;
    bool have_forward = false;
    void drop_graphs() {
        fwd_nodes.clear();
        bwd_nodes.clear();
        for (auto g : fwd_graphs)
            if (g) cudaGraphExecDestroy(g);
        for (auto g : bwd_graphs)
            if (g) cudaGraphExecDestroy(g);
        if (replay_graph) cudaGraphExecDestroy(replay_graph);
        replay_graph = nullptr;
        fwd_graphs.clear();
        bwd_graphs.clear();
    }
    ~bsnn_adjoint() {
        drop_graphs();
        if (arena) cudaFree(arena);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

template <class F>
bsnn_status guarded_adj(bsnn_adjoint* a, F&& f) {
    try {
        if (a) cuda_check(cudaSetDevice(a->device), "cudaSetDevice");
        f();
        return BSNN_OK;
    } catch (const ApiError& e) {
        if (a) a->err = e.what();
        g_thread_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        if (a) a->err = e.what();
        g_thread_error = e.what();
        return BSNN_ERR_RUNTIME;
    }
}

AdjGroupP adj_group(const bsnn_neuron_group_params& p) {
    AdjGroupP G{};
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
    return G;
}

// One forward step t: the neuron update (tape rows where the pointers are set; the step's E spike
// count and voltage sums in the forward pass), then the propagation of x_{t+1}.
// Both kernels are launched with programmatic dependent launch: each may launch while its
// predecessor finishes, and waits for it (pdl_enter) before reading anything, which hides the
// launch gap between the two kernels of a step and between steps.
void adj_step(bsnn_adjoint* a, uint32_t t, size_t tape_row, bool tape, float* x_next, bool forward) {
    const uint32_t N = a->h.N;
    const dim3 pg((N + kAdjBlock - 1) / kAdjBlock, 2 * kAdjChunks);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.blockDim = dim3(kAdjBlock);
    cfg.stream = a->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(a->nb);
    const bool stim = t < a->stim_off.size() - 1;
    const uint32_t ev_lo = stim ? a->stim_off[t] : 0u, ev_hi = stim ? a->stim_off[t + 1] : 0u;
    cuda_check(cudaLaunchKernelEx(&cfg, bsnn_adj_neuron_fwd, a->h, t, ev_lo, ev_hi, static_cast<const float*>(a->part),
                                  tape ? a->tv + tape_row : nullptr, tape ? a->tu + tape_row : nullptr,
                                  tape ? a->tge + tape_row : nullptr, tape ? a->tgi + tape_row : nullptr,
                                  tape ? a->ts + tape_row : nullptr, tape ? a->tref + tape_row : nullptr, x_next,
                                  forward ? a->counts + t : nullptr,
                                  forward ? a->vsum + static_cast<size_t>(t) * a->nb : nullptr),
               "adjoint neuron launch");
    cfg.gridDim = pg;
    cuda_check(cudaLaunchKernelEx(&cfg, bsnn_adj_propagate, static_cast<const float*>(a->WE),
                                  static_cast<const float*>(a->WI), a->h.E, a->h.I, N, a->ld,
                                  static_cast<const float*>(x_next), a->part),
               "adjoint propagate launch");
}

// The last segment's steps from its restored checkpoint, keeping the tape (x_t in tape row k of
// tx, x_{t+1} in row k + 1); `forward` adds the forward pass's per-step outputs.  Restoring the
// checkpoint just saved changes no bit: the saved g is g_base plus the chunk sums, restored as
// g_base with zero chunks.
void adj_tape_segment(bsnn_adjoint* a, uint32_t c, bool forward) {
    const uint32_t T = a->d.num_steps, C = a->d.checkpoint_interval, N = a->h.N;
    const uint32_t t0 = c * C, t1 = std::min(T, t0 + C);
    const float* slot = a->ckpt + static_cast<size_t>(c) * kAdjCkptArrays * N;
    bsnn_adj_restore<<<a->nb, kAdjBlock, 0, a->stream>>>(a->h, a->part, a->tx, slot);
    for (uint32_t k = 0; k < t1 - t0; ++k) {
        const size_t o = static_cast<size_t>(k) * N;
        adj_step(a, t0 + k, o, true, a->tx + o + N, forward);
    }
}

// Forward segment c: save the checkpoint, then run its steps (the last one keeping the tape).
void adj_forward_segment(bsnn_adjoint* a, uint32_t c) {
    const uint32_t T = a->d.num_steps, C = a->d.checkpoint_interval;
    const uint32_t t0 = c * C, t1 = std::min(T, t0 + C);
    float* slot = a->ckpt + static_cast<size_t>(c) * kAdjCkptArrays * a->h.N;
    bsnn_adj_save<<<a->nb, kAdjBlock, 0, a->stream>>>(a->h, a->part, a->x_cur, slot);
    if (c + 1 == a->n_ckpt) {
        adj_tape_segment(a, c, true);
        return;
    }
    for (uint32_t t = t0; t < t1; ++t) adj_step(a, t, 0, false, a->x_cur, true);
}

// Backward segment c: restore its checkpoint and replay its steps keeping the tape (the last
// segment's tape is the forward pass's), then walk them backwards in one persistent launch
// (bsnn_adj_backward_kernel: neuron adjoints, pull-back of the g adjoints through the weights),
// then add the segment's x_t lambda_ge(t)^T to dW_EE.
void adj_backward_segment(bsnn_adjoint* a, uint32_t c) {
    const uint32_t T = a->d.num_steps, C = a->d.checkpoint_interval, N = a->h.N, E = a->h.E;
    const uint32_t t0 = c * C, t1 = std::min(T, t0 + C), steps = t1 - t0;
    if (c + 1 != a->n_ckpt) adj_tape_segment(a, c, false);
    AdjBwd B{};
    B.tv = a->tv;
    B.tu = a->tu;
    B.tge = a->tge;
    B.tgi = a->tgi;
    B.ts = a->ts;
    B.tref = a->tref;
    B.lam_v = a->lam_v;
    B.lam_d = a->lam_d;
    B.lam_r = a->lam_r;
    B.lam_x = a->lam_x;
    B.c_s = a->c_s;
    B.c_v = a->c_v;
    B.lge_all = a->lge_all;
    B.lgi2 = a->lam_gi;
    B.gl_acc = a->gl_acc;
    B.barrier = a->barrier;
    B.error = a->error;
    B.wait_limit_ns = kDefaultWaitLimitNs;
    B.t0 = t0;
    B.steps = steps;
    B.ld = a->ld;
    B.max_own = a->bwd_max_own;
    B.n_res = a->bwd_res;
    B.beta = a->d.surrogate_beta;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(a->bwd_grid);
    cfg.blockDim = dim3(kAdjBwdThreads);
    cfg.dynamicSmemBytes = a->bwd_smem;
    cfg.stream = a->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cuda_check(cudaLaunchKernelEx(&cfg, bsnn_adj_backward_kernel, a->h, B), "adjoint backward launch");
    const dim3 og((E + kOuterTile - 1) / kOuterTile, (E + kOuterTile - 1) / kOuterTile);
    bsnn_adj_outer<<<og, 256, 0, a->stream>>>(a->tx, N, a->lge_all, a->ld, steps, E, a->dW);
}

// Captures fn(c) for every segment c into one graph each (once), then launches them in `order`.
template <class F>
void adj_run_graphs(bsnn_adjoint* a, std::vector<cudaGraphExec_t>& graphs, std::vector<size_t>& nodes, bool reverse,
                    F&& fn, const char* what) {
    if (graphs.empty()) {
        graphs.assign(a->n_ckpt, nullptr);
        nodes.assign(a->n_ckpt, 0);
        for (uint32_t c = 0; c < a->n_ckpt; ++c) {
            cudaGraph_t g = nullptr;
            cuda_check(cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal), what);
            fn(c);
            const cudaError_t launch_err = cudaGetLastError();
            cuda_check(cudaStreamEndCapture(a->stream, &g), what);
            cuda_check(launch_err, what);
            cudaGraphGetNodes(g, nullptr, &nodes[c]);
            const cudaError_t ie = cudaGraphInstantiate(&graphs[c], g, 0);
            cudaGraphDestroy(g);
            cuda_check(ie, what);
        }
    }
    for (uint32_t k = 0; k < a->n_ckpt; ++k) {
        const uint32_t c = reverse ? a->n_ckpt - 1 - k : k;
        cuda_check(cudaGraphLaunch(graphs[c], a->stream), what);
        a->launches += nodes[c];
    }
}

}  // namespace

extern "C" {

BSNN_API bsnn_status bsnn_adjoint_create(const bsnn_adjoint_desc* desc, const bsnn_neuron_group_params* e_group,
                                         const bsnn_neuron_group_params* i_group,
                                         const bsnn_connection_params* excitatory_pre,
                                         const bsnn_connection_params* inhibitory_pre, const float* w_ee,
                                         const float* w_ei, const float* w_ie, const float* w_ii,
                                         const uint32_t* stimulus_counts, uint32_t stimulus_steps,
                                         const uint32_t* stimulus_neurons, const float* stimulus_deltas,
                                         uint32_t num_events, int32_t device, bsnn_adjoint** out) {
    if (!out) return BSNN_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    return guarded_adj(nullptr, [&] {
        require(desc && e_group && i_group && excitatory_pre && inhibitory_pre && w_ee && w_ei && w_ie && w_ii,
                BSNN_ERR_INVALID_ARGUMENT, "null argument");
        require(desc->num_excitatory > 0 && desc->num_inhibitory > 0 && desc->num_steps > 0 &&
                    desc->checkpoint_interval > 0,
                BSNN_ERR_INVALID_ARGUMENT, "sizes must be > 0");
        require((stimulus_counts || stimulus_steps == 0) && ((stimulus_neurons && stimulus_deltas) || num_events == 0),
                BSNN_ERR_INVALID_ARGUMENT, "null stimulus arrays");
        int nd = 0;
        cuda_check(cudaGetDeviceCount(&nd), "cudaGetDeviceCount");
        require(device >= 0 && device < nd, BSNN_ERR_INVALID_ARGUMENT, "device ordinal out of range");
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        auto a = std::make_unique<bsnn_adjoint>();
        a->device = device;
        a->d = *desc;
        cuda_check(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        const uint32_t E = desc->num_excitatory, I = desc->num_inhibitory, N = E + I, T = desc->num_steps;
        const uint32_t C = desc->checkpoint_interval;
        ADev& h = a->h;
        h.E = E;
        h.I = I;
        h.N = N;
        h.seed = static_cast<uint32_t>(desc->rng_seed);
        h.noise_on = desc->noise_on ? 1u : 0u;
        h.g[0] = adj_group(*e_group);
        h.g[1] = adj_group(*i_group);
        const bsnn_connection_params* cp[2] = {excitatory_pre, inhibitory_pre};
        for (int sd = 0; sd < 2; ++sd) {
            h.r_decay[sd] = std::exp(-1.0f * cp[sd]->timestep / cp[sd]->rise_time);
            h.d_decay[sd] = std::exp(-1.0f * cp[sd]->timestep / cp[sd]->decay_time);
            h.norm[sd] = cp[sd]->postsynaptic_kernel_normalization_value;
        }
        a->n_ckpt = (T + C - 1) / C;
        a->nb = (N + kAdjBlock - 1) / kAdjBlock;
        a->ld = (N + 3u) & ~3u;
        const uint32_t ld = a->ld;
        // stimulus CSR
        std::vector<std::vector<std::pair<uint32_t, float>>> per(stimulus_steps);
        size_t e = 0;
        for (uint32_t t = 0; t < stimulus_steps; ++t)
            for (uint32_t k = 0; k < stimulus_counts[t]; ++k, ++e) {
                require(e < num_events, BSNN_ERR_INVALID_ARGUMENT, "stimulus counts exceed num_events");
                require(stimulus_neurons[e] < N, BSNN_ERR_OUT_OF_RANGE, "stimulus neuron out of range");
                per[t].emplace_back(stimulus_neurons[e], stimulus_deltas[e]);
            }
        require(e == num_events, BSNN_ERR_INVALID_ARGUMENT, "stimulus counts must add up to num_events");
        std::vector<uint32_t> soff(stimulus_steps + 1, 0), evn;
        std::vector<float> evd;
        for (uint32_t t = 0; t < stimulus_steps; ++t) {
            std::stable_sort(per[t].begin(), per[t].end(), [](const auto& x, const auto& y) { return x.first < y.first; });
            for (const auto& ev : per[t]) {
                evn.push_back(ev.first);
                evd.push_back(ev.second);
            }
            soff[t + 1] = static_cast<uint32_t>(evn.size());
        }
        Arena A;
        const size_t fN = 4ull * N;
        size_t o_state[11];
        for (auto& o : o_state) o = A.take(fN);
        const size_t o_cs = A.take(4ull * T), o_cv = A.take(4ull * T);
        const size_t o_we = A.take(4ull * E * ld), o_wi = A.take(4ull * I * ld);
        const size_t o_part = A.take(4ull * 2 * kAdjChunks * N), o_x = A.take(fN);
        const size_t Ct = std::min(C, T);  // tape rows: one segment's steps
        const size_t o_tv = A.take(fN * Ct), o_tu = A.take(fN * Ct), o_tge = A.take(fN * Ct), o_tgi = A.take(fN * Ct);
        const size_t o_tx = A.take(fN * (Ct + 1)), o_lge = A.take(4ull * ld * Ct);
        const size_t o_ts = A.take(static_cast<size_t>(N) * Ct), o_tref = A.take(static_cast<size_t>(N) * Ct);
        const size_t o_lv = A.take(fN), o_ld = A.take(fN), o_lr = A.take(fN), o_lx = A.take(fN),
                     o_lgi = A.take(4ull * 2 * ld);
        const size_t o_dw = A.take(4ull * E * E);
        // the persistent backward kernel: one CTA per SM, at least 8 neurons each
        int sms = 0, optin = 0;
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
        cuda_check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device), "smem attr");
        a->bwd_grid = std::max<uint32_t>(1u, std::min<uint32_t>(static_cast<uint32_t>(sms), (N + 7u) / 8u));
        a->bwd_max_own = (N + a->bwd_grid - 1) / a->bwd_grid;
        require(a->bwd_max_own <= kAdjBwdThreads, BSNN_ERR_INVALID_ARGUMENT,
                "network too large for the adjoint's backward kernel (one thread per neuron of a CTA)");
        // lambda_g vectors, own state and row pieces, then as many own rows of W as fit
        const size_t fixed = sizeof(float) * (2ull * ld + ((4ull * a->bwd_max_own + kPbChunks * a->bwd_max_own + 3u) & ~3ull));
        require(fixed + 2048 <= static_cast<size_t>(optin), BSNN_ERR_INVALID_ARGUMENT,
                "network too large for the adjoint's shared-memory lambda_g vectors");
        const size_t room = static_cast<size_t>(optin) - 2048 - fixed;
        a->bwd_res = static_cast<uint32_t>(std::min<size_t>(a->bwd_max_own, room / (sizeof(float) * ld)));
        a->bwd_smem = fixed + sizeof(float) * ld * a->bwd_res;
        cuda_check(cudaFuncSetAttribute(bsnn_adj_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(a->bwd_smem)),
                   "adjoint backward smem");
        int per_sm = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bsnn_adj_backward_kernel, kAdjBwdThreads,
                                                                 a->bwd_smem),
                   "adjoint backward occupancy");
        require(per_sm >= 1, BSNN_ERR_RUNTIME, "adjoint backward kernel does not fit on an SM");
        const size_t o_gl = A.take(8ull * a->bwd_grid);
        const size_t o_bar = A.take(sizeof(unsigned long long)), o_err = A.take(sizeof(int32_t));
        const size_t o_vs = A.take(8ull * a->nb * T);
        const size_t o_cnt = A.take(4ull * T);
        const size_t o_ck = A.take(fN * kAdjCkptArrays * a->n_ckpt);
        const size_t o_soff = A.take(4ull * soff.size()), o_evn = A.take(4ull * std::max<size_t>(evn.size(), 1)),
                     o_evd = A.take(4ull * std::max<size_t>(evd.size(), 1));
        cuda_check(cudaMalloc(&a->arena, A.size), "cudaMalloc adjoint arena");
        unsigned char* base = a->arena;
        cuda_check(cudaMemset(base, 0, A.size), "cudaMemset adjoint arena");
        auto F = [&](size_t o) { return reinterpret_cast<float*>(base + o); };
        float** state[10] = {&h.v, &h.ge, &h.gi, &h.istim, &h.er, &h.ed, &h.ir, &h.id, &h.tr, &h.td};
        for (int k = 0; k < 10; ++k) *state[k] = F(o_state[k]);
        h.refrac = reinterpret_cast<uint32_t*>(base + o_state[10]);
        a->c_s = F(o_cs);
        a->c_v = F(o_cv);
        a->WE = F(o_we);
        a->WI = F(o_wi);
        h.WE = a->WE;
        h.WI = a->WI;
        a->part = F(o_part);
        a->x_cur = F(o_x);
        a->tv = F(o_tv);
        a->tu = F(o_tu);
        a->tge = F(o_tge);
        a->tgi = F(o_tgi);
        a->tx = F(o_tx);
        a->lge_all = F(o_lge);
        a->ts = base + o_ts;
        a->tref = base + o_tref;
        a->lam_v = F(o_lv);
        a->lam_d = F(o_ld);
        a->lam_r = F(o_lr);
        a->lam_x = F(o_lx);
        a->lam_gi = F(o_lgi);
        a->dW = F(o_dw);
        a->gl_acc = reinterpret_cast<double*>(base + o_gl);
        a->barrier = reinterpret_cast<unsigned long long*>(base + o_bar);
        a->error = reinterpret_cast<int32_t*>(base + o_err);
        a->vsum = reinterpret_cast<double*>(base + o_vs);
        a->counts = reinterpret_cast<uint32_t*>(base + o_cnt);
        a->ckpt = F(o_ck);
        h.stim_len = stimulus_steps;
        h.stim_off = reinterpret_cast<const uint32_t*>(base + o_soff);
        h.ev_neuron = reinterpret_cast<const uint32_t*>(base + o_evn);
        h.ev_delta = F(o_evd);
        cuda_check(cudaMemcpy(base + o_soff, soff.data(), 4ull * soff.size(), cudaMemcpyHostToDevice), "H2D");
        a->stim_off = soff;
        if (!evn.empty()) {
            cuda_check(cudaMemcpy(base + o_evn, evn.data(), 4ull * evn.size(), cudaMemcpyHostToDevice), "H2D");
            cuda_check(cudaMemcpy(base + o_evd, evd.data(), 4ull * evd.size(), cudaMemcpyHostToDevice), "H2D");
        }
        // W_E = [W_EE | W_EI], W_I = [W_IE | W_II], row-major [pre][ld], zero beyond N
        std::vector<float> row(ld, 0.0f);
        for (uint32_t i = 0; i < E; ++i) {
            std::memcpy(row.data(), w_ee + static_cast<size_t>(i) * E, 4ull * E);
            std::memcpy(row.data() + E, w_ei + static_cast<size_t>(i) * I, 4ull * I);
            cuda_check(cudaMemcpy(a->WE + static_cast<size_t>(i) * ld, row.data(), 4ull * ld, cudaMemcpyHostToDevice),
                       "H2D W");
        }
        for (uint32_t i = 0; i < I; ++i) {
            std::memcpy(row.data(), w_ie + static_cast<size_t>(i) * E, 4ull * E);
            std::memcpy(row.data() + E, w_ii + static_cast<size_t>(i) * I, 4ull * I);
            cuda_check(cudaMemcpy(a->WI + static_cast<size_t>(i) * ld, row.data(), 4ull * ld, cudaMemcpyHostToDevice),
                       "H2D W");
        }
        *out = a.release();
    });
}

BSNN_API bsnn_status bsnn_adjoint_destroy(bsnn_adjoint* a) {
    if (!a) return BSNN_ERR_INVALID_ARGUMENT;
    cudaSetDevice(a->device);
    if (a->stream) cudaStreamSynchronize(a->stream);
    delete a;
    return BSNN_OK;
}

BSNN_API const char* bsnn_adjoint_last_error(const bsnn_adjoint* a) { return a ? a->err.c_str() : g_thread_error.c_str(); }

BSNN_API bsnn_status bsnn_adjoint_get_stream(bsnn_adjoint* a, void** out_stream) {
    if (!a || !out_stream) return BSNN_ERR_INVALID_ARGUMENT;
    *out_stream = a->stream;
    return BSNN_OK;
}

BSNN_API bsnn_status bsnn_adjoint_kernel_launches(bsnn_adjoint* a, uint64_t* out) {
    if (!a || !out) return BSNN_ERR_INVALID_ARGUMENT;
    *out = a->launches;
    return BSNN_OK;
}

// New parameter values: the E->E weights (row-major [E][E]; null keeps them) and g_leak of both
// groups (a NaN keeps it).
BSNN_API bsnn_status bsnn_adjoint_set_params(bsnn_adjoint* a, const float* w_ee, float g_leak) {
    if (!a) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_adj(a, [&] {
        const uint32_t E = a->h.E;
        if (w_ee) {
            cuda_check(cudaStreamSynchronize(a->stream), "adjoint sync");
            cuda_check(cudaMemcpy2D(a->WE, 4ull * a->ld, w_ee, 4ull * E, 4ull * E, E, cudaMemcpyHostToDevice),
                       "H2D W_EE");
        }
        if (!std::isnan(g_leak) && (g_leak != a->h.g[0].g_leak || g_leak != a->h.g[1].g_leak)) {
            cuda_check(cudaStreamSynchronize(a->stream), "adjoint sync");
            a->h.g[0].g_leak = g_leak;
            a->h.g[1].g_leak = g_leak;
            a->drop_graphs();
        }
        a->have_forward = false;
    });
}

// Runs the forward pass; rate_target and voltage_target hold num_steps values (voltage_target may
// be null when voltage_weight is 0).  Optional outputs: the loss, rho_t and vbar_{t+1}.
BSNN_API bsnn_status bsnn_adjoint_forward(bsnn_adjoint* a, const float* rate_target, const float* voltage_target,
                                          float* loss_out, float* rate_out, float* mean_voltage_out) {
    if (!a) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_adj(a, [&] {
        const uint32_t T = a->d.num_steps, E = a->h.E;
        require(rate_target != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null rate target");
        require(voltage_target != nullptr || !(a->d.voltage_weight != 0.0f), BSNN_ERR_INVALID_ARGUMENT,
                "null voltage target with a voltage weight");
        bsnn_adj_restore<<<a->nb, kAdjBlock, 0, a->stream>>>(a->h, a->part, a->x_cur, nullptr);
        cuda_check(cudaMemsetAsync(a->counts, 0, 4ull * T, a->stream), "memset counts");
        a->launches += 1;
        adj_run_graphs(a, a->fwd_graphs, a->fwd_nodes, false, [&](uint32_t c) { adj_forward_segment(a, c); },
                       "adjoint forward");
        a->tape_last = true;
        std::vector<uint32_t> cnt(T);
        std::vector<double> vs(static_cast<size_t>(T) * a->nb);
        cuda_check(cudaMemcpyAsync(cnt.data(), a->counts, 4ull * T, cudaMemcpyDeviceToHost, a->stream), "D2H counts");
        cuda_check(cudaMemcpyAsync(vs.data(), a->vsum, 8ull * vs.size(), cudaMemcpyDeviceToHost, a->stream), "D2H vsum");
        cuda_check(cudaStreamSynchronize(a->stream), "adjoint forward");
        const double dt = a->h.g[0].timestep, ka = std::exp(-dt / static_cast<double>(a->d.rate_tau));
        a->rho.assign(T, 0.0);
        a->vbar.assign(T, 0.0);
        a->rate_target.assign(rate_target, rate_target + T);
        a->v_target.assign(T, 0.0f);
        if (voltage_target) a->v_target.assign(voltage_target, voltage_target + T);
        double rho = 0.0, loss = 0.0;
        for (uint32_t t = 0; t < T; ++t) {
            rho = ka * rho + (1.0 - ka) * static_cast<double>(cnt[t]) / (static_cast<double>(E) * dt);
            a->rho[t] = rho;
            double s = 0.0;
            for (uint32_t b = 0; b < a->nb; ++b) s += vs[static_cast<size_t>(t) * a->nb + b];
            a->vbar[t] = s / E;
            const double er = rho - rate_target[t], ev = a->vbar[t] - a->v_target[t];
            loss += a->d.rate_weight * er * er + a->d.voltage_weight * ev * ev;
            if (rate_out) rate_out[t] = static_cast<float>(rho);
            if (mean_voltage_out) mean_voltage_out[t] = static_cast<float>(a->vbar[t]);
        }
        if (loss_out) *loss_out = static_cast<float>(loss / T);
        a->have_forward = true;
    });
}

// The gradients of the last forward pass's loss: dL/dW_EE (row-major [E][E]) and dL/dg_leak.
BSNN_API bsnn_status bsnn_adjoint_backward(bsnn_adjoint* a, float* grad_w_ee, double* grad_g_leak) {
    if (!a) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_adj(a, [&] {
        require(a->have_forward, BSNN_ERR_STATE, "run bsnn_adjoint_forward first");
        const uint32_t T = a->d.num_steps, N = a->h.N, E = a->h.E;
        const size_t fN = 4ull * N;
        const double dt = a->h.g[0].timestep, ka = std::exp(-dt / static_cast<double>(a->d.rate_tau));
        // the loss's sensitivities to the step's E spikes (through rho) and to vbar_{t+1}
        std::vector<float> c_s(T), c_v(T);
        double lrho = 0.0;
        for (uint32_t t = T; t-- > 0;) {
            lrho = ka * lrho + a->d.rate_weight * 2.0 / T * (a->rho[t] - a->rate_target[t]);
            c_s[t] = static_cast<float>(lrho * (1.0 - ka) / (static_cast<double>(E) * dt));
            c_v[t] = static_cast<float>(a->d.voltage_weight * 2.0 / T * (a->vbar[t] - a->v_target[t]) / E);
        }
        cuda_check(cudaMemcpyAsync(a->c_s, c_s.data(), 4ull * T, cudaMemcpyHostToDevice, a->stream), "H2D c_s");
        cuda_check(cudaMemcpyAsync(a->c_v, c_v.data(), 4ull * T, cudaMemcpyHostToDevice, a->stream), "H2D c_v");
        for (float* p : {a->lam_v, a->lam_d, a->lam_r, a->lam_x})
            cuda_check(cudaMemsetAsync(p, 0, fN, a->stream), "memset adjoints");
        cuda_check(cudaMemsetAsync(a->dW, 0, 4ull * E * E, a->stream), "memset dW");
        cuda_check(cudaMemsetAsync(a->gl_acc, 0, 8ull * a->bwd_grid, a->stream), "memset g_leak");
        if (!a->tape_last) {  // an earlier backward pass replayed other segments over the tape
            if (!a->replay_graph) {
                cudaGraph_t g = nullptr;
                cuda_check(cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal), "adjoint replay");
                adj_tape_segment(a, a->n_ckpt - 1, false);
                const cudaError_t launch_err = cudaGetLastError();
                cuda_check(cudaStreamEndCapture(a->stream, &g), "adjoint replay");
                cuda_check(launch_err, "adjoint replay");
                cudaGraphGetNodes(g, nullptr, &a->replay_nodes);
                const cudaError_t ie = cudaGraphInstantiate(&a->replay_graph, g, 0);
                cudaGraphDestroy(g);
                cuda_check(ie, "adjoint replay");
            }
            cuda_check(cudaGraphLaunch(a->replay_graph, a->stream), "adjoint replay");
            a->launches += a->replay_nodes;
            a->tape_last = true;
        }
        adj_run_graphs(a, a->bwd_graphs, a->bwd_nodes, true, [&](uint32_t c) { adj_backward_segment(a, c); },
                       "adjoint backward");
        if (a->n_ckpt > 1) a->tape_last = false;
        std::vector<double> gl(a->bwd_grid);
        int32_t err = 0;
        cuda_check(cudaMemcpyAsync(gl.data(), a->gl_acc, 8ull * a->bwd_grid, cudaMemcpyDeviceToHost, a->stream),
                   "D2H g_leak");
        cuda_check(cudaMemcpyAsync(&err, a->error, sizeof(err), cudaMemcpyDeviceToHost, a->stream), "D2H error");
        if (grad_w_ee)
            cuda_check(cudaMemcpyAsync(grad_w_ee, a->dW, 4ull * E * E, cudaMemcpyDeviceToHost, a->stream), "D2H dW");
        cuda_check(cudaStreamSynchronize(a->stream), "adjoint backward");
        if (err != kErrNone) {
            a->have_forward = false;
            throw ApiError(BSNN_ERR_DEVICE_TIMEOUT, "adjoint backward: a grid-barrier wait timed out");
        }
        if (grad_g_leak) {
            double s = 0.0;
            for (double x : gl) s += x;
            *grad_g_leak = s;
        }
    });
}

}  // extern "C"
