// adjoint_api.cuh -- host side of the differentiation form (bsnn_adjoint_* in include/bsnn.h);
// included at the end of bsnn_api.cu.
//
// bsnn_adjoint_forward runs the network for num_steps, checkpointing the state every
// checkpoint_interval steps, and evaluates
//     L = rate_weight / T * sum_t (rho_t - rho*_t)^2 + voltage_weight / T * sum_t (vbar_{t+1} - v*_t)^2
// with rho_t = a rho_{t-1} + (1 - a) n_E(t) / (N_E dt), a = exp(-dt / rate_tau) (the smoothed
// excitatory population rate) and vbar the mean excitatory membrane potential after the step.
// bsnn_adjoint_backward replays each segment from its checkpoint and propagates the adjoints back
// (adjoint_kernel.cuh), returning dL/dW_EE and dL/dg_leak (one g_leak shared by both groups).
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
    float *lam_v = nullptr, *lam_d = nullptr, *lam_r = nullptr, *lam_x = nullptr, *lam_gi = nullptr;
    float* dW = nullptr;
    double* gl_acc = nullptr;
    double* vsum = nullptr;       // [T][vblocks] partial sums of the E voltages after each step
    uint32_t* counts = nullptr;   // [T] E spikes per step
    float* ckpt = nullptr;        // [n_ckpt][12][N]: 11 state arrays + x
    uint32_t n_ckpt = 0, vblocks = 0;
    std::vector<float> v0;        // initial voltages
    // forward results
    std::vector<double> rho, vbar;
    std::vector<float> rate_target, v_target;
    bool have_forward = false;
    ~bsnn_adjoint() {
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

// Partial sums of the E voltages (after a forward step) per block of 256 neurons, fixed order.
__global__ void bsnn_adj_vsum(const float* v, uint32_t E, double* out) {
    __shared__ double red[256];
    const uint32_t n = blockIdx.x * 256u + threadIdx.x;
    red[threadIdx.x] = n < E ? static_cast<double>(v[n]) : 0.0;
    __syncthreads();
    for (uint32_t o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

float** adj_state(bsnn_adjoint* a, int k) {
    float** f[11] = {&a->h.v, &a->h.ge, &a->h.gi, &a->h.istim, &a->h.er, &a->h.ed, &a->h.ir, &a->h.id, &a->h.tr, &a->h.td,
                     reinterpret_cast<float**>(&a->h.refrac)};
    return f[k];
}

void adj_reset(bsnn_adjoint* a) {
    const size_t bytes = 4ull * a->h.N;
    for (int k = 0; k < 11; ++k) cuda_check(cudaMemsetAsync(*adj_state(a, k), 0, bytes, a->stream), "memset state");
    cuda_check(cudaMemcpyAsync(a->h.v, a->v0.data(), bytes, cudaMemcpyHostToDevice, a->stream), "H2D v0");
    cuda_check(cudaMemsetAsync(a->x_cur, 0, bytes, a->stream), "memset x");
}

void adj_checkpoint(bsnn_adjoint* a, uint32_t c, bool save) {
    const size_t bytes = 4ull * a->h.N;
    float* base = a->ckpt + static_cast<size_t>(c) * 12u * a->h.N;
    for (int k = 0; k < 12; ++k) {
        float* dev = k < 11 ? *adj_state(a, k) : a->x_cur;
        float* slot = base + static_cast<size_t>(k) * a->h.N;
        cuda_check(cudaMemcpyAsync(save ? slot : dev, save ? dev : slot, bytes, cudaMemcpyDeviceToDevice, a->stream),
                   "checkpoint copy");
    }
}

// One forward step t: neuron update (tape rows at the given pointers), then g += W^T x_{t+1}.
void adj_step(bsnn_adjoint* a, uint32_t t, float* tv, float* tu, float* tge, float* tgi, uint8_t* ts, uint8_t* tref,
              float* x_next) {
    const uint32_t N = a->h.N, E = a->h.E, I = a->h.I;
    const uint32_t nb = (N + 255) / 256;
    bsnn_adj_neuron_fwd<<<nb, 256, 0, a->stream>>>(a->h, t, tv, tu, tge, tgi, ts, tref, x_next, a->counts + t);
    const dim3 pg((N + 255) / 256, kAdjChunks);
    bsnn_adj_propagate<<<pg, 256, 0, a->stream>>>(a->WE, E, N, x_next, a->part);
    bsnn_adj_reduce<<<nb, 256, 0, a->stream>>>(a->part, kAdjChunks, N, a->h.ge);
    bsnn_adj_propagate<<<pg, 256, 0, a->stream>>>(a->WI, I, N, x_next + E, a->part);
    bsnn_adj_reduce<<<nb, 256, 0, a->stream>>>(a->part, kAdjChunks, N, a->h.gi);
    cuda_check(cudaGetLastError(), "adjoint forward step");
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
        a->vblocks = (E + 255) / 256;
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
        const size_t o_we = A.take(4ull * E * N), o_wi = A.take(4ull * I * N);
        const size_t o_part = A.take(4ull * kAdjChunks * N), o_x = A.take(fN);
        const size_t o_tv = A.take(fN * C), o_tu = A.take(fN * C), o_tge = A.take(fN * C), o_tgi = A.take(fN * C);
        const size_t o_tx = A.take(fN * (C + 1)), o_lge = A.take(fN * C);
        const size_t o_ts = A.take(static_cast<size_t>(N) * C), o_tref = A.take(static_cast<size_t>(N) * C);
        const size_t o_lv = A.take(fN), o_ld = A.take(fN), o_lr = A.take(fN), o_lx = A.take(fN), o_lgi = A.take(fN);
        const size_t o_dw = A.take(4ull * E * E);
        const uint32_t nb = (N + 255) / 256;
        const size_t o_gl = A.take(8ull * nb);
        const size_t o_vs = A.take(8ull * a->vblocks * T);
        const size_t o_cnt = A.take(4ull * T);
        const size_t o_ck = A.take(fN * 12u * a->n_ckpt);
        const size_t o_soff = A.take(4ull * soff.size()), o_evn = A.take(4ull * std::max<size_t>(evn.size(), 1)),
                     o_evd = A.take(4ull * std::max<size_t>(evd.size(), 1));
        cuda_check(cudaMalloc(&a->arena, A.size), "cudaMalloc adjoint arena");
        unsigned char* base = a->arena;
        cuda_check(cudaMemset(base, 0, A.size), "cudaMemset adjoint arena");
        auto F = [&](size_t o) { return reinterpret_cast<float*>(base + o); };
        for (int k = 0; k < 11; ++k) *adj_state(a.get(), k) = F(o_state[k]);
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
        a->vsum = reinterpret_cast<double*>(base + o_vs);
        a->counts = reinterpret_cast<uint32_t*>(base + o_cnt);
        a->ckpt = F(o_ck);
        h.stim_len = stimulus_steps;
        h.stim_off = reinterpret_cast<const uint32_t*>(base + o_soff);
        h.ev_neuron = reinterpret_cast<const uint32_t*>(base + o_evn);
        h.ev_delta = F(o_evd);
        cuda_check(cudaMemcpy(base + o_soff, soff.data(), 4ull * soff.size(), cudaMemcpyHostToDevice), "H2D");
        if (!evn.empty()) {
            cuda_check(cudaMemcpy(base + o_evn, evn.data(), 4ull * evn.size(), cudaMemcpyHostToDevice), "H2D");
            cuda_check(cudaMemcpy(base + o_evd, evd.data(), 4ull * evd.size(), cudaMemcpyHostToDevice), "H2D");
        }
        // W_E = [W_EE | W_EI], W_I = [W_IE | W_II], row-major [pre][N]
        std::vector<float> row(N);
        for (uint32_t i = 0; i < E; ++i) {
            std::memcpy(row.data(), w_ee + static_cast<size_t>(i) * E, 4ull * E);
            std::memcpy(row.data() + E, w_ei + static_cast<size_t>(i) * I, 4ull * I);
            cuda_check(cudaMemcpy(a->WE + static_cast<size_t>(i) * N, row.data(), fN, cudaMemcpyHostToDevice), "H2D W");
        }
        for (uint32_t i = 0; i < I; ++i) {
            std::memcpy(row.data(), w_ie + static_cast<size_t>(i) * E, 4ull * E);
            std::memcpy(row.data() + E, w_ii + static_cast<size_t>(i) * I, 4ull * I);
            cuda_check(cudaMemcpy(a->WI + static_cast<size_t>(i) * N, row.data(), fN, cudaMemcpyHostToDevice), "H2D W");
        }
        a->v0.resize(N);
        for (uint32_t n = 0; n < N; ++n) a->v0[n] = n < E ? e_group->v_rest : i_group->v_rest;
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

// New parameter values: the E->E weights (row-major [E][E]; null keeps them) and g_leak of both
// groups (a NaN keeps it).
BSNN_API bsnn_status bsnn_adjoint_set_params(bsnn_adjoint* a, const float* w_ee, float g_leak) {
    if (!a) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_adj(a, [&] {
        const uint32_t E = a->h.E, N = a->h.N;
        if (w_ee)
            cuda_check(cudaMemcpy2D(a->WE, 4ull * N, w_ee, 4ull * E, 4ull * E, E, cudaMemcpyHostToDevice), "H2D W_EE");
        if (!std::isnan(g_leak)) {
            a->h.g[0].g_leak = g_leak;
            a->h.g[1].g_leak = g_leak;
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
        const uint32_t T = a->d.num_steps, C = a->d.checkpoint_interval, N = a->h.N, E = a->h.E;
        require(rate_target != nullptr, BSNN_ERR_INVALID_ARGUMENT, "null rate target");
        require(voltage_target != nullptr || !(a->d.voltage_weight != 0.0f), BSNN_ERR_INVALID_ARGUMENT,
                "null voltage target with a voltage weight");
        adj_reset(a);
        cuda_check(cudaMemsetAsync(a->counts, 0, 4ull * T, a->stream), "memset counts");
        for (uint32_t t = 0; t < T; ++t) {
            if (t % C == 0) adj_checkpoint(a, t / C, true);
            // tape rows go to slot 0 (not kept in the forward pass); x_{t+1} into x_cur
            adj_step(a, t, a->tv, a->tu, a->tge, a->tgi, a->ts, a->tref, a->x_cur);
            bsnn_adj_vsum<<<a->vblocks, 256, 0, a->stream>>>(a->h.v, E, a->vsum + static_cast<size_t>(t) * a->vblocks);
        }
        std::vector<uint32_t> cnt(T);
        std::vector<double> vs(static_cast<size_t>(T) * a->vblocks);
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
            for (uint32_t b = 0; b < a->vblocks; ++b) s += vs[static_cast<size_t>(t) * a->vblocks + b];
            a->vbar[t] = s / E;
            const double er = rho - rate_target[t], ev = a->vbar[t] - a->v_target[t];
            loss += a->d.rate_weight * er * er + a->d.voltage_weight * ev * ev;
            if (rate_out) rate_out[t] = static_cast<float>(rho);
            if (mean_voltage_out) mean_voltage_out[t] = static_cast<float>(a->vbar[t]);
        }
        if (loss_out) *loss_out = static_cast<float>(loss / T);
        a->have_forward = true;
        (void)N;
    });
}

// The gradients of the last forward pass's loss: dL/dW_EE (row-major [E][E]) and dL/dg_leak.
BSNN_API bsnn_status bsnn_adjoint_backward(bsnn_adjoint* a, float* grad_w_ee, double* grad_g_leak) {
    if (!a) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded_adj(a, [&] {
        require(a->have_forward, BSNN_ERR_STATE, "run bsnn_adjoint_forward first");
        const uint32_t T = a->d.num_steps, C = a->d.checkpoint_interval, N = a->h.N, E = a->h.E, I = a->h.I;
        const size_t fN = 4ull * N;
        const uint32_t nb = (N + 255) / 256;
        const double dt = a->h.g[0].timestep, ka = std::exp(-dt / static_cast<double>(a->d.rate_tau));
        // the loss's sensitivities to the step's E spikes (through rho) and to vbar_{t+1}
        std::vector<float> c_s(T), c_v(T);
        double lrho = 0.0;
        for (uint32_t t = T; t-- > 0;) {
            lrho = ka * lrho + a->d.rate_weight * 2.0 / T * (a->rho[t] - a->rate_target[t]);
            c_s[t] = static_cast<float>(lrho * (1.0 - ka) / (static_cast<double>(E) * dt));
            c_v[t] = static_cast<float>(a->d.voltage_weight * 2.0 / T * (a->vbar[t] - a->v_target[t]) / E);
        }
        for (float* p : {a->lam_v, a->lam_d, a->lam_r, a->lam_x})
            cuda_check(cudaMemsetAsync(p, 0, fN, a->stream), "memset adjoints");
        cuda_check(cudaMemsetAsync(a->dW, 0, 4ull * E * E, a->stream), "memset dW");
        cuda_check(cudaMemsetAsync(a->gl_acc, 0, 8ull * nb, a->stream), "memset g_leak");
        const float beta = a->d.surrogate_beta;
        for (uint32_t c = a->n_ckpt; c-- > 0;) {
            const uint32_t t0 = c * C, t1 = std::min(T, t0 + C), steps = t1 - t0;
            // replay the segment, keeping every step's tape row
            adj_checkpoint(a, c, false);
            cuda_check(cudaMemcpyAsync(a->tx, a->x_cur, fN, cudaMemcpyDeviceToDevice, a->stream), "x_t0");
            for (uint32_t k = 0; k < steps; ++k) {
                const size_t o = static_cast<size_t>(k) * N;
                adj_step(a, t0 + k, a->tv + o, a->tu + o, a->tge + o, a->tgi + o, a->ts + o, a->tref + o,
                         a->tx + o + N);
            }
            // backwards through the segment
            for (uint32_t k = steps; k-- > 0;) {
                const size_t o = static_cast<size_t>(k) * N;
                float* lge = a->lge_all + o;
                bsnn_adj_neuron_bwd<<<nb, 256, 0, a->stream>>>(a->h, a->tv + o, a->tu + o, a->tge + o, a->tgi + o,
                                                               a->ts + o, a->tref + o, a->lam_v, a->lam_d, a->lam_r,
                                                               a->lam_x, c_s[t0 + k], c_v[t0 + k], beta, lge, a->lam_gi,
                                                               a->gl_acc);
                // lambda_x(t) = W lambda_g(t), for step t - 1
                bsnn_adj_pullback<<<(E * 32 + 255) / 256, 256, 0, a->stream>>>(a->WE, E, N, lge, a->lam_x);
                bsnn_adj_pullback<<<(I * 32 + 255) / 256, 256, 0, a->stream>>>(a->WI, I, N, a->lam_gi, a->lam_x + E);
            }
            // dW_EE += sum over the segment of x_t lambda_ge(t)^T
            const dim3 og((E + 31) / 32, (E + 31) / 32);
            bsnn_adj_outer<<<og, 256, 0, a->stream>>>(a->tx, a->lge_all, steps, N, E, a->dW);
            cuda_check(cudaGetLastError(), "adjoint backward segment");
        }
        std::vector<double> gl(nb);
        cuda_check(cudaMemcpyAsync(gl.data(), a->gl_acc, 8ull * nb, cudaMemcpyDeviceToHost, a->stream), "D2H g_leak");
        if (grad_w_ee)
            cuda_check(cudaMemcpyAsync(grad_w_ee, a->dW, 4ull * E * E, cudaMemcpyDeviceToHost, a->stream), "D2H dW");
        cuda_check(cudaStreamSynchronize(a->stream), "adjoint backward");
        if (grad_g_leak) {
            double s = 0.0;
            for (double x : gl) s += x;
            *grad_g_leak = s;
        }
    });
}

}  // extern "C"
