// bsnn_oracle.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY; see bsnn_oracle.h).
//
// Each function below restates one kernel of the reference, in the reference's launch order,
// and cites the file:line it follows.  The FP32 instantiation repeats the reference's
// statement-level float arithmetic (built with -ffp-contract=off so no FMA is introduced);
// the FP64 instantiation runs the same statements in double.
//
// Deliberate differences from the reference, each because the reference's arithmetic lives in
// a closed library that must not be restated:
//  * Background Poisson counts come from this project's counter-based Philox4x32-10 (Salmon,
//    Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11) keyed by
//    (rng_seed, neuron, step) and Knuth's multiplication method (TAOCP vol. 2, 3.4.1), not
//    curand_poisson on a curandStatePhilox4_32_10_t (kernel_neuron_group_evolve.cu:53-54).
//    The replay mode feeds externally recorded counts instead.
//  * The cublasSgemv dot products (kernel_connection_propagate.cu:79-94) are accumulated in
//    double and rounded once, since cuBLAS's summation order is unspecified.
#include "bsnn_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <thread>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 (SC'11, section 5): 10 rounds of two 32x32->64 multiplies with Weyl-sequence
// key schedule.  Round constants are the published ones.
constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

void philox4x32_10(const uint32_t in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = static_cast<uint64_t>(kPhiloxM0) * c0;
        const uint64_t p1 = static_cast<uint64_t>(kPhiloxM1) * c2;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Poisson(mean) by Knuth's multiplication method: multiply uniforms u in (0, 1] until the
// product drops to exp(-mean).  Counter = (neuron, step lo, step hi, channel << 16 | block),
// key = (seed, 0).  Counts saturate at 255.
uint32_t poisson_knuth(float exp_neg_mean, uint32_t seed, uint32_t neuron, uint64_t step, uint32_t channel) {
    const uint32_t key[2] = {seed, 0u};
    float p = 1.0f;
    uint32_t k = 0;
    for (uint32_t block = 0;; ++block) {
        const uint32_t ctr[4] = {neuron, static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32),
                                 (channel << 16) | (block & 0xFFFFu)};
        uint32_t r[4];
        philox4x32_10(ctr, key, r);
        for (int i = 0; i < 4; ++i) {
            const float u = static_cast<float>((r[i] >> 8) + 1u) * 5.9604644775390625e-8f;  // 2^-24
            p = p * u;
            if (p <= exp_neg_mean) return k;
            ++k;
            if (k >= 255u) return 255u;
        }
    }
}

// Deterministic parallel loop for the O(N^2) kernels: static contiguous partition over host
// threads; each index is computed by exactly one thread, so results do not depend on the count.
unsigned g_threads = 0;
unsigned thread_count() {
    if (g_threads == 0) {
        const char* e = std::getenv("ORACLE_THREADS");
        g_threads = e ? static_cast<unsigned>(std::max(1, std::atoi(e))) : std::max(1u, std::thread::hardware_concurrency());
    }
    return g_threads;
}
template <class F>
void parallel_for(uint32_t n, F&& f) {
    const unsigned T = std::min<unsigned>(thread_count(), std::max<uint32_t>(1u, n / 256u));
    if (T <= 1) {
        for (uint32_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(T);
    for (unsigned t = 0; t < T; ++t) {
        const uint32_t a = static_cast<uint32_t>(static_cast<uint64_t>(n) * t / T);
        const uint32_t b = static_cast<uint32_t>(static_cast<uint64_t>(n) * (t + 1) / T);
        pool.emplace_back([a, b, &f] { for (uint32_t i = a; i < b; ++i) f(i); });
    }
    for (auto& th : pool) th.join();
}

float exp_neg_mean_of(float mean) { return static_cast<float>(std::exp(-static_cast<double>(mean))); }

struct Err : std::runtime_error {
    int32_t code;
    Err(int32_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};

template <class R>
R r_exp(R x);
template <>
float r_exp<float>(float x) { return expf(x); }
template <>
double r_exp<double>(double x) { return std::exp(x); }

template <class R>
struct Group {
    bsnn_neuron_group_params p;
    float exp_neg_mean_e = 1.0f, exp_neg_mean_i = 1.0f;
};

template <class R>
struct Conn {
    uint32_t pre, post;  // group indices
    bsnn_connection_params p;
    R r_decay, d_decay, norm;
    uint32_t n_pre, n_post, pre_off, post_off;
    bool pre_inhib;
    std::vector<R> w;  // row-major [pre][post]
    std::vector<R> r, d, x;
};

template <class R>
struct Plast {
    int32_t kind;
    uint32_t conn;
    bsnn_plasticity_params p;
    std::vector<R> pre, post, tpre, tpost, sums;
};

struct Mon {
    int kind;  // 0 spikes, 1 voltage
    uint32_t group, interval;
    std::vector<uint32_t> sel;
    std::vector<uint32_t> sh;  // [n_group][interval]
    std::vector<float> vh;     // [n_group][interval]
};

struct Stim {
    std::vector<uint32_t> counts, ids, offs;
    std::vector<float> deltas;
    uint32_t cursor_t = 0, cursor_e = 0;
};

struct SimBase {
    virtual ~SimBase() = default;
    std::string err;
};

template <class R>
struct Sim : SimBase {
    bsnn_state_desc desc{};
    uint32_t N = 0;
    std::vector<Group<R>> groups;
    std::vector<Conn<R>> conns;
    std::vector<Plast<R>> plasts;
    std::vector<Mon> mons;
    std::vector<Stim> stims;
    // per-neuron state (GpuSimulationState SoA buffers, gpu_simulation_state.cu:35-52)
    std::vector<R> v, ge, gi, istim, bg_ge, bg_gi, bg_er, bg_ed, bg_ir, bg_id;
    std::vector<uint32_t> refrac, spikes;
    std::vector<uint8_t> last_counts;
    int32_t noise_mode = BSNN_NOISE_PHILOX;
    std::vector<uint8_t> replay;
    uint32_t replay_steps = 0;
    uint64_t steps_done = 0;

    explicit Sim(const bsnn_state_desc& d) : desc(d) {
        if (desc.recording_interval_steps == 0) desc.recording_interval_steps = 10000;
        N = desc.num_excitatory_neurons + desc.num_inhibitory_neurons;
        v.assign(N, R(0)); ge.assign(N, R(0)); gi.assign(N, R(0)); istim.assign(N, R(0));
        bg_ge.assign(N, R(0)); bg_gi.assign(N, R(0)); bg_er.assign(N, R(0)); bg_ed.assign(N, R(0));
        bg_ir.assign(N, R(0)); bg_id.assign(N, R(0));
        refrac.assign(N, 0u); spikes.assign(N, 0u);
        last_counts.assign(static_cast<size_t>(N) * 2, 0);
    }

    // kernel_update_background_conductances (cpp_src/neuron_groups/kernel_neuron_group_evolve.cu:11-83)
    void background(const Group<R>& g) {
        const auto& p = g.p;
        for (uint32_t i = 0; i < p.num_neurons; ++i) {
            const uint32_t j = p.offset + i;
            R t;
            t = bg_er[j] * R(p.background_excitatory_postsynaptic_r_trace_decay); if (t < R(1e-30f)) t = R(0); bg_er[j] = t;
            t = bg_ir[j] * R(p.background_inhibitory_postsynaptic_r_trace_decay); if (t < R(1e-30f)) t = R(0); bg_ir[j] = t;
            t = bg_ed[j] * R(p.background_excitatory_postsynaptic_d_trace_decay); if (t < R(1e-30f)) t = R(0); bg_ed[j] = t;
            t = bg_id[j] * R(p.background_inhibitory_postsynaptic_d_trace_decay); if (t < R(1e-30f)) t = R(0); bg_id[j] = t;
            uint32_t ne = 0, ni = 0;
            if (noise_mode == BSNN_NOISE_PHILOX) {
                if (p.mean_background_excitatory_spikes > 0.0f)
                    ne = poisson_knuth(g.exp_neg_mean_e, static_cast<uint32_t>(desc.rng_seed), j, steps_done, 0);
                if (p.mean_background_inhibitory_spikes > 0.0f)
                    ni = poisson_knuth(g.exp_neg_mean_i, static_cast<uint32_t>(desc.rng_seed), j, steps_done, 1);
            } else if (noise_mode == BSNN_NOISE_REPLAY && steps_done < replay_steps) {
                const size_t base = (static_cast<size_t>(steps_done) * N + j) * 2;
                ne = replay[base];
                ni = replay[base + 1];
            }
            last_counts[static_cast<size_t>(j) * 2] = static_cast<uint8_t>(ne);
            last_counts[static_cast<size_t>(j) * 2 + 1] = static_cast<uint8_t>(ni);
            if (ne > 0u) { const R inc = R(static_cast<float>(ne)); bg_er[j] += inc; bg_ed[j] += inc; }
            bg_ge[j] = (bg_ed[j] - bg_er[j]) * R(p.background_excitatory_scaling_factor);
            if (ni > 0u) { const R inc = R(static_cast<float>(ni)); bg_ir[j] += inc; bg_id[j] += inc; }
            bg_gi[j] = (bg_id[j] - bg_ir[j]) * R(p.background_inhibitory_scaling_factor);
        }
    }

    // kernel_neuron_group_evolve (cpp_src/neuron_groups/kernel_neuron_group_evolve.cu:85-130)
    void evolve(const Group<R>& g) {
        const auto& p = g.p;
        for (uint32_t i = 0; i < p.num_neurons; ++i) {
            const uint32_t j = p.offset + i;
            if (refrac[j] > 0) {
                --refrac[j];
                spikes[j] = 0;
                v[j] = R(p.v_reset);
            } else {
                const R vv = v[j];
                const R lin = R(-1.0f) * R(p.g_leak) * (vv - R(p.v_rest));
                const R ex = R(p.g_leak) * R(p.depolarization_slope_factor) *
                             r_exp<R>((vv - R(p.v_effective_spike_threshold)) / R(p.depolarization_slope_factor));
                const R es = R(-1.0f) * ge[j] * (vv - R(p.v_excitatory_reversal));
                const R is = R(-1.0f) * gi[j] * (vv - R(p.v_inhibitory_reversal));
                const R st = istim[j];
                const R dv = (R(p.timestep) / R(p.membrane_capacitance)) * (lin + ex + es + is + st);
                const R vn = vv + dv;
                if (vn >= R(p.v_threshold)) {
                    refrac[j] = p.refractory_steps;
                    spikes[j] = 1;
                    v[j] = R(p.v_threshold);
                } else {
                    spikes[j] = 0;
                    v[j] = vn;
                }
            }
            ge[j] = bg_ge[j];
            gi[j] = bg_gi[j];
        }
    }

    // kernel_connection_decay_d_traces / _r_traces / _update_conductances_with_spikes and the
    // cublasSgemv accumulate (cpp_src/connections/kernel_connection_propagate.cu:8-46, 64-111)
    void propagate(Conn<R>& c) {
        for (uint32_t i = 0; i < c.n_pre; ++i) {
            R t = c.d[i] * c.d_decay; if (t < R(1e-30f)) t = R(0); c.d[i] = t;
        }
        for (uint32_t i = 0; i < c.n_pre; ++i) {
            R t = c.r[i] * c.r_decay; if (t < R(1e-30f)) t = R(0); c.r[i] = t;
        }
        for (uint32_t i = 0; i < c.n_pre; ++i) {
            if (spikes[c.pre_off + i] == 1) { c.r[i] += c.norm; c.d[i] += c.norm; }
            c.x[i] = c.d[i] - c.r[i];
        }
        std::vector<R>& y = c.pre_inhib ? gi : ge;
        parallel_for(c.n_post, [&](uint32_t q) {
            double acc = 0.0;
            for (uint32_t i = 0; i < c.n_pre; ++i)
                acc += static_cast<double>(c.w[static_cast<size_t>(i) * c.n_post + q]) * static_cast<double>(c.x[i]);
            y[c.post_off + q] = static_cast<R>(acc) + y[c.post_off + q];
        });
    }

    // Stimulus::apply + kernel_stimulus_apply (cpp_src/stimuli/stimulus.cpp:46-60,
    // cpp_src/stimuli/kernel_stimulus_apply.cu:7-21); atomicAdd order taken as event order.
    void apply_stimulus(Stim& st) {
        if (st.cursor_t >= st.counts.size()) return;
        const uint32_t n = st.counts[st.cursor_t];
        if (static_cast<uint64_t>(st.cursor_e) + n > st.ids.size())
            throw Err(BSNN_ERR_RUNTIME, "Stimulus event indexing exceeded uploaded event buffers");
        for (uint32_t e = 0; e < n; ++e) {
            const uint32_t k = st.cursor_e + e;
            const uint32_t j = st.ids[k] + st.offs[k];
            if (j >= N) throw Err(BSNN_ERR_OUT_OF_RANGE, "stimulus event neuron out of range");
            istim[j] = istim[j] + R(st.deltas[k]);
        }
        st.cursor_e += n;
        ++st.cursor_t;
    }

    static R clampw(R w, const bsnn_plasticity_params& p) {
        if (w < R(p.weight_min)) return R(p.weight_min);
        if (w > R(p.weight_max)) return R(p.weight_max);
        return w;
    }

    // kernel_triplet_plasticity_update_normalize_launch (cpp_src/plasticities/kernel_triplet_plasticity_update.cu:181-216)
    // with its kernels :16-145.
    void triplet(Plast<R>& pl) {
        Conn<R>& c = conns[pl.conn];
        const auto& p = pl.p;
        const uint32_t* pre_s = &spikes[c.pre_off];
        const uint32_t* post_s = &spikes[c.post_off];
        for (uint32_t i = 0; i < c.n_pre; ++i) {  // decay pre (:16-33)
            R t = pl.pre[i] * R(p.pre_trace_decay); if (t < R(1e-30f)) t = R(0); pl.pre[i] = t;
            t = pl.tpre[i] * R(p.triplet_pre_trace_decay); if (t < R(1e-30f)) t = R(0); pl.tpre[i] = t;
        }
        for (uint32_t q = 0; q < c.n_post; ++q) {  // decay post (:35-52)
            R t = pl.post[q] * R(p.post_trace_decay); if (t < R(1e-30f)) t = R(0); pl.post[q] = t;
            t = pl.tpost[q] * R(p.triplet_post_trace_decay); if (t < R(1e-30f)) t = R(0); pl.tpost[q] = t;
        }
        parallel_for(c.n_post, [&](uint32_t q) {  // LTP (:54-72)
            if (post_s[q] != 1) return;
            for (uint32_t i = 0; i < c.n_pre; ++i) {
                if (i == q) continue;
                R& w = c.w[static_cast<size_t>(i) * c.n_post + q];
                const R delta = pl.pre[i] * (R(p.ltp_A) + (R(p.ltp_B) * pl.tpost[q]));
                w = clampw(w + delta, p);
            }
        });
        parallel_for(c.n_pre, [&](uint32_t i) {  // LTD (:74-93)
            if (pre_s[i] != 1) return;
            for (uint32_t q = 0; q < c.n_post; ++q) {
                if (i == q) continue;
                R& w = c.w[static_cast<size_t>(i) * c.n_post + q];
                const R delta = R(-1.0f) * pl.post[q] * (R(p.ltd_A) + (R(p.ltd_B) * pl.tpre[i]));
                w = clampw(w + delta, p);
            }
        });
        parallel_for(c.n_pre, [&](uint32_t i) {  // normalize (:117-145)
            R* row = &c.w[static_cast<size_t>(i) * c.n_post];
            R sum = R(0);
            for (uint32_t q = 0; q < c.n_post; ++q) sum += row[q];
            if (sum <= R(0)) return;
            const R scale = pl.sums[i] / sum;
            for (uint32_t q = 0; q < c.n_post; ++q) row[q] *= scale;
        });
        for (uint32_t i = 0; i < c.n_pre; ++i)  // increment pre (:106-115)
            if (pre_s[i] == 1) { pl.pre[i] += R(1.0f); pl.tpre[i] += R(1.0f); }
        for (uint32_t q = 0; q < c.n_post; ++q)  // increment post (:95-104)
            if (post_s[q] == 1) { pl.post[q] += R(1.0f); pl.tpost[q] += R(1.0f); }
    }

    // kernel_istdp_plasticity_update_launch (cpp_src/plasticities/kernel_istdp_plasticity_update.cu:103-135)
    // and kernel_stdp_plasticity_update_launch (kernel_stdp_plasticity_update.cu:104-137);
    // they differ only in the LTD delta (:77 in either file).
    void pair_rule(Plast<R>& pl, bool istdp) {
        Conn<R>& c = conns[pl.conn];
        const auto& p = pl.p;
        const uint32_t* pre_s = &spikes[c.pre_off];
        const uint32_t* post_s = &spikes[c.post_off];
        for (uint32_t i = 0; i < c.n_pre; ++i) {
            R t = pl.pre[i] * R(p.pre_trace_decay); if (t < R(1e-30f)) t = R(0); pl.pre[i] = t;
        }
        for (uint32_t q = 0; q < c.n_post; ++q) {
            R t = pl.post[q] * R(p.post_trace_decay); if (t < R(1e-30f)) t = R(0); pl.post[q] = t;
        }
        parallel_for(c.n_post, [&](uint32_t q) {  // LTP (:42-60)
            if (post_s[q] != 1) return;
            for (uint32_t i = 0; i < c.n_pre; ++i) {
                if (i == q) continue;
                R& w = c.w[static_cast<size_t>(i) * c.n_post + q];
                const R delta = R(p.ltp_A) * pl.pre[i];
                w = clampw(w + delta, p);
            }
        });
        parallel_for(c.n_pre, [&](uint32_t i) {  // LTD (:62-81)
            if (pre_s[i] != 1) return;
            for (uint32_t q = 0; q < c.n_post; ++q) {
                if (i == q) continue;
                R& w = c.w[static_cast<size_t>(i) * c.n_post + q];
                const R delta = istdp ? R(-1.0f) * R(p.ltd_A) * (pl.post[q] - R(p.ltd_B))
                                      : R(-1.0f) * R(p.ltd_A) * pl.post[q];
                w = clampw(w + delta, p);
            }
        });
        for (uint32_t i = 0; i < c.n_pre; ++i)
            if (pre_s[i] == 1) pl.pre[i] += R(1.0f);
        for (uint32_t q = 0; q < c.n_post; ++q)
            if (post_s[q] == 1) pl.post[q] += R(1.0f);
    }

    // SpikeRecorder::historicize / VoltageRecorder::historicize with
    // kernel_historicize_spikes / _membrane_potentials (cpp_src/monitors/kernel_historicize_spikes.cu:7-21,
    // kernel_historicize_membrane_potentials.cu:7-21)
    void historicize(Mon& m, uint32_t clock) {
        const auto& gp = groups[m.group].p;
        const uint32_t slot = clock % m.interval;
        for (uint32_t i = 0; i < gp.num_neurons; ++i) {
            if (m.kind == 0) m.sh[static_cast<size_t>(i) * m.interval + slot] = spikes[gp.offset + i];
            else m.vh[static_cast<size_t>(i) * m.interval + slot] = static_cast<float>(v[gp.offset + i]);
        }
    }

    // System::step_the_clock (cpp_src/core/system.cpp:43-63)
    void step(uint32_t clock) {
        for (auto& g : groups) { background(g); evolve(g); }
        for (auto& c : conns) propagate(c);
        for (auto& s : stims) apply_stimulus(s);
        for (auto& pl : plasts) {
            if (pl.kind == BSNN_PLASTICITY_TRIPLET) triplet(pl);
            else pair_rule(pl, pl.kind == BSNN_PLASTICITY_ISTDP);
        }
        for (auto& m : mons) historicize(m, clock);
        ++steps_done;
    }

    std::vector<R>* field_vec(int32_t f, uint32_t idx, uint32_t* len) {
        *len = N;
        switch (f) {
            case BSNN_FIELD_MEMBRANE_POTENTIALS: return &v;
            case BSNN_FIELD_G_EXCITATORY: return &ge;
            case BSNN_FIELD_G_INHIBITORY: return &gi;
            case BSNN_FIELD_I_STIMULUS: return &istim;
            case BSNN_FIELD_BG_G_EXCITATORY: return &bg_ge;
            case BSNN_FIELD_BG_G_INHIBITORY: return &bg_gi;
            case BSNN_FIELD_BG_E_R_TRACES: return &bg_er;
            case BSNN_FIELD_BG_E_D_TRACES: return &bg_ed;
            case BSNN_FIELD_BG_I_R_TRACES: return &bg_ir;
            case BSNN_FIELD_BG_I_D_TRACES: return &bg_id;
            default: break;
        }
        if (f >= BSNN_FIELD_CONN_R_TRACES && f <= BSNN_FIELD_CONN_SUMMED) {
            if (idx >= conns.size()) throw Err(BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
            auto& c = conns[idx];
            *len = c.n_pre;
            return f == BSNN_FIELD_CONN_R_TRACES ? &c.r : f == BSNN_FIELD_CONN_D_TRACES ? &c.d : &c.x;
        }
        if (f >= BSNN_FIELD_PLAST_PRE_TRACES && f <= BSNN_FIELD_PLAST_PRE_WEIGHT_SUMS) {
            if (idx >= plasts.size()) throw Err(BSNN_ERR_OUT_OF_RANGE, "plasticity index out of range");
            auto& pl = plasts[idx];
            auto& c = conns[pl.conn];
            switch (f) {
                case BSNN_FIELD_PLAST_PRE_TRACES: *len = c.n_pre; return &pl.pre;
                case BSNN_FIELD_PLAST_POST_TRACES: *len = c.n_post; return &pl.post;
                case BSNN_FIELD_PLAST_TRIPLET_PRE: *len = c.n_pre; return &pl.tpre;
                case BSNN_FIELD_PLAST_TRIPLET_POST: *len = c.n_post; return &pl.tpost;
                default: *len = static_cast<uint32_t>(pl.sums.size()); return &pl.sums;
            }
        }
        return nullptr;
    }
};

SimBase* base(or_sim* s) { return reinterpret_cast<SimBase*>(s); }

template <class F>
int32_t guarded(or_sim* s, F&& f) {
    try {
        f();
        return BSNN_OK;
    } catch (const Err& e) {
        if (s) base(s)->err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        if (s) base(s)->err = e.what();
        return BSNN_ERR_RUNTIME;
    }
}

// Dispatches a generic lambda on the concrete precision of `s`.
template <class F>
int32_t with_sim(or_sim* s, F&& f) {
    if (!s) return BSNN_ERR_INVALID_ARGUMENT;
    return guarded(s, [&] {
        if (auto* a = dynamic_cast<Sim<float>*>(base(s))) f(*a);
        else if (auto* b = dynamic_cast<Sim<double>*>(base(s))) f(*b);
        else throw Err(BSNN_ERR_INVALID_ARGUMENT, "bad oracle handle");
    });
}

template <class R>
void add_group(Sim<R>& s, const bsnn_neuron_group_params* p, uint32_t* out) {
    if (!p) throw Err(BSNN_ERR_INVALID_ARGUMENT, "null params");
    if (p->offset > s.N || p->num_neurons > s.N - p->offset)
        throw Err(BSNN_ERR_INVALID_ARGUMENT, "neuron_group slice is out of bounds");
    Group<R> g;
    g.p = *p;
    g.exp_neg_mean_e = exp_neg_mean_of(p->mean_background_excitatory_spikes);
    g.exp_neg_mean_i = exp_neg_mean_of(p->mean_background_inhibitory_spikes);
    // NeuronGroup::initialize_data (cpp_src/neuron_groups/neuron_group.cpp:19-34)
    for (uint32_t i = 0; i < p->num_neurons; ++i) {
        const uint32_t j = p->offset + i;
        s.v[j] = R(p->v_rest);
        s.ge[j] = s.gi[j] = s.istim[j] = R(0);
        s.refrac[j] = 0; s.spikes[j] = 0;
        s.bg_ge[j] = s.bg_gi[j] = s.bg_er[j] = s.bg_ed[j] = s.bg_ir[j] = s.bg_id[j] = R(0);
    }
    s.groups.push_back(g);
    if (out) *out = static_cast<uint32_t>(s.groups.size() - 1);
}

}  // namespace

extern "C" {

BSNN_API or_sim* or_create(const bsnn_state_desc* desc, int32_t precision) {
    if (!desc) return nullptr;
    SimBase* s = nullptr;
    if (precision == OR_PREC_F64) s = new Sim<double>(*desc);
    else s = new Sim<float>(*desc);
    return reinterpret_cast<or_sim*>(s);
}

BSNN_API void or_destroy(or_sim* s) { delete base(s); }

BSNN_API const char* or_last_error(const or_sim* s) {
    return s ? reinterpret_cast<const SimBase*>(s)->err.c_str() : "null oracle handle";
}

BSNN_API int32_t or_add_neuron_group(or_sim* s, const bsnn_neuron_group_params* p, uint32_t* out) {
    return with_sim(s, [&](auto& sim) { add_group(sim, p, out); });
}

BSNN_API int32_t or_add_connection(or_sim* s, uint32_t pre, uint32_t post, const float* w,
                                   const bsnn_connection_params* p, uint32_t* out) {
    return with_sim(s, [&](auto& sim) {
        using R = typename std::decay_t<decltype(sim.v)>::value_type;
        if (!w || !p) throw Err(BSNN_ERR_INVALID_ARGUMENT, "null weights or params");
        if (pre >= sim.groups.size() || post >= sim.groups.size())
            throw Err(BSNN_ERR_OUT_OF_RANGE, "group index out of range");
        Conn<R> c;
        c.pre = pre; c.post = post; c.p = *p;
        // Connection::make_gpu_view (cpp_src/connections/connection.cpp:46-47): decays in float.
        c.r_decay = R(std::exp(-1.0f * p->timestep / p->rise_time));
        c.d_decay = R(std::exp(-1.0f * p->timestep / p->decay_time));
        c.norm = R(p->postsynaptic_kernel_normalization_value);
        const auto& gp = sim.groups[pre].p;
        const auto& gq = sim.groups[post].p;
        c.n_pre = gp.num_neurons; c.n_post = gq.num_neurons;
        c.pre_off = gp.offset; c.post_off = gq.offset;
        c.pre_inhib = gp.is_inhibitory;
        const size_t n = static_cast<size_t>(c.n_pre) * c.n_post;
        c.w.resize(n);
        for (size_t k = 0; k < n; ++k) {
            if (w[k] < 0.0f)
                throw Err(BSNN_ERR_INVALID_ARGUMENT,
                          "connection weight_matrix must be non-negative to preserve inhibitory routing contract");
            c.w[k] = R(w[k]);
        }
        c.r.assign(c.n_pre, R(0)); c.d.assign(c.n_pre, R(0)); c.x.assign(c.n_pre, R(0));
        sim.conns.push_back(std::move(c));
        if (out) *out = static_cast<uint32_t>(sim.conns.size() - 1);
    });
}

BSNN_API int32_t or_add_stimulus(or_sim* s, const uint32_t* counts, uint32_t n_steps, const uint32_t* ids,
                                 const uint32_t* offsets, const float* deltas, uint32_t n_events) {
    return with_sim(s, [&](auto& sim) {
        if (n_steps != sim.desc.total_simulation_length || n_events != sim.desc.num_stimulus_events)
            throw Err(BSNN_ERR_INVALID_ARGUMENT,
                      "upload_stimulus_view host data vectors must match gpu_view.num_stimulus_events and "
                      "total_simulation_length");
        Stim st;
        st.counts.assign(counts, counts + n_steps);
        st.ids.assign(ids, ids + n_events);
        st.offs.assign(offsets, offsets + n_events);
        st.deltas.assign(deltas, deltas + n_events);
        sim.stims.push_back(std::move(st));
    });
}

BSNN_API int32_t or_add_plasticity(or_sim* s, int32_t kind, uint32_t conn, const bsnn_plasticity_params* p,
                                   uint32_t* out) {
    return with_sim(s, [&](auto& sim) {
        using R = typename std::decay_t<decltype(sim.v)>::value_type;
        if (!p) throw Err(BSNN_ERR_INVALID_ARGUMENT, "null params");
        if (conn >= sim.conns.size()) throw Err(BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        if (kind != BSNN_PLASTICITY_TRIPLET && kind != BSNN_PLASTICITY_ISTDP && kind != BSNN_PLASTICITY_STDP)
            throw Err(BSNN_ERR_INVALID_ARGUMENT, "unknown plasticity kind");
        Plast<R> pl;
        pl.kind = kind; pl.conn = conn; pl.p = *p;
        auto& c = sim.conns[conn];
        pl.pre.assign(c.n_pre, R(0)); pl.post.assign(c.n_post, R(0));
        pl.tpre.assign(c.n_pre, R(0)); pl.tpost.assign(c.n_post, R(0));
        if (kind == BSNN_PLASTICITY_TRIPLET) {
            if (c.n_pre > c.n_post)
                throw Err(BSNN_ERR_INVALID_ARGUMENT, "triplet normalisation needs num_pre <= num_post");
            // TripletPlasticity::initialize_data (cpp_src/plasticities/triplet_plasticity.cpp:21-31):
            // column sums in float, ascending pre; used as row targets.
            // (rows in the outer loop: every column still adds in ascending pre order)
            std::vector<float> fsum(c.n_post, 0.0f);
            for (uint32_t i = 0; i < c.n_pre; ++i)
                for (uint32_t q = 0; q < c.n_post; ++q)
                    fsum[q] += static_cast<float>(c.w[static_cast<size_t>(i) * c.n_post + q]);
            std::vector<R> cols(c.n_post, R(0));
            for (uint32_t q = 0; q < c.n_post; ++q) cols[q] = R(fsum[q]);
            pl.sums.assign(cols.begin(), cols.begin() + c.n_pre);
        }
        sim.plasts.push_back(std::move(pl));
        if (out) *out = static_cast<uint32_t>(sim.plasts.size() - 1);
    });
}

BSNN_API int32_t or_add_spike_recorder(or_sim* s, uint32_t group, uint32_t interval, uint32_t* out) {
    return with_sim(s, [&](auto& sim) {
        if (group >= sim.groups.size()) throw Err(BSNN_ERR_OUT_OF_RANGE, "group index out of range");
        Mon m;
        m.kind = 0; m.group = group; m.interval = interval ? interval : sim.desc.recording_interval_steps;
        m.sh.assign(static_cast<size_t>(sim.groups[group].p.num_neurons) * m.interval, 0u);
        sim.mons.push_back(std::move(m));
        if (out) *out = static_cast<uint32_t>(sim.mons.size() - 1);
    });
}

BSNN_API int32_t or_add_voltage_recorder(or_sim* s, uint32_t group, const uint32_t* ids, uint32_t n_ids,
                                         uint32_t interval, uint32_t* out) {
    return with_sim(s, [&](auto& sim) {
        if (group >= sim.groups.size()) throw Err(BSNN_ERR_OUT_OF_RANGE, "group index out of range");
        Mon m;
        m.kind = 1; m.group = group; m.interval = interval ? interval : sim.desc.recording_interval_steps;
        const uint32_t ng = sim.groups[group].p.num_neurons;
        for (uint32_t k = 0; k < n_ids; ++k)
            if (ids[k] >= ng)
                throw Err(BSNN_ERR_OUT_OF_RANGE, "Selected neuron ID " + std::to_string(ids[k]) +
                                                     " is out of range for the neuron group.");
        if (n_ids == 0) { m.sel.resize(ng); for (uint32_t k = 0; k < ng; ++k) m.sel[k] = k; }
        else m.sel.assign(ids, ids + n_ids);
        m.vh.assign(static_cast<size_t>(ng) * m.interval, 0.0f);
        sim.mons.push_back(std::move(m));
        if (out) *out = static_cast<uint32_t>(sim.mons.size() - 1);
    });
}

BSNN_API int32_t or_set_noise_mode(or_sim* s, int32_t mode) {
    return with_sim(s, [&](auto& sim) {
        if (mode < BSNN_NOISE_PHILOX || mode > BSNN_NOISE_REPLAY) throw Err(BSNN_ERR_INVALID_ARGUMENT, "bad mode");
        sim.noise_mode = mode;
    });
}

BSNN_API int32_t or_set_noise_replay(or_sim* s, const uint8_t* counts, uint32_t n_steps) {
    return with_sim(s, [&](auto& sim) {
        sim.replay.assign(counts, counts + static_cast<size_t>(n_steps) * sim.N * 2);
        sim.replay_steps = n_steps;
        sim.noise_mode = BSNN_NOISE_REPLAY;
    });
}

BSNN_API int32_t or_step(or_sim* s, uint32_t clock) {
    return with_sim(s, [&](auto& sim) { sim.step(clock); });
}

BSNN_API int32_t or_run(or_sim* s, uint32_t first, uint32_t n) {
    return with_sim(s, [&](auto& sim) {
        for (uint32_t k = 0; k < n; ++k) sim.step(first + k);
    });
}

BSNN_API int32_t or_skip_steps(or_sim* s, uint32_t n) {
    return with_sim(s, [&](auto& sim) {
        for (uint32_t k = 0; k < n; ++k) {
            for (auto& st : sim.stims) {
                if (st.cursor_t >= st.counts.size()) continue;
                st.cursor_e += st.counts[st.cursor_t];
                ++st.cursor_t;
            }
            ++sim.steps_done;
        }
    });
}

BSNN_API int32_t or_read_state(or_sim* s, int32_t field, uint32_t index, uint32_t offset, uint32_t count, void* out) {
    return with_sim(s, [&](auto& sim) {
        if (field == BSNN_FIELD_REFRACTORY_COUNTER || field == BSNN_FIELD_SPIKES) {
            const auto& vec = field == BSNN_FIELD_SPIKES ? sim.spikes : sim.refrac;
            if (offset > sim.N || count > sim.N - offset) throw Err(BSNN_ERR_OUT_OF_RANGE, "read out of range");
            std::memcpy(out, vec.data() + offset, count * sizeof(uint32_t));
            return;
        }
        uint32_t len = 0;
        auto* vec = sim.field_vec(field, index, &len);
        if (!vec) throw Err(BSNN_ERR_INVALID_ARGUMENT, "unknown field");
        if (offset > len || count > len - offset) throw Err(BSNN_ERR_OUT_OF_RANGE, "read out of range");
        float* o = static_cast<float*>(out);
        for (uint32_t k = 0; k < count; ++k) o[k] = static_cast<float>((*vec)[offset + k]);
    });
}

BSNN_API int32_t or_read_state_f64(or_sim* s, int32_t field, uint32_t index, uint32_t offset, uint32_t count,
                                   double* out) {
    return with_sim(s, [&](auto& sim) {
        uint32_t len = 0;
        auto* vec = sim.field_vec(field, index, &len);
        if (!vec) throw Err(BSNN_ERR_INVALID_ARGUMENT, "unknown field");
        if (offset > len || count > len - offset) throw Err(BSNN_ERR_OUT_OF_RANGE, "read out of range");
        for (uint32_t k = 0; k < count; ++k) out[k] = static_cast<double>((*vec)[offset + k]);
    });
}

BSNN_API int32_t or_write_state(or_sim* s, int32_t field, uint32_t index, uint32_t offset, uint32_t count,
                                const void* in) {
    return with_sim(s, [&](auto& sim) {
        using R = typename std::decay_t<decltype(sim.v)>::value_type;
        if (field == BSNN_FIELD_REFRACTORY_COUNTER || field == BSNN_FIELD_SPIKES) {
            auto& vec = field == BSNN_FIELD_SPIKES ? sim.spikes : sim.refrac;
            if (offset > sim.N || count > sim.N - offset) throw Err(BSNN_ERR_OUT_OF_RANGE, "write out of range");
            std::memcpy(vec.data() + offset, in, count * sizeof(uint32_t));
            return;
        }
        uint32_t len = 0;
        auto* vec = sim.field_vec(field, index, &len);
        if (!vec) throw Err(BSNN_ERR_INVALID_ARGUMENT, "unknown field");
        if (offset > len || count > len - offset) throw Err(BSNN_ERR_OUT_OF_RANGE, "write out of range");
        const float* i = static_cast<const float*>(in);
        for (uint32_t k = 0; k < count; ++k) (*vec)[offset + k] = R(i[k]);
    });
}

BSNN_API int32_t or_read_weights(or_sim* s, uint32_t conn, float* out) {
    return with_sim(s, [&](auto& sim) {
        if (conn >= sim.conns.size()) throw Err(BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        const auto& w = sim.conns[conn].w;
        for (size_t k = 0; k < w.size(); ++k) out[k] = static_cast<float>(w[k]);
    });
}

BSNN_API int32_t or_write_weights(or_sim* s, uint32_t conn, const float* in) {
    return with_sim(s, [&](auto& sim) {
        using R = typename std::decay_t<decltype(sim.v)>::value_type;
        if (conn >= sim.conns.size()) throw Err(BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        auto& w = sim.conns[conn].w;
        for (size_t k = 0; k < w.size(); ++k) w[k] = R(in[k]);
    });
}

BSNN_API int32_t or_read_weights_f64(or_sim* s, uint32_t conn, double* out) {
    return with_sim(s, [&](auto& sim) {
        if (conn >= sim.conns.size()) throw Err(BSNN_ERR_OUT_OF_RANGE, "connection index out of range");
        const auto& w = sim.conns[conn].w;
        for (size_t k = 0; k < w.size(); ++k) out[k] = static_cast<double>(w[k]);
    });
}

BSNN_API int32_t or_read_spike_history(or_sim* s, uint32_t mon, uint32_t* out, int32_t flush) {
    return with_sim(s, [&](auto& sim) {
        if (mon >= sim.mons.size() || sim.mons[mon].kind != 0) throw Err(BSNN_ERR_OUT_OF_RANGE, "bad monitor");
        auto& m = sim.mons[mon];
        std::memcpy(out, m.sh.data(), m.sh.size() * sizeof(uint32_t));
        if (flush) std::fill(m.sh.begin(), m.sh.end(), 0u);
    });
}

BSNN_API int32_t or_read_voltage_history(or_sim* s, uint32_t mon, float* out, int32_t flush) {
    return with_sim(s, [&](auto& sim) {
        if (mon >= sim.mons.size() || sim.mons[mon].kind != 1) throw Err(BSNN_ERR_OUT_OF_RANGE, "bad monitor");
        auto& m = sim.mons[mon];
        // selected neurons only: out[k * interval + slot]
        for (size_t k = 0; k < m.sel.size(); ++k)
            std::memcpy(out + k * m.interval, m.vh.data() + static_cast<size_t>(m.sel[k]) * m.interval,
                        m.interval * sizeof(float));
        if (flush) std::fill(m.vh.begin(), m.vh.end(), 0.0f);
    });
}

BSNN_API int32_t or_last_noise_counts(or_sim* s, uint8_t* out) {
    return with_sim(s, [&](auto& sim) { std::memcpy(out, sim.last_counts.data(), sim.last_counts.size()); });
}

BSNN_API void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    philox4x32_10(ctr, key, out);
}

BSNN_API uint32_t or_poisson(float exp_neg_mean, uint32_t seed, uint32_t neuron, uint64_t step, uint32_t channel) {
    return poisson_knuth(exp_neg_mean, seed, neuron, step, channel);
}

BSNN_API void or_connection_propagate(float r_decay, float d_decay, float norm, uint32_t n_pre, uint32_t n_post,
                                      const float* w, float* r, float* d, float* x, float* g,
                                      const uint32_t* spikes) {
    for (uint32_t i = 0; i < n_pre; ++i) {  // kernel_connection_decay_d_traces (:22-33)
        float t = d[i] * d_decay; if (t < 1e-30f) t = 0.0f; d[i] = t;
    }
    for (uint32_t i = 0; i < n_pre; ++i) {  // kernel_connection_decay_r_traces (:8-20)
        float t = r[i] * r_decay; if (t < 1e-30f) t = 0.0f; r[i] = t;
    }
    for (uint32_t i = 0; i < n_pre; ++i) {  // kernel_connection_update_conductances_with_spikes (:35-46)
        if (spikes[i] == 1) { r[i] += norm; d[i] += norm; }
        x[i] = d[i] - r[i];
    }
    parallel_for(n_post, [&](uint32_t q) {  // cublasSgemv, alpha = beta = 1 (:79-94)
        double acc = 0.0;
        for (uint32_t i = 0; i < n_pre; ++i)
            acc += static_cast<double>(w[static_cast<size_t>(i) * n_post + q]) * static_cast<double>(x[i]);
        g[q] = static_cast<float>(acc) + g[q];
    });
}

}  // extern "C"
