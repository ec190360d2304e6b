// ref_harness.cu -- drives the reference's own CUDA implementation (TEST / BASELINE
// INFRASTRUCTURE ONLY).
//
// Linked against the reference's unmodified component objects (everything under cpp_src except
// main_buryn.cpp, compiled in place by oracle/Makefile).  It builds the components exactly as
// cpp_src/main_buryn.cpp:98-340 does, but from a network description file instead of the
// generators, so the reference and libbsnn see identical matrices and parameters.
//
//   ref_harness <net.bin> dump <steps> <out.bin> <every>
//       runs <steps> calls of System::step_the_clock and writes, for every <every>-th step (and the
//       last), the full device state; plus, for every step, the background Poisson counts the
//       reference drew (read with a copy of each neuron's curand state, so the reference's own
//       draws are unchanged).  Weights of every connection are written after the last step.
//   ref_harness <net.bin> bench <warm_steps> <samples> <steps_per_sample>
//       the bench's reference arm: times each sample of steps separately, L2 flushed between them
//   ref_harness <net.bin> time <warmup> <steps>
//       times <steps> calls of System::step_the_clock (the hot path; Monitor::record's text
//       output is not part of it) and prints one JSON line.
//   ref_harness <net.bin> record <steps> <outdir>
//       the step loop of System::run with the network's recorders (and a WeightRecorder per
//       connection) writing their text files into <outdir>, plus the Poisson counts of every step
//       in <outdir>/noise.bin, so the files can be reproduced with the noise replayed, and the
//       final weights of every connection in <outdir>/weights_final_c<c>.bin.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "buryn_definitions.h"
#include "connection.h"
#include "gpu_simulation_state.h"
#include "istdp_plasticity.h"
#include "neuron_group.h"
#include "spike_recorder.h"
#include "stdp_plasticity.h"
#include "stimulus.h"
#include "system.h"
#include "triplet_plasticity.h"
#include "voltage_recorder.h"
#include "weight_recorder.h"

namespace {

struct Reader {
    std::ifstream in;
    explicit Reader(const char* path) : in(path, std::ios::binary) {
        if (!in) throw std::runtime_error(std::string("cannot open ") + path);
    }
    template <class T>
    T get() {
        T v;
        in.read(reinterpret_cast<char*>(&v), sizeof(T));
        if (!in) throw std::runtime_error("truncated network file");
        return v;
    }
    template <class T>
    std::vector<T> vec(size_t n) {
        std::vector<T> v(n);
        if (n) in.read(reinterpret_cast<char*>(v.data()), sizeof(T) * n);
        if (!in) throw std::runtime_error("truncated network file");
        return v;
    }
};

struct GroupInfo {
    uint32_t offset, n;
    float mean_e, mean_i;
};

// Reads the counts curand_poisson is about to draw for every neuron of a group, from a copy of the
// neuron's Philox state in the same order as kernel_update_background_conductances
// (cpp_src/neuron_groups/kernel_neuron_group_evolve.cu:53-54); the stored state is not advanced.
__global__ void peek_poisson_counts(const void* states_v, uint32_t offset, uint32_t n, float mean_e, float mean_i,
                                    uint8_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    curandStatePhilox4_32_10_t st = static_cast<const curandStatePhilox4_32_10_t*>(states_v)[offset + i];
    const unsigned int ne = mean_e > 0.0f ? curand_poisson(&st, mean_e) : 0u;
    const unsigned int ni = mean_i > 0.0f ? curand_poisson(&st, mean_i) : 0u;
    out[(offset + i) * 2] = static_cast<uint8_t>(ne > 255u ? 255u : ne);
    out[(offset + i) * 2 + 1] = static_cast<uint8_t>(ni > 255u ? 255u : ni);
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
void d2h_append(std::ofstream& out, const T* dptr, size_t n) {
    std::vector<T> h(n);
    if (n) check(cudaMemcpy(h.data(), dptr, n * sizeof(T), cudaMemcpyDeviceToHost), "dump D2H");
    out.write(reinterpret_cast<const char*>(h.data()), static_cast<std::streamsize>(n * sizeof(T)));
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc < 3) {
            std::fprintf(stderr,
                         "usage: %s net.bin dump <steps> <out.bin> <every> | time <warmup> <steps> | bench <warm> <samples> <per> | "
                         "record <steps> <outdir>\n",
                         argv[0]);
            return 2;
        }
        Reader r(argv[1]);
        char magic[8];
        r.in.read(magic, 8);
        if (std::memcmp(magic, "BSNNNET1", 8) != 0) throw std::runtime_error("bad network file magic");
        const uint32_t n_e = r.get<uint32_t>(), n_i = r.get<uint32_t>(), total_steps = r.get<uint32_t>();
        const uint32_t n_events = r.get<uint32_t>(), n_plast = r.get<uint32_t>(), interval = r.get<uint32_t>();
        const int32_t seed = r.get<int32_t>();
        const float timestep = r.get<float>();
        buryn::rng_seed = seed;
        buryn::timestep = timestep;
        buryn::recording_interval_steps = interval;
        const uint32_t N = n_e + n_i;

        GpuSimulationState state(total_steps, n_e, n_i, n_events, n_plast);
        System system;

        const uint32_t n_groups = r.get<uint32_t>();
        std::vector<NeuronGroup*> groups;
        std::vector<GroupInfo> ginfo;
        for (uint32_t g = 0; g < n_groups; ++g) {
            static_assert(sizeof(NeuronGroupParams) == 88, "NeuronGroupParams layout");
            NeuronGroupParams p = r.get<NeuronGroupParams>();
            std::vector<std::vector<float>> loc(p.num_neurons, std::vector<float>{0.0f, 0.0f});
            auto ng = std::make_unique<NeuronGroup>(loc, p, state);
            groups.push_back(ng.get());
            ginfo.push_back(GroupInfo{p.offset, p.num_neurons, p.mean_background_excitatory_spikes,
                                      p.mean_background_inhibitory_spikes});
            system.add_neuron_group(std::move(ng));
        }
        const uint32_t n_conns = r.get<uint32_t>();
        std::vector<Connection*> conns;
        std::vector<uint32_t> conn_idx;
        for (uint32_t c = 0; c < n_conns; ++c) {
            const uint32_t pre = r.get<uint32_t>(), post = r.get<uint32_t>();
            static_assert(sizeof(ConnectionParams) == 20, "ConnectionParams layout");
            ConnectionParams p = r.get<ConnectionParams>();
            const uint32_t np = groups[pre]->num_neurons(), nq = groups[post]->num_neurons();
            std::vector<float> flat = r.vec<float>(static_cast<size_t>(np) * nq);
            std::vector<std::vector<float>> w(np, std::vector<float>(nq));
            for (uint32_t i = 0; i < np; ++i)
                std::memcpy(w[i].data(), &flat[static_cast<size_t>(i) * nq], sizeof(float) * nq);
            auto cn = std::make_unique<Connection>(*groups[pre], *groups[post], w, p, state);
            conns.push_back(cn.get());
            conn_idx.push_back(p.weight_matrix_idx);
            system.add_connection(std::move(cn));
        }
        const uint32_t n_counts = r.get<uint32_t>();
        std::vector<uint32_t> counts = r.vec<uint32_t>(n_counts);
        const uint32_t n_ev = r.get<uint32_t>();
        std::vector<uint32_t> ids = r.vec<uint32_t>(n_ev), offs = r.vec<uint32_t>(n_ev);
        std::vector<float> deltas = r.vec<float>(n_ev);
        if (n_counts) system.add_stimulus(std::make_unique<Stimulus>(counts, ids, offs, deltas, state));
        const uint32_t n_pl = r.get<uint32_t>();
        for (uint32_t k = 0; k < n_pl; ++k) {
            const int32_t kind = r.get<int32_t>();
            const uint32_t conn = r.get<uint32_t>();
            static_assert(sizeof(PlasticityParams) == 44, "PlasticityParams layout");
            PlasticityParams p = r.get<PlasticityParams>();
            if (kind == 1) system.add_plasticity(std::make_unique<TripletPlasticity>(*conns[conn], p, state));
            else if (kind == 2) system.add_plasticity(std::make_unique<IstdpPlasticity>(*conns[conn], p, state));
            else system.add_plasticity(std::make_unique<StdpPlasticity>(*conns[conn], p, state));
        }
        // In record mode the recorders write their real files into <outdir> (spikes_m<k>.txt,
        // voltage_m<k>.txt, weights_c<c>.txt); otherwise their output goes to /dev/null.
        const std::string mode = argv[2];
        const bool recording = mode == "record" && argc >= 5;
        const std::string outdir = recording ? std::string(argv[4]) : std::string();
        static const std::string null_path = "/dev/null";
        // VoltageRecorder keeps a reference to its path (voltage_recorder.h:40), so the strings
        // must outlive the recorders.
        std::deque<std::string> paths;
        std::vector<Monitor*> monitors;
        const uint32_t n_mons = r.get<uint32_t>();
        for (uint32_t m = 0; m < n_mons; ++m) {
            const int32_t kind = r.get<int32_t>();
            const uint32_t group = r.get<uint32_t>();
            const uint32_t n_ids = r.get<uint32_t>();
            std::vector<uint32_t> sel = r.vec<uint32_t>(n_ids);
            std::unique_ptr<Monitor> mon;
            paths.push_back(recording ? outdir + (kind == 0 ? "/spikes_m" : "/voltage_m") + std::to_string(m) + ".txt"
                                      : null_path);
            if (kind == 0)
                mon = std::make_unique<SpikeRecorder>(*groups[group], paths.back(), interval, state);
            else
                mon = std::make_unique<VoltageRecorder>(*groups[group], paths.back(), sel, interval, state);
            monitors.push_back(mon.get());
            system.add_monitor(std::move(mon));
        }
        if (recording)
            for (uint32_t c = 0; c < n_conns; ++c) {
                paths.push_back(outdir + "/weights_c" + std::to_string(c) + ".txt");
                auto mon = std::make_unique<WeightRecorder>(*conns[c], paths.back(), state);
                monitors.push_back(mon.get());
                system.add_monitor(std::move(mon));
            }

        if (recording) {
            // The loop of System::run (cpp_src/core/system.cpp:65-84) with the Poisson counts of every
            // step recorded (as in dump mode) into <outdir>/noise.bin: [steps][N][2] uint8.
            const uint32_t steps = static_cast<uint32_t>(std::atoi(argv[3]));
            uint8_t* d_counts = nullptr;
            check(cudaMalloc(&d_counts, N * 2), "cudaMalloc counts");
            check(cudaMemset(d_counts, 0, N * 2), "memset counts");
            std::vector<uint8_t> all_counts, h_counts(N * 2);
            for (uint32_t s = 0; s < steps; ++s) {
                for (const auto& g : ginfo)
                    peek_poisson_counts<<<(g.n + 255) / 256, 256>>>(state.d_neuron_rng_states(), g.offset, g.n,
                                                                    g.mean_e, g.mean_i, d_counts);
                check(cudaGetLastError(), "peek launch");
                check(cudaMemcpy(h_counts.data(), d_counts, N * 2, cudaMemcpyDeviceToHost), "counts D2H");
                all_counts.insert(all_counts.end(), h_counts.begin(), h_counts.end());
                system.step_the_clock(s);
                if (s % buryn::recording_interval_steps == 0)
                    for (Monitor* mon : monitors) mon->record(s);
            }
            check(cudaFree(d_counts), "cudaFree");
            std::ofstream nf(outdir + "/noise.bin", std::ios::binary);
            nf.write(reinterpret_cast<const char*>(all_counts.data()), static_cast<std::streamsize>(all_counts.size()));
            for (uint32_t c = 0; c < n_conns; ++c) {  // final weights, raw float32 row-major
                const std::vector<float> w = state.download_weight_matrix(conn_idx[c]);
                std::ofstream wf(outdir + "/weights_final_c" + std::to_string(c) + ".bin", std::ios::binary);
                wf.write(reinterpret_cast<const char*>(w.data()), static_cast<std::streamsize>(w.size() * sizeof(float)));
            }
            return 0;
        }
        if (mode == "bench") {
            if (argc < 6) throw std::runtime_error("bench mode needs <warm_steps> <samples> <steps_per_sample>");
            // <warm_steps> <samples> <steps_per_sample>: after the warm-up steps, times each sample of
            // consecutive steps separately (host wall clock around the reference's own synchronous
            // step calls), with a 256 MB write between samples so no sample starts from a warm L2.
            const uint32_t warm = static_cast<uint32_t>(std::atoi(argv[3]));
            const uint32_t samples = static_cast<uint32_t>(std::atoi(argv[4]));
            const uint32_t per = static_cast<uint32_t>(std::atoi(argv[5]));
            void* flush = nullptr;
            const size_t flush_bytes = size_t(256) << 20;
            check(cudaMalloc(&flush, flush_bytes), "cudaMalloc flush");
            uint32_t clock_step = 0;
            for (; clock_step < warm; ++clock_step) system.step_the_clock(clock_step);
            check(cudaDeviceSynchronize(), "sync");
            std::printf("{\"steps_per_sample\": %u, \"neurons\": %u, \"seconds\": [", per, N);
            for (uint32_t k = 0; k < samples; ++k) {
                check(cudaMemset(flush, k & 0xff, flush_bytes), "flush L2");
                check(cudaDeviceSynchronize(), "sync");
                const auto t0 = std::chrono::steady_clock::now();
                for (uint32_t s = 0; s < per; ++s) system.step_the_clock(clock_step++);
                check(cudaDeviceSynchronize(), "sync");
                const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                std::printf("%s%.6f", k ? ", " : "", sec);
            }
            std::printf("]}\n");
            cudaFree(flush);
            return 0;
        }
        if (mode == "time") {
            const uint32_t warm = static_cast<uint32_t>(std::atoi(argv[3]));
            const uint32_t steps = static_cast<uint32_t>(std::atoi(argv[4]));
            for (uint32_t s = 0; s < warm; ++s) system.step_the_clock(s);
            check(cudaDeviceSynchronize(), "sync");
            const auto t0 = std::chrono::steady_clock::now();
            for (uint32_t s = 0; s < steps; ++s) system.step_the_clock(warm + s);
            check(cudaDeviceSynchronize(), "sync");
            const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::printf("{\"steps\": %u, \"seconds\": %.6f, \"neurons\": %u}\n", steps, sec, N);
            return 0;
        }
        if (mode != "dump" || argc < 6) throw std::runtime_error("bad mode");
        const uint32_t steps = static_cast<uint32_t>(std::atoi(argv[3]));
        const uint32_t every = static_cast<uint32_t>(std::max(1, std::atoi(argv[5])));
        std::ofstream out(argv[4], std::ios::binary);
        out.write("BSNNDMP1", 8);
        out.write(reinterpret_cast<const char*>(&N), 4);
        out.write(reinterpret_cast<const char*>(&steps), 4);
        uint8_t* d_counts = nullptr;
        check(cudaMalloc(&d_counts, N * 2), "cudaMalloc counts");
        check(cudaMemset(d_counts, 0, N * 2), "memset counts");
        std::vector<uint8_t> all_counts;
        all_counts.reserve(static_cast<size_t>(steps) * N * 2);
        std::vector<uint8_t> h_counts(N * 2);
        // every step's spike vector, packed 8 neurons per byte (bit 7 first), for the raster
        const size_t row_bytes = (N + 7) / 8;
        std::vector<uint8_t> raster(static_cast<size_t>(steps) * row_bytes, 0);
        std::vector<uint32_t> h_spikes(N);
        for (uint32_t s = 0; s < steps; ++s) {
            for (const auto& g : ginfo) {
                peek_poisson_counts<<<(g.n + 255) / 256, 256>>>(state.d_neuron_rng_states(), g.offset, g.n, g.mean_e,
                                                                g.mean_i, d_counts);
            }
            check(cudaGetLastError(), "peek launch");
            check(cudaMemcpy(h_counts.data(), d_counts, N * 2, cudaMemcpyDeviceToHost), "counts D2H");
            all_counts.insert(all_counts.end(), h_counts.begin(), h_counts.end());
            system.step_the_clock(s);
            check(cudaMemcpy(h_spikes.data(), state.d_spikes(), N * sizeof(uint32_t), cudaMemcpyDeviceToHost),
                  "spikes D2H");
            for (uint32_t j = 0; j < N; ++j)
                if (h_spikes[j]) raster[static_cast<size_t>(s) * row_bytes + j / 8] |= static_cast<uint8_t>(0x80u >> (j % 8));
            if ((s + 1) % every == 0 || s + 1 == steps) {
                const uint32_t tag = s;
                out.write("STEP", 4);
                out.write(reinterpret_cast<const char*>(&tag), 4);
                d2h_append(out, state.d_membrane_potentials(), N);
                d2h_append(out, state.d_g_excitatory(), N);
                d2h_append(out, state.d_g_inhibitory(), N);
                d2h_append(out, state.d_i_stimulus(), N);
                d2h_append(out, state.d_refractory_counter(), N);
                d2h_append(out, state.d_spikes(), N);
                d2h_append(out, state.d_background_g_excitatory_synaptic_conductances(), N);
                d2h_append(out, state.d_background_g_inhibitory_synaptic_conductances(), N);
                d2h_append(out, state.d_background_excitatory_postsynaptic_r_traces(), N);
                d2h_append(out, state.d_background_excitatory_postsynaptic_d_traces(), N);
                d2h_append(out, state.d_background_inhibitory_postsynaptic_r_traces(), N);
                d2h_append(out, state.d_background_inhibitory_postsynaptic_d_traces(), N);
                // x = d - r per connection, in weight-matrix-index order (ee, ei, ie, ii)
                d2h_append(out, state.d_ee_summed_postsynaptic_conductances(), n_e);
                d2h_append(out, state.d_ei_summed_postsynaptic_conductances(), n_e);
                d2h_append(out, state.d_ie_summed_postsynaptic_conductances(), n_i);
                d2h_append(out, state.d_ii_summed_postsynaptic_conductances(), n_i);
                d2h_append(out, state.d_pre_traces(), static_cast<size_t>(n_plast) * N);
                d2h_append(out, state.d_post_traces(), static_cast<size_t>(n_plast) * N);
            }
        }
        out.write("WGTS", 4);
        for (uint32_t c = 0; c < n_conns; ++c) {
            std::vector<float> w = state.download_weight_matrix(conn_idx[c]);
            const uint32_t n = static_cast<uint32_t>(w.size());
            out.write(reinterpret_cast<const char*>(&n), 4);
            out.write(reinterpret_cast<const char*>(w.data()), static_cast<std::streamsize>(w.size() * sizeof(float)));
        }
        out.write("NOIS", 4);
        out.write(reinterpret_cast<const char*>(all_counts.data()), static_cast<std::streamsize>(all_counts.size()));
        out.write("SPKS", 4);
        out.write(reinterpret_cast<const char*>(raster.data()), static_cast<std::streamsize>(raster.size()));
        check(cudaFree(d_counts), "cudaFree");
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_harness: %s\n", e.what());
        return 1;
    }
}
