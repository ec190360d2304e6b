// facade_run.cpp -- builds a network through the C++ component facade (include/bsnn.hpp) the way
// the reference's main does (NeuronGroup, Connection, Stimulus, plasticities and recorders against
// one GpuSimulationState, moved into a System), then System::run.  Test program for
// tests/test_cpp_facade.py.
//
//   facade_run <net.bin> <steps> <outdir> [callbacks]
//
// <net.bin> is the network description tests write with oracle/refnet.py (magic "BSNNNET1").
// Recorder files go to <outdir> (spikes_m<k>.txt, voltage_m<k>.txt); the final membrane
// potentials to <outdir>/v.bin.  With "callbacks" a step callback is added, so System::run takes
// its per-step path; it counts the calls.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "bsnn.hpp"

namespace {

struct Reader {
    std::ifstream in;
    explicit Reader(const char* path) : in(path, std::ios::binary) {
        if (!in) throw std::runtime_error("cannot open network file");
    }
    template <class T>
    T get() {
        T v{};
        in.read(reinterpret_cast<char*>(&v), sizeof(T));
        if (!in) throw std::runtime_error("truncated network file");
        return v;
    }
    template <class T>
    std::vector<T> vec(size_t n) {
        std::vector<T> v(n);
        if (n) in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(n * sizeof(T)));
        if (!in) throw std::runtime_error("truncated network file");
        return v;
    }
};

}  // namespace

int main(int argc, char** argv) {
    using namespace bsnn;
    try {
        if (argc < 4) {
            std::fprintf(stderr, "usage: %s net.bin steps outdir [callbacks]\n", argv[0]);
            return 2;
        }
        Reader r(argv[1]);
        char magic[8];
        r.in.read(magic, 8);
        if (std::memcmp(magic, "BSNNNET1", 8) != 0) throw std::runtime_error("bad network file magic");
        const uint32_t n_e = r.get<uint32_t>(), n_i = r.get<uint32_t>(), total = r.get<uint32_t>();
        const uint32_t n_events = r.get<uint32_t>(), n_plast = r.get<uint32_t>(), interval = r.get<uint32_t>();
        buryn::rng_seed = r.get<int32_t>();
        buryn::timestep = r.get<float>();
        buryn::recording_interval_steps = interval;
        const std::string outdir = argv[3];

        GpuSimulationState state(total, n_e, n_i, n_events, n_plast);
        System system;
        std::vector<NeuronGroup*> groups;
        const uint32_t n_groups = r.get<uint32_t>();
        for (uint32_t g = 0; g < n_groups; ++g) {
            NeuronGroupParams p;
            static_cast<bsnn_neuron_group_params&>(p) = r.get<bsnn_neuron_group_params>();
            std::vector<std::vector<float>> loc(p.num_neurons, std::vector<float>{0.0f, 0.0f});
            auto ng = std::make_unique<NeuronGroup>(loc, p, state);
            groups.push_back(ng.get());
            system.add_neuron_group(std::move(ng));
        }
        std::vector<Connection*> conns;
        const uint32_t n_conns = r.get<uint32_t>();
        for (uint32_t c = 0; c < n_conns; ++c) {
            const uint32_t pre = r.get<uint32_t>(), post = r.get<uint32_t>();
            ConnectionParams p;
            static_cast<bsnn_connection_params&>(p) = r.get<bsnn_connection_params>();
            const uint32_t np = groups[pre]->num_neurons(), nq = groups[post]->num_neurons();
            const std::vector<float> flat = r.vec<float>(static_cast<size_t>(np) * nq);
            std::vector<std::vector<float>> w(np);
            for (uint32_t i = 0; i < np; ++i)
                w[i].assign(flat.begin() + static_cast<size_t>(i) * nq, flat.begin() + static_cast<size_t>(i + 1) * nq);
            auto cn = std::make_unique<Connection>(*groups[pre], *groups[post], w, p, state);
            conns.push_back(cn.get());
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
            PlasticityParams p;
            static_cast<bsnn_plasticity_params&>(p) = r.get<bsnn_plasticity_params>();
            if (kind == BSNN_PLASTICITY_TRIPLET) system.add_plasticity(std::make_unique<TripletPlasticity>(*conns[conn], p, state));
            else if (kind == BSNN_PLASTICITY_ISTDP) system.add_plasticity(std::make_unique<IstdpPlasticity>(*conns[conn], p, state));
            else system.add_plasticity(std::make_unique<StdpPlasticity>(*conns[conn], p, state));
        }
        const uint32_t n_mons = r.get<uint32_t>();
        for (uint32_t m = 0; m < n_mons; ++m) {
            const int32_t kind = r.get<int32_t>();
            const uint32_t group = r.get<uint32_t>();
            std::vector<uint32_t> sel = r.vec<uint32_t>(r.get<uint32_t>());
            if (kind == 0)
                system.add_monitor(std::make_unique<SpikeRecorder>(
                    *groups[group], outdir + "/spikes_m" + std::to_string(m) + ".txt", interval, state));
            else
                system.add_monitor(std::make_unique<VoltageRecorder>(
                    *groups[group], outdir + "/voltage_m" + std::to_string(m) + ".txt", sel, interval, state));
        }
        uint32_t calls = 0;
        if (argc > 4 && std::string(argv[4]) == "callbacks") system.add_step_callback([&calls](uint32_t) { ++calls; });

        system.run(static_cast<uint32_t>(std::atoi(argv[2])));

        const std::vector<float> v = state.download_field(BSNN_FIELD_MEMBRANE_POTENTIALS);
        std::ofstream vf(outdir + "/v.bin", std::ios::binary);
        vf.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(float)));
        std::printf("{\"callbacks\": %u, \"weights_ee\": %zu}\n", calls, state.download_weight_matrix(0).size());
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "facade_run: %s\n", e.what());
        return 1;
    }
}
