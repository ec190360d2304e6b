// bsnn.hpp -- C++17 component facade over the C-ABI of bsnn.h.
//
// The reference builds a simulation from components that share one GpuSimulationState
// (cpp_src/main_buryn.cpp:109-343): NeuronGroup, Connection, Stimulus, the plasticities and the
// monitors are constructed against the state, moved into a System, and System::run steps it.
// This header offers the same classes, constructor signatures, parameter PODs (with the same
// default member values) and exception types, so code written against the reference compiles
// against libbsnn with `#include "bsnn.hpp"` and `using namespace bsnn;`.  Every constructor
// records its component in the library at once, as the reference uploads at construction;
// System::step_the_clock / System::run advance the fused sm_100a kernel.
//
// Differences a caller can see:
//  * Monitor::record / Monitor::historicize do nothing on their own: System records every
//    monitor at the reference's cadence (bsnn_record), and historicizing happens inside the step.
//  * Components must all be constructed before the first step (the library plans the kernel's
//    work then); constructing one later throws std::runtime_error.
#pragma once

#include <chrono>
#include <cstdint>
#include <functional>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "bsnn.h"

namespace bsnn {

// The reference's globals (cpp_src/core/buryn_definitions.h:11-13), read when a
// GpuSimulationState is constructed.
namespace buryn {
inline int rng_seed = 314;
inline float timestep = 1e-4f;
inline uint32_t recording_interval_steps = 10000;
}  // namespace buryn

// Status codes back to the exception types the reference throws (cuda_utils.h:10-20).
inline void check(bsnn_status st, const bsnn_sim* sim) {
    if (st == BSNN_OK) return;
    const std::string msg = bsnn_last_error(sim);
    if (st == BSNN_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    if (st == BSNN_ERR_OUT_OF_RANGE) throw std::out_of_range(msg);
    throw std::runtime_error(msg);
}

// cpp_src/neuron_groups/neuron_group_params.h:7-31, with its defaults.
struct NeuronGroupParams : bsnn_neuron_group_params {
    NeuronGroupParams() : bsnn_neuron_group_params{} {
        timestep = 1e-4f;
        g_leak = 10.0f;
        membrane_capacitance = 0.1f;
        depolarization_slope_factor = 2.0f;
        v_effective_spike_threshold = -50.0f;
        v_excitatory_reversal = 0.0f;
        v_inhibitory_reversal = -80.0f;
        v_threshold = -45.0f;
        v_reset = -55.0f;
        v_rest = -65.0f;
    }
};

// cpp_src/connections/connection_params.h:7-14 (all defaults zero).
struct ConnectionParams : bsnn_connection_params {
    ConnectionParams() : bsnn_connection_params{} {}
};

// cpp_src/plasticities/plasticity_params.h:7-20 (weight_max defaults to 1).
struct PlasticityParams : bsnn_plasticity_params {
    PlasticityParams() : bsnn_plasticity_params{} { weight_max = 1.0f; }
};

// cpp_src/gpu_core/gpu_simulation_state.h:19-30: owns the simulation (one bsnn_sim).
class GpuSimulationState {
public:
    explicit GpuSimulationState(uint32_t total_simulation_length, uint32_t num_excitatory_neurons,
                                uint32_t num_inhibitory_neurons, uint32_t num_stimulus_events,
                                uint32_t num_plasticities, int device = 0) {
        const bsnn_state_desc d{total_simulation_length, num_excitatory_neurons, num_inhibitory_neurons,
                                num_stimulus_events,     num_plasticities,       buryn::recording_interval_steps,
                                buryn::rng_seed,         device};
        check(bsnn_create(&d, &sim_), nullptr);
        desc_ = d;
    }
    ~GpuSimulationState() { bsnn_destroy(sim_); }
    GpuSimulationState(const GpuSimulationState&) = delete;
    GpuSimulationState& operator=(const GpuSimulationState&) = delete;

    bsnn_sim* handle() const { return sim_; }
    uint32_t total_simulation_length() const { return desc_.total_simulation_length; }
    uint32_t num_excitatory_neurons() const { return desc_.num_excitatory_neurons; }
    uint32_t num_inhibitory_neurons() const { return desc_.num_inhibitory_neurons; }
    uint32_t total_neurons() const { return desc_.num_excitatory_neurons + desc_.num_inhibitory_neurons; }
    uint32_t num_stimulus_events() const { return desc_.num_stimulus_events; }
    uint32_t num_plasticities() const { return desc_.num_plasticities; }
    uint32_t recording_interval_steps() const { return desc_.recording_interval_steps; }
    uint64_t total_allocated_bytes() const {
        bsnn_info info{};
        check(bsnn_get_info(sim_, &info), sim_);
        return info.device_bytes;
    }
    // GpuSimulationState::memory_report (gpu_simulation_state.cu:357-362).  bsnn allocates once the
    // network is complete, so call it after the components are added.
    std::string memory_report() const {
        char buf[256];
        check(bsnn_memory_report(sim_, buf, sizeof(buf)), sim_);
        return std::string(buf);
    }
    // GpuSimulationState::download_weight_matrix (gpu_simulation_state.cu:287-306), by the
    // ConnectionParams::weight_matrix_idx of the connection.
    std::vector<float> download_weight_matrix(uint32_t weight_matrix_idx) const {
        for (const auto& c : conns_)
            if (c.idx == weight_matrix_idx) {
                std::vector<float> w(static_cast<size_t>(c.n_pre) * c.n_post);
                check(bsnn_read_weights(sim_, c.conn, w.data()), sim_);
                return w;
            }
        throw std::invalid_argument("Unknown weight matrix index: " + std::to_string(weight_matrix_idx));
    }
    // A per-neuron field (BSNN_FIELD_*) of the whole network.
    std::vector<float> download_field(int32_t field) const {
        std::vector<float> out(total_neurons());
        check(bsnn_read_state(sim_, field, 0, 0, total_neurons(), out.data()), sim_);
        return out;
    }

    // bookkeeping for download_weight_matrix
    struct ConnInfo {
        uint32_t conn, idx, n_pre, n_post;
    };
    void note_connection(const ConnInfo& c) { conns_.push_back(c); }

private:
    bsnn_sim* sim_ = nullptr;
    bsnn_state_desc desc_{};
    std::vector<ConnInfo> conns_;
};

// cpp_src/neuron_groups/neuron_group.h:18-35.
class NeuronGroup {
public:
    explicit NeuronGroup(std::vector<std::vector<float>> neuron_locations, NeuronGroupParams params,
                         GpuSimulationState& gpu_state)
        : locations_(std::move(neuron_locations)), params_(params), state_(gpu_state) {
        check(bsnn_add_neuron_group(state_.handle(), &params_, &index_), state_.handle());
    }
    virtual ~NeuronGroup() = default;
    const std::vector<std::vector<float>>& neuron_locations() const { return locations_; }
    bool is_inhibitory() const { return params_.is_inhibitory; }
    uint32_t num_neurons() const { return params_.num_neurons; }
    uint32_t offset() const { return params_.offset; }
    uint32_t index() const { return index_; }
    GpuSimulationState& state() const { return state_; }
    void evolve() {}  // done by the fused step kernel

private:
    std::vector<std::vector<float>> locations_;
    NeuronGroupParams params_;
    GpuSimulationState& state_;
    uint32_t index_ = 0;
};

// cpp_src/connections/connection.h:24-46: `weight_matrix` is [pre][post].
class Connection {
public:
    Connection(NeuronGroup& pre_group, NeuronGroup& post_group, std::vector<std::vector<float>>& weight_matrix,
               ConnectionParams params, GpuSimulationState& gpu_state)
        : params_(params), state_(gpu_state), pre_offset_(pre_group.offset()), post_offset_(post_group.offset()),
          n_pre_(pre_group.num_neurons()), n_post_(post_group.num_neurons()) {
        if (weight_matrix.size() != n_pre_) throw std::invalid_argument("weight matrix rows != presynaptic neurons");
        std::vector<float> flat(static_cast<size_t>(n_pre_) * n_post_);
        for (uint32_t i = 0; i < n_pre_; ++i) {
            if (weight_matrix[i].size() != n_post_)
                throw std::invalid_argument("weight matrix columns != postsynaptic neurons");
            std::copy(weight_matrix[i].begin(), weight_matrix[i].end(), flat.begin() + static_cast<size_t>(i) * n_post_);
        }
        check(bsnn_add_connection(state_.handle(), pre_group.index(), post_group.index(), flat.data(), &params_, &index_),
              state_.handle());
        state_.note_connection({index_, params_.weight_matrix_idx, n_pre_, n_post_});
    }
    virtual ~Connection() = default;
    uint32_t weight_matrix_idx() const { return params_.weight_matrix_idx; }
    uint32_t pre_group_offset() const { return pre_offset_; }
    uint32_t post_group_offset() const { return post_offset_; }
    uint32_t pre_group_num_neurons() const { return n_pre_; }
    uint32_t post_group_num_neurons() const { return n_post_; }
    uint32_t index() const { return index_; }
    GpuSimulationState& state() const { return state_; }
    void propagate() {}  // done by the fused step kernel

private:
    ConnectionParams params_;
    GpuSimulationState& state_;
    uint32_t pre_offset_, post_offset_, n_pre_, n_post_, index_ = 0;
};

// cpp_src/stimuli/stimulus.h:20-30.
class Stimulus {
public:
    Stimulus(std::vector<uint32_t> timestep_event_count, std::vector<uint32_t> stimulus_event_neuron_ids,
             std::vector<uint32_t> stimulus_event_post_group_offsets, std::vector<float> stimulus_event_amplitude_changes,
             GpuSimulationState& gpu_state) {
        if (stimulus_event_neuron_ids.size() != stimulus_event_post_group_offsets.size() ||
            stimulus_event_neuron_ids.size() != stimulus_event_amplitude_changes.size())
            throw std::invalid_argument("stimulus event arrays differ in length");
        check(bsnn_add_stimulus(gpu_state.handle(), timestep_event_count.data(),
                                static_cast<uint32_t>(timestep_event_count.size()), stimulus_event_neuron_ids.data(),
                                stimulus_event_post_group_offsets.data(), stimulus_event_amplitude_changes.data(),
                                static_cast<uint32_t>(stimulus_event_neuron_ids.size())),
              gpu_state.handle());
    }
    virtual ~Stimulus() = default;
    void apply() {}  // done by the fused step kernel
};

// cpp_src/plasticities/plasticity.h:10-26 and its three rules.
class Plasticity {
public:
    Plasticity(Connection& connection, PlasticityParams params, GpuSimulationState& gpu_state, int32_t kind) {
        check(bsnn_add_plasticity(gpu_state.handle(), kind, connection.index(), &params, &index_), gpu_state.handle());
    }
    virtual ~Plasticity() = default;
    virtual void update() {}  // done by the fused step kernel
    uint32_t index() const { return index_; }

private:
    uint32_t index_ = 0;
};
class TripletPlasticity : public Plasticity {
public:
    TripletPlasticity(Connection& connection, PlasticityParams params, GpuSimulationState& gpu_state)
        : Plasticity(connection, params, gpu_state, BSNN_PLASTICITY_TRIPLET) {}
};
class IstdpPlasticity : public Plasticity {
public:
    IstdpPlasticity(Connection& connection, PlasticityParams params, GpuSimulationState& gpu_state)
        : Plasticity(connection, params, gpu_state, BSNN_PLASTICITY_ISTDP) {}
};
class StdpPlasticity : public Plasticity {
public:
    StdpPlasticity(Connection& connection, PlasticityParams params, GpuSimulationState& gpu_state)
        : Plasticity(connection, params, gpu_state, BSNN_PLASTICITY_STDP) {}
};

// cpp_src/monitors/monitor.h and the three recorders.
class Monitor {
public:
    explicit Monitor(GpuSimulationState& gpu_state) : state_(gpu_state) {}
    virtual ~Monitor() = default;
    virtual void record(uint32_t) {}       // System records every monitor at once (bsnn_record)
    virtual void historicize(uint32_t) {}  // done inside the step

protected:
    GpuSimulationState& state_;
};
class SpikeRecorder : public Monitor {
public:
    SpikeRecorder(const NeuronGroup& group, const std::string& output_filepath, uint32_t recording_interval_steps,
                  GpuSimulationState& gpu_state)
        : Monitor(gpu_state) {
        check(bsnn_add_spike_recorder(state_.handle(), group.index(), recording_interval_steps, &index_),
              state_.handle());
        check(bsnn_set_monitor_output(state_.handle(), index_, output_filepath.c_str()), state_.handle());
    }
    uint32_t index() const { return index_; }

private:
    uint32_t index_ = 0;
};
class VoltageRecorder : public Monitor {
public:
    VoltageRecorder(const NeuronGroup& group, const std::string& output_filepath,
                    std::vector<uint32_t> selected_neurons, uint32_t recording_interval_steps,
                    GpuSimulationState& gpu_state)
        : Monitor(gpu_state) {
        check(bsnn_add_voltage_recorder(state_.handle(), group.index(), selected_neurons.data(),
                                        static_cast<uint32_t>(selected_neurons.size()), recording_interval_steps,
                                        &index_),
              state_.handle());
        check(bsnn_set_monitor_output(state_.handle(), index_, output_filepath.c_str()), state_.handle());
    }
    uint32_t index() const { return index_; }

private:
    uint32_t index_ = 0;
};
class WeightRecorder : public Monitor {
public:
    WeightRecorder(const Connection& connection, const std::string& output_filepath, GpuSimulationState& gpu_state)
        : Monitor(gpu_state) {
        check(bsnn_add_weight_recorder(state_.handle(), connection.index(), output_filepath.c_str()), state_.handle());
    }
};

// cpp_src/core/system.h:16-35.
class System {
public:
    void add_neuron_group(std::unique_ptr<NeuronGroup> neuron_group) {
        bind(neuron_group->state());
        groups_.push_back(std::move(neuron_group));
    }
    void add_connection(std::unique_ptr<Connection> connection) {
        bind(connection->state());
        conns_.push_back(std::move(connection));
    }
    void add_stimulus(std::unique_ptr<Stimulus> stimulus) { stimuli_.push_back(std::move(stimulus)); }
    void add_plasticity(std::unique_ptr<Plasticity> plasticity) { plasticities_.push_back(std::move(plasticity)); }
    void add_monitor(std::unique_ptr<Monitor> monitor) { monitors_.push_back(std::move(monitor)); }
    void add_step_callback(std::function<void(uint32_t)> callback) { callbacks_.push_back(std::move(callback)); }

    // System::step_the_clock (system.cpp:43-63): every phase, one persistent-kernel step.
    void step_the_clock(uint32_t clock_step) { check(bsnn_step(sim(), clock_step), sim()); }

    // System::run (system.cpp:65-84): callbacks before each step, Monitor::record after every step
    // that is a multiple of the recording interval.  Without callbacks the steps between records
    // run as batched persistent launches.
    // Prints the reference's progress line after each record, as System::run does.
    void run(uint32_t total_clock_steps) {
        if (callbacks_.empty()) {
            check(bsnn_set_progress_output(sim(), 1), sim());
            check(bsnn_run_system(sim(), total_clock_steps), sim());
        } else {
            const uint32_t interval = state_->recording_interval_steps();
            const auto start_time = std::chrono::steady_clock::now();
            for (uint32_t s = 0; s < total_clock_steps; ++s) {
                for (auto& cb : callbacks_) cb(s);
                step_the_clock(s);
                if (s % interval == 0) {
                    check(bsnn_record(sim(), s), sim());
                    const std::chrono::duration<float> elapsed = std::chrono::steady_clock::now() - start_time;
                    std::cout << "Completed clock step: " << s << " | elapsed: " << elapsed.count() << "s\n";
                }
            }
        }
        check(bsnn_flush_records(sim()), sim());
    }

private:
    void bind(GpuSimulationState& state) {
        if (state_ && state_ != &state) throw std::invalid_argument("components of one System must share one state");
        state_ = &state;
    }
    bsnn_sim* sim() const {
        if (!state_) throw std::runtime_error("System has no neuron group");
        return state_->handle();
    }
    GpuSimulationState* state_ = nullptr;
    std::vector<std::unique_ptr<NeuronGroup>> groups_;
    std::vector<std::unique_ptr<Connection>> conns_;
    std::vector<std::unique_ptr<Stimulus>> stimuli_;
    std::vector<std::unique_ptr<Plasticity>> plasticities_;
    std::vector<std::unique_ptr<Monitor>> monitors_;
    std::vector<std::function<void(uint32_t)>> callbacks_;
};

}  // namespace bsnn
