// bsnn_main.cpp -- the reference's command-line driver (cpp_src/main_buryn.cpp) on libbsnn: one
// JSON run configuration in, the same output directory out (description, config copy, locations,
// weight files, stimulus schedules, spike / voltage / weight recordings).
//
//   bsnn_main [CONFIG]                      run (CONFIG defaults to config.json, as the reference)
//   bsnn_main --weight-format F CONFIG      run with a weight storage form (f32, f32_rowscaled,
//                                           bf16, fp8_e4m3; default f32 = the reference's arithmetic)
//   bsnn_main --print-config CONFIG         print the resolved configuration, one field per line
//   bsnn_main --generate-only CONFIG        prepare the output directory and generate the network
//                                           files, without a GPU
//
// The wiring is main_buryn.cpp:98-343's: groups E (offset 0) and I, connections E->E, E->I,
// I->E, I->I (weight_matrix_idx 0-3), one stimulus, triplet plasticity on E->E and iSTDP on I->E
// when enabled (decays exp(-dt / tau) in float, parameters validated as main_buryn.cpp:76-96),
// spike recorders on E and I, a voltage recorder on E and a weight recorder on E->E.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "../../include/bsnn.hpp"
#include "../../include/bsnn_config.hpp"
#include "../../include/bsnn_config_print.hpp"
#include "../../include/bsnn_generate.hpp"

namespace {

// main_buryn.cpp:31-74: empty the output directory (or create it), write description.txt,
// create the sub-directories and copy the config file in.
void clean_up(const std::string& output_directory, const std::string& description, const std::string& config_path) {
    const std::filesystem::path dir = output_directory;
    if (std::filesystem::exists(dir) && std::filesystem::is_directory(dir)) {
        for (const auto& entry : std::filesystem::directory_iterator(dir)) std::filesystem::remove_all(entry.path());
    } else {
        std::filesystem::create_directory(dir);
    }
    std::ofstream d(dir / "description.txt");
    if (!d) throw std::runtime_error("Failed to write description file in output directory");
    d << description;
    for (const char* sub : {"stimulus_schedules", "recordings", "locations", "videos", "weights", "plots"})
        std::filesystem::create_directory(dir / sub);
    const std::filesystem::path cfg(config_path);
    if (!std::filesystem::exists(cfg)) throw std::runtime_error("Config file does not exist: " + config_path);
    std::filesystem::copy_file(cfg, dir / cfg.filename(), std::filesystem::copy_options::overwrite_existing);
}

// main_buryn.cpp:76-96.
void validate_plasticity_params(const bsnn::PlasticityParams& p, bool triplet, const std::string& name) {
    if (p.pre_trace_decay < 0.0f || p.pre_trace_decay > 1.0f) throw std::runtime_error(name + ": pre_trace_decay must be in [0, 1]");
    if (p.post_trace_decay < 0.0f || p.post_trace_decay > 1.0f)
        throw std::runtime_error(name + ": post_trace_decay must be in [0, 1]");
    if (triplet) {
        if (p.triplet_pre_trace_decay < 0.0f || p.triplet_pre_trace_decay > 1.0f)
            throw std::runtime_error(name + ": triplet_pre_trace_decay must be in [0, 1]");
        if (p.triplet_post_trace_decay < 0.0f || p.triplet_post_trace_decay > 1.0f)
            throw std::runtime_error(name + ": triplet_post_trace_decay must be in [0, 1]");
    }
    if (p.weight_min > p.weight_max) throw std::runtime_error(name + ": weight_min must be <= weight_max");
}

struct Network {
    std::vector<std::vector<float>> loc_e, loc_i;
    std::vector<std::vector<float>> w_ee, w_ei, w_ie, w_ii;
    bsnn::generate::StimulusSchedule stim;
};

Network generate_network(const bsnn::Config& c) {
    Network n;
    std::cout << "Generating neuron locations...\n";
    n.loc_e = bsnn::generate::grid_locations(c.excitatory_locations_file, c.num_excitatory_neurons,
                                             c.excitatory_location_spacing, c.excitatory_side_points,
                                             c.excitatory_side_points);
    n.loc_i = bsnn::generate::grid_locations(c.inhibitory_locations_file, c.num_inhibitory_neurons,
                                             c.inhibitory_location_spacing, c.inhibitory_side_points,
                                             c.inhibitory_side_points);
    std::cout << "Generating weight files...\n";
    n.w_ee = bsnn::generate::distance_weights(c.weights_e_to_e_filename, n.loc_e, n.loc_e, c.weight_generation_params_e_to_e, c.rng_seed);
    n.w_ei = bsnn::generate::distance_weights(c.weights_e_to_i_filename, n.loc_e, n.loc_i, c.weight_generation_params_e_to_i, c.rng_seed);
    n.w_ie = bsnn::generate::distance_weights(c.weights_i_to_e_filename, n.loc_i, n.loc_e, c.weight_generation_params_i_to_e, c.rng_seed);
    n.w_ii = bsnn::generate::distance_weights(c.weights_i_to_i_filename, n.loc_i, n.loc_i, c.weight_generation_params_i_to_i, c.rng_seed);
    std::cout << "Generating stimulus schedules...\n";
    n.stim = bsnn::generate::square_waves(c.stimulus_schedules_folder, c.simulation_steps, c.stimulus_selected_input_ids,
                                          c.stimulus_selected_input_post_group_offsets, c.stimulus_start_clock_steps,
                                          c.stimulus_end_clock_steps, c.stimulus_input_values);
    return n;
}

bsnn::NeuronGroupParams group_params(const bsnn::Config& c, bool inhibitory) {
    bsnn::NeuronGroupParams g;
    g.timestep = bsnn::buryn::timestep;
    g.g_leak = c.g_leak;
    g.membrane_capacitance = c.membrane_capacitance;
    g.depolarization_slope_factor = c.depolarization_slope_factor;
    g.v_effective_spike_threshold = c.v_effective_spike_threshold;
    g.v_excitatory_reversal = c.v_excitatory_reversal;
    g.v_inhibitory_reversal = c.v_inhibitory_reversal;
    g.v_threshold = c.v_threshold;
    g.v_reset = c.v_reset;
    g.v_rest = c.v_rest;
    g.refractory_steps = c.refractory_steps;
    g.offset = inhibitory ? c.num_excitatory_neurons : 0u;
    g.num_neurons = inhibitory ? c.num_inhibitory_neurons : c.num_excitatory_neurons;
    g.is_inhibitory = inhibitory;
    if (!inhibitory) {
        g.mean_background_excitatory_spikes = c.group_e_mean_background_excitatory_spikes;
        g.mean_background_inhibitory_spikes = c.group_e_mean_background_inhibitory_spikes;
        g.background_excitatory_postsynaptic_r_trace_decay = c.group_e_background_excitatory_postsynaptic_r_trace_decay;
        g.background_excitatory_postsynaptic_d_trace_decay = c.group_e_background_excitatory_postsynaptic_d_trace_decay;
        g.background_inhibitory_postsynaptic_r_trace_decay = c.group_e_background_inhibitory_postsynaptic_r_trace_decay;
        g.background_inhibitory_postsynaptic_d_trace_decay = c.group_e_background_inhibitory_postsynaptic_d_trace_decay;
        g.background_excitatory_scaling_factor = c.group_e_background_excitatory_scaling_factor;
        g.background_inhibitory_scaling_factor = c.group_e_background_inhibitory_scaling_factor;
    } else {
        g.mean_background_excitatory_spikes = c.group_i_mean_background_excitatory_spikes;
        g.mean_background_inhibitory_spikes = c.group_i_mean_background_inhibitory_spikes;
        g.background_excitatory_postsynaptic_r_trace_decay = c.group_i_background_excitatory_postsynaptic_r_trace_decay;
        g.background_excitatory_postsynaptic_d_trace_decay = c.group_i_background_excitatory_postsynaptic_d_trace_decay;
        g.background_inhibitory_postsynaptic_r_trace_decay = c.group_i_background_inhibitory_postsynaptic_r_trace_decay;
        g.background_inhibitory_postsynaptic_d_trace_decay = c.group_i_background_inhibitory_postsynaptic_d_trace_decay;
        g.background_excitatory_scaling_factor = c.group_i_background_excitatory_scaling_factor;
        g.background_inhibitory_scaling_factor = c.group_i_background_inhibitory_scaling_factor;
    }
    return g;
}

bsnn::ConnectionParams connection_params(const bsnn::Config& c, bool inhibitory_pre, uint32_t idx) {
    bsnn::ConnectionParams p;
    p.timestep = bsnn::buryn::timestep;
    p.decay_time = inhibitory_pre ? c.tau_decay_i : c.tau_decay_e;
    p.rise_time = inhibitory_pre ? c.tau_rise_i : c.tau_rise_e;
    p.postsynaptic_kernel_normalization_value = c.postsynaptic_kernel_normalization_value;
    p.weight_matrix_idx = idx;
    return p;
}

int32_t weight_format_of(const std::string& f) {
    if (f == "f32") return BSNN_WEIGHTS_F32;
    if (f == "f32_rowscaled") return BSNN_WEIGHTS_F32_ROWSCALED;
    if (f == "bf16") return BSNN_WEIGHTS_BF16;
    if (f == "fp8_e4m3") return BSNN_WEIGHTS_FP8_E4M3;
    throw std::invalid_argument("unknown weight format: " + f);
}

int run(const bsnn::Config& cfg, const std::string& config_path, int32_t weight_format) {
    clean_up(cfg.output_directory, cfg.description, config_path);
    bsnn::buryn::rng_seed = cfg.rng_seed;
    bsnn::buryn::timestep = cfg.timestep;
    const uint32_t n_plast = static_cast<uint32_t>(cfg.e_e_plasticity_enabled) + static_cast<uint32_t>(cfg.i_e_plasticity_enabled);
    bsnn::GpuSimulationState state(cfg.simulation_steps, cfg.num_excitatory_neurons, cfg.num_inhibitory_neurons,
                                   static_cast<uint32_t>(cfg.stimulus_selected_input_ids.size() *
                                                         cfg.stimulus_start_clock_steps.size() * 2),
                                   n_plast);
    if (weight_format != BSNN_WEIGHTS_F32) bsnn::check(bsnn_set_weight_format(state.handle(), weight_format), state.handle());
    std::cout << std::ceil((5.0 * cfg.tau_decay_e) / bsnn::buryn::timestep) << "\n";
    Network net = generate_network(cfg);

    bsnn::System system;
    auto ge = std::make_unique<bsnn::NeuronGroup>(net.loc_e, group_params(cfg, false), state);
    auto gi = std::make_unique<bsnn::NeuronGroup>(net.loc_i, group_params(cfg, true), state);
    bsnn::NeuronGroup& e = *ge;
    bsnn::NeuronGroup& i = *gi;
    system.add_neuron_group(std::move(ge));
    system.add_neuron_group(std::move(gi));
    auto cee = std::make_unique<bsnn::Connection>(e, e, net.w_ee, connection_params(cfg, false, 0), state);
    auto cei = std::make_unique<bsnn::Connection>(e, i, net.w_ei, connection_params(cfg, false, 1), state);
    auto cie = std::make_unique<bsnn::Connection>(i, e, net.w_ie, connection_params(cfg, true, 2), state);
    auto cii = std::make_unique<bsnn::Connection>(i, i, net.w_ii, connection_params(cfg, true, 3), state);
    bsnn::Connection& ee = *cee;
    bsnn::Connection& ie = *cie;
    system.add_connection(std::move(cee));
    system.add_connection(std::move(cei));
    system.add_connection(std::move(cie));
    system.add_connection(std::move(cii));
    system.add_stimulus(std::make_unique<bsnn::Stimulus>(net.stim.timestep_event_counts, net.stim.neuron_ids,
                                                         net.stim.post_group_offsets, net.stim.amplitude_changes, state));
    const float dt = bsnn::buryn::timestep;
    uint32_t offset = 0;
    if (cfg.e_e_plasticity_enabled) {
        bsnn::PlasticityParams p;
        p.ltp_A = cfg.e_e_plasticity_ltp_A;
        p.ltd_A = cfg.e_e_plasticity_ltd_A;
        p.ltp_B = cfg.e_e_plasticity_ltp_B;
        p.ltd_B = cfg.e_e_plasticity_ltd_B;
        p.weight_min = cfg.e_e_plasticity_weight_min;
        p.weight_max = cfg.e_e_plasticity_weight_max;
        p.pre_trace_decay = std::exp(-1.0f * dt / cfg.e_e_plasticity_tau_ltp);
        p.post_trace_decay = std::exp(-1.0f * dt / cfg.e_e_plasticity_tau_ltd);
        p.triplet_pre_trace_decay = std::exp(-1.0f * dt / cfg.e_e_plasticity_triplet_tau_ltp);
        p.triplet_post_trace_decay = std::exp(-1.0f * dt / cfg.e_e_plasticity_triplet_tau_ltd);
        p.plasticity_offset = offset++;
        system.add_plasticity(std::make_unique<bsnn::TripletPlasticity>(ee, p, state));
        validate_plasticity_params(p, true, "e_e excitatory Triplet plasticity");
    }
    if (cfg.i_e_plasticity_enabled) {
        bsnn::PlasticityParams p;
        p.ltp_A = cfg.i_e_plasticity_ltp_A;
        p.ltd_A = cfg.i_e_plasticity_ltd_A;
        p.ltd_B = cfg.i_e_plasticity_ltd_B;
        p.weight_min = cfg.i_e_plasticity_weight_min;
        p.weight_max = cfg.i_e_plasticity_weight_max;
        p.pre_trace_decay = std::exp(-1.0f * dt / cfg.i_e_plasticity_tau_ltp);
        p.post_trace_decay = std::exp(-1.0f * dt / cfg.i_e_plasticity_tau_ltd);
        p.plasticity_offset = offset++;
        system.add_plasticity(std::make_unique<bsnn::IstdpPlasticity>(ie, p, state));
        validate_plasticity_params(p, false, "i_e inhibitory Istdp plasticity");
    }
    const uint32_t interval = bsnn::buryn::recording_interval_steps;
    system.add_monitor(std::make_unique<bsnn::SpikeRecorder>(e, cfg.e_spike_recording_file, interval, state));
    system.add_monitor(std::make_unique<bsnn::SpikeRecorder>(i, cfg.i_spike_recording_file, interval, state));
    system.add_monitor(std::make_unique<bsnn::VoltageRecorder>(e, cfg.voltage_recording_file,
                                                               cfg.voltage_recording_neuron_ids, interval, state));
    system.add_monitor(std::make_unique<bsnn::WeightRecorder>(ee, cfg.e_e_weight_recording_file, state));
    std::cout << state.memory_report() << "\n";
    std::cout << "Running simulation...\n";
    system.run(cfg.simulation_steps);
    std::cout << "Simulation complete.\n";
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        std::string mode = "run", config_path = "config.json", form = "f32";
        for (int a = 1; a < argc; ++a) {
            const std::string s = argv[a];
            if (s == "--print-config" || s == "--generate-only") mode = s;
            else if (s == "--weight-format" && a + 1 < argc) form = argv[++a];
            else config_path = s;
        }
        const bsnn::Config cfg = bsnn::load_config_json(config_path);
        if (mode == "--print-config") {
            std::fputs(bsnn::config_print::dump(cfg).c_str(), stdout);
            return 0;
        }
        if (mode == "--generate-only") {
            clean_up(cfg.output_directory, cfg.description, config_path);
            generate_network(cfg);
            return 0;
        }
        return run(cfg, config_path, weight_format_of(form));
    } catch (const std::exception& ex) {
        std::cerr << "bsnn_main: " << ex.what() << "\n";
        return 1;
    }
}
