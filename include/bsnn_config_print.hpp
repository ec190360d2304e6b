// bsnn_config_print.hpp -- one "key = value" line per resolved field of a run configuration
// (floats to 9 significant digits, so two loaders can be compared exactly).  Templated on the
// config type so the same printer serves any struct with the reference's field names.
#pragma once

#include <cstdio>
#include <string>
#include <vector>

namespace bsnn {
namespace config_print {

inline std::string v(float x) {
    char b[48];
    std::snprintf(b, sizeof b, "%.9g", static_cast<double>(x));
    return b;
}
inline std::string v(double x) { return v(static_cast<float>(x)); }
inline std::string v(int x) { return std::to_string(x); }
inline std::string v(unsigned x) { return std::to_string(x); }
inline std::string v(bool x) { return x ? "true" : "false"; }
inline std::string v(const std::string& x) { return "\"" + x + "\""; }
template <class T>
inline std::string v(const std::vector<T>& xs) {
    std::string s = "[";
    for (size_t k = 0; k < xs.size(); ++k) s += (k ? ", " : "") + v(xs[k]);
    return s + "]";
}
template <class W>
inline std::string wv(const W& p) {
    return "{" + v(p.x_location_length) + ", " + v(p.y_location_length) + ", " + v(p.max_distance) + ", " +
           v(p.spread_scale) + ", " + v(p.max_weight_value) + ", " + v(p.weight_value_normal_dropoff) + ", " +
           v(p.probabilistic_normal_not_uniform) + ", " + v(p.probability_multiplier) + ", " +
           v(p.no_diagonal_connections) + "}";
}

template <class C>
std::string dump(const C& c) {
    std::string o;
#define P(f) o += std::string(#f) + " = " + v(c.f) + "\n"
#define PW(f) o += std::string(#f) + " = " + wv(c.f) + "\n"
    P(simulation_steps); P(output_directory); P(description); P(rng_seed); P(timestep);
    P(num_excitatory_neurons); P(num_inhibitory_neurons); P(g_leak); P(membrane_capacitance);
    P(depolarization_slope_factor); P(v_effective_spike_threshold); P(v_excitatory_reversal);
    P(v_inhibitory_reversal); P(v_threshold); P(v_reset); P(v_rest); P(refractory_steps);
    P(group_e_mean_background_excitatory_spikes); P(group_e_mean_background_inhibitory_spikes);
    P(group_e_background_excitatory_postsynaptic_r_trace_decay); P(group_e_background_excitatory_postsynaptic_d_trace_decay);
    P(group_e_background_inhibitory_postsynaptic_r_trace_decay); P(group_e_background_inhibitory_postsynaptic_d_trace_decay);
    P(group_e_background_excitatory_scaling_factor); P(group_e_background_inhibitory_scaling_factor);
    P(group_i_mean_background_excitatory_spikes); P(group_i_mean_background_inhibitory_spikes);
    P(group_i_background_excitatory_postsynaptic_r_trace_decay); P(group_i_background_excitatory_postsynaptic_d_trace_decay);
    P(group_i_background_inhibitory_postsynaptic_r_trace_decay); P(group_i_background_inhibitory_postsynaptic_d_trace_decay);
    P(group_i_background_excitatory_scaling_factor); P(group_i_background_inhibitory_scaling_factor);
    P(excitatory_locations_file); P(inhibitory_locations_file); P(excitatory_location_spacing);
    P(inhibitory_location_spacing); P(excitatory_side_points); P(inhibitory_side_points); P(side_length);
    P(e_max_weight_value); P(i_max_weight_value); P(max_connection_distance); P(connection_spread_scale);
    P(connection_probability_multiplier);
    PW(weight_generation_params_e_to_e); PW(weight_generation_params_e_to_i);
    PW(weight_generation_params_i_to_e); PW(weight_generation_params_i_to_i);
    P(weights_e_to_i_filename); P(weights_i_to_e_filename); P(weights_e_to_e_filename); P(weights_i_to_i_filename);
    P(tau_decay_e); P(tau_rise_e); P(tau_decay_i); P(tau_rise_i); P(postsynaptic_kernel_normalization_value);
    P(e_e_plasticity_enabled); P(e_e_plasticity_ltp_A); P(e_e_plasticity_ltd_A); P(e_e_plasticity_ltp_B);
    P(e_e_plasticity_ltd_B); P(e_e_plasticity_tau_ltp); P(e_e_plasticity_tau_ltd); P(e_e_plasticity_triplet_tau_ltp);
    P(e_e_plasticity_triplet_tau_ltd); P(e_e_plasticity_weight_min); P(e_e_plasticity_weight_max);
    P(i_e_plasticity_enabled); P(i_e_plasticity_ltp_A); P(i_e_plasticity_ltd_A); P(i_e_plasticity_ltd_B);
    P(i_e_plasticity_tau_ltp); P(i_e_plasticity_tau_ltd); P(i_e_plasticity_weight_min); P(i_e_plasticity_weight_max);
    P(stimulus_input_values); P(stimulus_schedules_folder); P(stimulus_selected_input_ids);
    P(stimulus_selected_input_post_group_offsets); P(stimulus_start_clock_steps); P(stimulus_end_clock_steps);
    P(e_spike_recording_file); P(i_spike_recording_file); P(voltage_recording_file); P(voltage_recording_neuron_ids);
    P(e_e_weight_recording_file);
#undef P
#undef PW
    return o;
}

}  // namespace config_print
}  // namespace bsnn
