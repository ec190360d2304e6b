// bsnn_generate.hpp -- host-side network generation for a run configuration (one-shot set-up,
// outside the per-step hot path): grid locations, distance-dependent weight matrices and the
// square-wave stimulus schedule, with the files the reference writes for each.
//
// These restate cpp_src/generation/generate_location.cpp:5-47, generate_weights.cpp:10-107 (with
// cpp_src/utils/math_functions.cpp:8-16) and generate_stimulus_schedules.cpp:20-228.  The steps
// and their order are kept on purpose: the weight matrix is a function of the exact sequence of
// std::mt19937 draws (one per candidate synapse inside the distance cutoff, pre-major), so a
// different loop order or arithmetic would give a different network from the same seed.  Built
// with the same C++ standard library as the reference, the matrices and files are identical.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <utility>
#include <vector>

#include "bsnn_config.hpp"

namespace bsnn {
namespace generate {

// Neuron id -> (column, row) * spacing on a rows x cols grid, row-major; also written to
// `path` as "neuron_id, locationdim_0, locationdim_1" lines.
inline std::vector<std::vector<float>> grid_locations(const std::string& path, uint32_t num_neurons, float spacing,
                                                      uint32_t rows, uint32_t cols) {
    std::vector<std::vector<float>> loc;
    if (num_neurons == 0) return loc;
    if (rows == 0 || cols == 0) throw std::invalid_argument("rows and cols must be > 0");
    if (rows < (num_neurons + cols - 1) / cols) throw std::invalid_argument("grid too small: need at least num_neurons cells");
    loc.resize(num_neurons);
    std::ofstream out(path, std::ios::trunc);
    if (!out.is_open() || !out.good()) throw std::runtime_error("failed to open output file: " + path);
    out << "neuron_id, locationdim_0, locationdim_1\n";
    for (uint32_t id = 0; id < num_neurons; ++id) {
        const float x = static_cast<float>(id % cols) * spacing;
        const float y = static_cast<float>(id / cols) * spacing;
        loc[id] = {x, y};
        out << id << ", " << x << ", " << y << "\n";
    }
    if (!out.good()) throw std::runtime_error("failed while writing output file: " + path);
    return loc;
}

// Euclidean distance on a periodic lx x ly domain.
inline float periodic_distance(float x0, float y0, float x1, float y1, float lx, float ly) {
    float dx = std::fabs(x0 - x1);
    float dy = std::fabs(y0 - y1);
    dx = std::min(dx, lx - dx);
    dy = std::min(dy, ly - dy);
    return std::sqrt(dx * dx + dy * dy);
}

inline float connection_probability(float distance, float spread_scale) {
    return std::exp(-1.0f * (std::pow(distance, 2.0f)) / (spread_scale));
}

// Distance-dependent weights [pre][post], also written to `path` as "pre, post, weight" lines
// (every pair).  A candidate synapse (not on the diagonal when that is excluded, within
// max_distance) draws one uniform float u from mt19937(seed); it exists when u < p, with
// p = probability_multiplier (times exp(-d^2 / spread_scale) when probabilistic_normal_not_uniform),
// and then weighs max_weight_value (times the same Gaussian when weight_value_normal_dropoff).
// An unopenable file or an empty group gives an empty matrix (as the reference does).
inline std::vector<std::vector<float>> distance_weights(const std::string& path, const std::vector<std::vector<float>>& pre,
                                                        const std::vector<std::vector<float>>& post,
                                                        const WeightGenerationParams& p, int seed) {
    std::ofstream out(path, std::ios::trunc);
    if (!out.is_open()) {
        std::cerr << "Failed to create weights file: " << path << "\n";
        return {};
    }
    const uint32_t n_pre = static_cast<uint32_t>(pre.size()), n_post = static_cast<uint32_t>(post.size());
    if (n_pre == 0 || n_post == 0) {
        std::cerr << "Neuron groups must not be empty.\n";
        return {};
    }
    std::vector<std::vector<float>> w(n_pre, std::vector<float>(n_post, 0.0f));
    out << "pre_neuron_id, post_neuron_id, weight\n";
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> unif(0.0f, 1.0f);
    for (uint32_t i = 0; i < n_pre; ++i) {
        for (uint32_t q = 0; q < n_post; ++q) {
            const float d = periodic_distance(pre[i][0], pre[i][1], post[q][0], post[q][1], p.x_location_length,
                                              p.y_location_length);
            float v = 0.0f;
            const bool candidate = !(p.no_diagonal_connections && i == q) && !(std::abs(d) > p.max_distance);
            if (candidate) {
                const float u = unif(rng);
                float prob = p.probability_multiplier;
                if (p.probabilistic_normal_not_uniform) prob *= connection_probability(d, p.spread_scale);
                if (u < prob) {
                    v = p.max_weight_value;
                    if (p.weight_value_normal_dropoff) v *= std::exp(-1.0f * (std::pow(d, 2.0f)) / (p.spread_scale));
                    if (v < 0)
                        throw std::runtime_error(
                            "distance_weights: negative weight value calculated (pre=" + std::to_string(i) +
                            ", post=" + std::to_string(q) + ", weight=" + std::to_string(v) + ")");
                }
            }
            w[i][q] = v;
            out << i << ", " << q << ", " << v << '\n';
        }
    }
    return w;
}

// The stimulus as per-step events (generate_stimulus_schedules.h StimulusGenerationResult).
struct StimulusSchedule {
    std::vector<uint32_t> timestep_event_counts;
    std::vector<uint32_t> neuron_ids;
    std::vector<uint32_t> post_group_offsets;
    std::vector<float> amplitude_changes;
};

namespace detail {
inline bool write_lines(const std::filesystem::path& p, const std::vector<uint32_t>& v) {
    std::ofstream out(p);
    if (!out.is_open()) return false;
    for (uint32_t x : v) out << x << '\n';
    return true;
}
inline bool write_lines(const std::filesystem::path& p, const std::vector<float>& v) {
    std::ofstream out(p);
    if (!out.is_open()) return false;
    for (float x : v) out << x << '\n';
    return true;
}
}  // namespace detail

// Square waves into selected neurons: +amp at each start step, -amp at end + 1 (inclusive end),
// events of one step sorted by (post_group_offset, neuron), duplicates of (offset, neuron) in the
// selection dropped, a single amplitude broadcast to every wave.  Invalid parameters print a
// message and give an empty schedule; two events for one neuron in one step are an error (the
// reference exits the process; this throws).  The schedule files go to `folder`.
inline StimulusSchedule square_waves(const std::string& folder, uint32_t max_timestep, const std::vector<uint32_t>& ids,
                                     const std::vector<uint32_t>& offsets, const std::vector<uint32_t>& starts,
                                     const std::vector<uint32_t>& ends, std::vector<float> values) {
    StimulusSchedule r;
    if (ids.size() != offsets.size()) {
        std::cerr << "Selected neuron vectors must have the same size: selected_input_ids=" << ids.size()
                  << ", selected_input_post_group_offsets=" << offsets.size() << "\n";
        return r;
    }
    if (starts.size() != ends.size()) {
        std::cerr << "Multi square wave parameter vectors must have the same size: start_clock_steps=" << starts.size()
                  << ", end_clock_steps=" << ends.size() << "\n";
        return r;
    }
    if (values.size() != starts.size()) {
        if (values.size() == 1) {
            values.resize(starts.size(), values[0]);
        } else {
            std::cerr << "Multi square wave parameter vectors must have the same size: stimulus_input_values="
                      << values.size() << ", start_clock_steps=" << starts.size() << "\n";
            return r;
        }
    }
    for (size_t k = 0; k < starts.size(); ++k)
        if (starts[k] > ends[k]) {
            std::cerr << "Square wave start has to be before end: start_clock_step (" << starts[k]
                      << ") > end_clock_step (" << ends[k] << ")\n";
            return r;
        }
    if (max_timestep == 0) {
        std::cerr << "params.max_timestep must be > 0\n";
        return r;
    }
    const uint32_t T = max_timestep;
    const std::filesystem::path dir(folder);
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) {
        std::cerr << "Failed to create stimulus schedules folder: " << dir << "\n";
        return r;
    }
    std::vector<std::pair<uint32_t, uint32_t>> sel;  // (offset, neuron), first occurrence order
    std::unordered_set<uint64_t> seen;
    for (size_t k = 0; k < ids.size(); ++k) {
        const uint64_t key = (static_cast<uint64_t>(offsets[k]) << 32) | ids[k];
        if (seen.insert(key).second) sel.emplace_back(offsets[k], ids[k]);
    }
    struct Ev {
        uint32_t t, off, neuron;
        float delta;
    };
    std::vector<Ev> ev;
    for (const auto& s : sel)
        for (size_t k = 0; k < starts.size(); ++k) {
            if (starts[k] < T) ev.push_back(Ev{starts[k], s.first, s.second, +values[k]});
            const uint32_t off_t = ends[k] + 1;
            if (off_t < T) ev.push_back(Ev{off_t, s.first, s.second, -values[k]});
        }
    std::sort(ev.begin(), ev.end(), [](const Ev& a, const Ev& b) {
        if (a.t != b.t) return a.t < b.t;
        if (a.off != b.off) return a.off < b.off;
        return a.neuron < b.neuron;
    });
    for (size_t k = 1; k < ev.size(); ++k)
        if (ev[k].t == ev[k - 1].t && ev[k].off == ev[k - 1].off && ev[k].neuron == ev[k - 1].neuron)
            throw std::runtime_error("duplicate events detected for time step " + std::to_string(ev[k].t) +
                                     ", post_group_offset " + std::to_string(ev[k].off) + ", neuron_id " +
                                     std::to_string(ev[k].neuron));
    r.timestep_event_counts.assign(T, 0u);
    for (const auto& e : ev) {
        r.timestep_event_counts[e.t] += 1u;
        r.neuron_ids.push_back(e.neuron);
        r.post_group_offsets.push_back(e.off);
        r.amplitude_changes.push_back(e.delta);
    }
    if (!detail::write_lines(dir / "timestep_event_counts.txt", r.timestep_event_counts))
        std::cerr << "Failed to write timestep_event_counts.txt\n";
    if (!detail::write_lines(dir / "stimulus_event_neuron_ids.txt", r.neuron_ids))
        std::cerr << "Failed to write stimulus_event_neuron_ids.txt\n";
    if (!detail::write_lines(dir / "stimulus_event_post_group_offsets.txt", r.post_group_offsets))
        std::cerr << "Failed to write stimulus_event_post_group_offsets.txt\n";
    if (!detail::write_lines(dir / "stimulus_event_delta_amplitudes.txt", r.amplitude_changes))
        std::cerr << "Failed to write stimulus_event_delta_amplitudes.txt\n";
    if (!sel.empty()) {
        std::ofstream out(dir / "stimulus_events_compact.txt");
        if (out.is_open()) {
            out << "# idx time_step post_group_offset neuron_id delta\n";
            uint32_t idx = 0;
            for (const auto& e : ev) out << idx++ << " " << e.t << " " << e.off << " " << e.neuron << " " << e.delta << "\n";
        }
    }
    return r;
}

}  // namespace generate
}  // namespace bsnn
