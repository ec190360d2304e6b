// ref_config.cpp -- test infrastructure: the reference's own configuration loader and network
// generators (cpp_src/core/config.cpp, cpp_src/generation/*.cpp, compiled from the reference
// sources in place by `make refcfg`), driven the way cpp_src/main_buryn.cpp:98-160 drives them,
// so that the JSON loader and generators of this project can be checked against them on the CPU.
//
//   ref_config --print-config CONFIG    the resolved Config, one field per line (same printer as
//                                       bsnn_main --print-config)
//   ref_config --generate-only CONFIG   locations, weight files and stimulus schedules into the
//                                       configured paths (the output directory must exist)
#include <cstdio>
#include <exception>
#include <filesystem>
#include <iostream>
#include <string>

#include "buryn_definitions.h"
#include "config.h"
#include "generate_location.h"
#include "generate_stimulus_schedules.h"
#include "generate_weights.h"

#include "../include/bsnn_config_print.hpp"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: ref_config --print-config|--generate-only CONFIG\n");
        return 2;
    }
    try {
        const std::string mode = argv[1];
        Config c = load_config_json(argv[2]);
        if (mode == "--print-config") {
            std::fputs(bsnn::config_print::dump(c).c_str(), stdout);
            return 0;
        }
        buryn::rng_seed = c.rng_seed;
        buryn::timestep = c.timestep;
        for (const char* sub : {"stimulus_schedules", "recordings", "locations", "videos", "weights", "plots"})
            std::filesystem::create_directories(std::filesystem::path(c.output_directory) / sub);
        auto le = generate_location::generate_2d_grid_locations(c.excitatory_locations_file, c.num_excitatory_neurons,
                                                                 c.excitatory_location_spacing, c.excitatory_side_points,
                                                                 c.excitatory_side_points);
        auto li = generate_location::generate_2d_grid_locations(c.inhibitory_locations_file, c.num_inhibitory_neurons,
                                                                 c.inhibitory_location_spacing, c.inhibitory_side_points,
                                                                 c.inhibitory_side_points);
        generate_weights::distance_2d_weights_file(c.weights_e_to_e_filename, le, le, c.weight_generation_params_e_to_e);
        generate_weights::distance_2d_weights_file(c.weights_e_to_i_filename, le, li, c.weight_generation_params_e_to_i);
        generate_weights::distance_2d_weights_file(c.weights_i_to_e_filename, li, le, c.weight_generation_params_i_to_e);
        generate_weights::distance_2d_weights_file(c.weights_i_to_i_filename, li, li, c.weight_generation_params_i_to_i);
        generate_stimulus_schedules::StimulusGenerationParams sp{};
        sp.max_timestep = c.simulation_steps;
        sp.selected_input_ids = c.stimulus_selected_input_ids;
        sp.selected_input_post_group_offsets = c.stimulus_selected_input_post_group_offsets;
        sp.start_clock_steps = c.stimulus_start_clock_steps;
        sp.end_clock_steps = c.stimulus_end_clock_steps;
        sp.stimulus_input_values = c.stimulus_input_values;
        generate_stimulus_schedules::partial_group_multiple_square_waves(c.stimulus_schedules_folder, sp);
        return 0;
    } catch (const std::exception& ex) {
        std::cerr << "ref_config: " << ex.what() << "\n";
        return 1;
    }
}
