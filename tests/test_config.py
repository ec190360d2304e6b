"""The JSON run configuration and the network generation of the command-line driver (CPU).

bsnn_main (example-cuda-spiking-nn_b200/csrc/bsnn_main.cpp, on include/bsnn_config.hpp and
include/bsnn_generate.hpp) against the reference's own loader and generators built from its sources
(oracle/_ref/ref_config, `make -C oracle refcfg`): the resolved configuration must print
identically, errors must carry the same message, and the generated location, weight and stimulus
files must be byte-identical.  The checks against the reference are skipped where it is not built;
the self-contained checks of defaults and path handling always run.
"""
from __future__ import annotations

import filecmp
import json
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
MAIN = ROOT / "example-cuda-spiking-nn_b200" / "bsnn_main"
REF = ROOT / "oracle" / "_ref" / "ref_config"
REF_EXAMPLE = Path(os.environ.get("BSNN_REFERENCE_ROOT", ROOT.parent / "reference")) / "configs_to_run" / "config01.json"

needs_main = pytest.mark.skipif(not MAIN.exists(), reason="bsnn_main not built")
needs_ref = pytest.mark.skipif(not REF.exists(), reason="reference loader not built (make -C oracle refcfg)")


def run(exe, *args, cwd=None):
    p = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=300)
    return p.returncode, p.stdout, p.stderr


def parse_dump(text):
    out = {}
    for line in text.splitlines():
        k, _, v = line.partition(" = ")
        out[k] = v
    return out


def small_config(out_dir, **over):
    """A 100 E (10 x 10) + 25 I (5 x 5) network in the reference's example style."""
    c = {
        "simulation_steps": 3001, "output_directory": str(out_dir), "description": "small test network",
        "rng_seed": 751, "timestep": 1e-4, "num_excitatory_neurons": 100, "num_inhibitory_neurons": 25,
        "g_leak": 0.05e-6, "membrane_capacitance": 100.0e-12, "refractory_steps": 20,
        "group_e_mean_background_excitatory_spikes": 0.5,
        "group_e_background_excitatory_postsynaptic_r_trace_decay": 0.71653,
        "group_e_background_excitatory_postsynaptic_d_trace_decay": 0.95122,
        "group_e_background_excitatory_scaling_factor": 2.5e-9,
        "excitatory_locations_file": "locations/group_e_locations.txt",
        "inhibitory_locations_file": "locations/group_i_locations.txt",
        "excitatory_location_spacing": 1.0, "inhibitory_location_spacing": 2.0,
        "excitatory_side_points": 10, "inhibitory_side_points": 5, "side_length": 10.0,
        "e_to_e_max_weight_value": 1.5e-9, "e_to_e_max_distance": 9.0, "e_to_e_spread_scale": 16.0,
        "e_to_e_probabilistic_normal_not_uniform": True, "e_to_e_probability_multiplier": 0.4,
        "e_to_e_no_diagonal_connections": True,
        "e_to_i_max_weight_value": 1.5e-9, "e_to_i_probability_multiplier": 0.6, "e_to_i_spread_scale": 16.0,
        "e_to_i_max_distance": 9.0, "e_to_i_weight_value_normal_dropoff": True,
        "i_to_e_max_weight_value": 5.0e-9, "i_to_e_probability_multiplier": 0.6, "i_to_e_spread_scale": 64.0,
        "i_to_e_max_distance": 9.0, "i_to_i_max_weight_value": 5.0e-9, "i_to_i_probability_multiplier": 0.6,
        "i_to_i_max_distance": 9.0, "i_to_i_no_diagonal_connections": True,
        "weights_e_to_e_filename": "weights/weights_e_to_e.txt", "weights_e_to_i": "weights/weights_e_to_i.txt",
        "weights_i_to_e_filename": "weights/weights_i_to_e.txt", "weights_i_to_i_filename": "weights/weights_i_to_i.txt",
        "tau_decay_e": 5e-3, "tau_rise_e": 1e-3, "tau_decay_i": 10e-3, "tau_rise_i": 0.5e-3,
        "postsynaptic_kernel_normalization_value": 1.7,
        "e_e_plasticity_enabled": True, "e_e_plasticity_weight_max": 3e-9,
        "i_e_plasticity_enabled": True, "i_e_plasticity_weight_max": 3e-9,
        "stimulus_input_values": [0.5e-9, 0.3e-9], "stimulus_schedules_folder": "stimulus_schedules",
        "stimulus_selected_input_ids": [3, 1, 4, 1, 5, 9, 2, 6],
        "stimulus_selected_input_post_group_offsets": [0, 0, 0, 0, 0, 0, 0, 0],
        "stimulus_start_clock_steps": [100, 1500], "stimulus_end_clock_steps": [900, 2400],
        "e_spike_recording_file": "recordings/spikes_e.txt", "i_spike_recording_file": "recordings/spikes_i.txt",
        "voltage_recording_file": "recordings/voltages.txt", "voltage_recording_neuron_ids": [0, 17, 99],
        "e_e_weight_recording_file": "weights/weights_e_to_e_recordings.txt",
    }
    c.update(over)
    return c


def write(path, obj):
    path.write_text(json.dumps(obj, indent=2) if not isinstance(obj, str) else obj)
    return path


@needs_main
def test_defaults_and_paths_without_the_reference(tmp_path):
    cfg = write(tmp_path / "c.json", {"output_directory": "out/run1", "weights_e_to_e": "w/ee.txt",
                                      "e_spike_recording_file": "out/x/s.txt", "voltage_recording_file": "/abs/v.txt",
                                      "connection_probability_multiplier": 0.25, "e_to_i_probability_multiplier": 0.5,
                                      "rng_seed": 7.0})
    rc, out, err = run(MAIN, "--print-config", cfg)
    assert rc == 0, err
    d = parse_dump(out)
    assert d["simulation_steps"] == "10000" and d["refractory_steps"] == "50" and d["rng_seed"] == "7"
    assert d["weights_e_to_e_filename"] == '"out/run1/w/ee.txt"'  # legacy key, prefixed
    assert d["e_spike_recording_file"] == '"out/x/s.txt"'  # already under the directory's first component
    assert d["voltage_recording_file"] == '"/abs/v.txt"'  # absolute stays
    ee = d["weight_generation_params_e_to_e"].strip("{}").split(", ")
    ei = d["weight_generation_params_e_to_i"].strip("{}").split(", ")
    assert ee[7] == "0.25" and ei[7] == "0.5"  # global, then the per-connection override
    assert d["stimulus_selected_input_post_group_offsets"] == "[0, 0, 0, 0, 0, 0, 0, 0, 0, 0]"


BAD = [
    ("[1, 2]", "Config JSON must be an object at the top level"),
    ('{"num_excitatory_neurons": 0}', "Neuron counts must be > 0"),
    ('{"membrane_capacitance": -1.0}', "membrane_capacitance must be > 0"),
    ('{"stimulus_selected_input_ids": 3}', "stimulus_selected_input_ids must be an array"),
    ('{"stimulus_selected_input_ids": [1, -2]}', "stimulus_selected_input_ids must not contain negative values"),
    ('{"stimulus_start_clock_steps": [1.5]}', "stimulus_start_clock_steps must contain only integers"),
    ('{"voltage_recording_neuron_ids": ["a"]}', "voltage_recording_neuron_ids must contain only integers"),
    ('{"stimulus_input_values": {}}', "stimulus_input_values must be an array"),
    ('{"stimulus_selected_input_ids": [1, 2], "stimulus_selected_input_post_group_offsets": [0]}',
     "stimulus_selected_input_post_group_offsets size must match stimulus_selected_input_ids size"),
]


@needs_main
@pytest.mark.parametrize("text,msg", BAD)
def test_config_errors(tmp_path, text, msg):
    cfg = write(tmp_path / "bad.json", text)
    rc, _, err = run(MAIN, "--print-config", cfg)
    assert rc == 1 and msg in err, err
    if REF.exists():
        rc2, _, err2 = run(REF, "--print-config", cfg)
        assert rc2 == 1 and msg in err2, err2


@needs_main
def test_malformed_json_and_wrong_types_fail(tmp_path):
    for text in ('{"a": 1,}', '{"g_leak": "x"}', '{"e_e_plasticity_enabled": 1}', '{"description": 3}', "{"):
        rc, _, err = run(MAIN, "--print-config", write(tmp_path / "m.json", text))
        assert rc == 1, (text, err)
    rc, _, err = run(MAIN, "--print-config", tmp_path / "missing.json")
    assert rc == 1 and "Failed to open config file" in err


@needs_main
@needs_ref
def test_resolved_config_matches_the_reference_loader(tmp_path):
    configs = [write(tmp_path / "small.json", small_config("out/small")),
               write(tmp_path / "empty.json", {}),
               write(tmp_path / "types.json", {"simulation_steps": 12.0, "rng_seed": -5, "timestep": 1,
                                               "e_e_plasticity_enabled": False, "description": "café \\n",
                                               "i_to_i_x_location_length": 7, "side_length": 3.5,
                                               "stimulus_input_values": [1, 2.5e-10]})]
    if REF_EXAMPLE.exists():
        configs.append(REF_EXAMPLE)
    for cfg in configs:
        rc, ours, err = run(MAIN, "--print-config", cfg)
        assert rc == 0, err
        rc, theirs, err = run(REF, "--print-config", cfg)
        assert rc == 0, err
        assert ours == theirs, cfg


@needs_main
@needs_ref
@pytest.mark.parametrize("variant", ["small", "dropoff_and_duplicates"])
def test_generated_files_match_the_reference_generators(tmp_path, variant):
    over = {} if variant == "small" else {"e_to_e_weight_value_normal_dropoff": True, "i_to_e_no_diagonal_connections": True,
                                          "stimulus_selected_input_ids": [],
                                          "stimulus_selected_input_post_group_offsets": [], "rng_seed": 3}
    ours_cfg = write(tmp_path / "ours.json", small_config(tmp_path / "ours", **over))
    ref_cfg = write(tmp_path / "ref.json", small_config(tmp_path / "ref", **over))
    rc, _, err = run(MAIN, "--generate-only", ours_cfg)
    assert rc == 0, err
    rc, _, err = run(REF, "--generate-only", ref_cfg)
    assert rc == 0, err
    files = sorted(p.relative_to(tmp_path / "ref") for p in (tmp_path / "ref").rglob("*") if p.is_file())
    assert len(files) >= 9, files
    for rel in files:
        assert filecmp.cmp(tmp_path / "ours" / rel, tmp_path / "ref" / rel, shallow=False), rel
    # the driver's own outputs beside them: description and the config copy
    assert (tmp_path / "ours" / "description.txt").read_text() == "small test network"
    assert (tmp_path / "ours" / "ours.json").exists()
    for sub in ("stimulus_schedules", "recordings", "locations", "videos", "weights", "plots"):
        assert (tmp_path / "ours" / sub).is_dir()


@needs_main
def test_output_directory_is_emptied_first(tmp_path):
    out = tmp_path / "out"
    (out / "old").mkdir(parents=True)
    (out / "old" / "stale.txt").write_text("x")
    cfg = write(tmp_path / "c.json", small_config(out, simulation_steps=50))
    rc, _, err = run(MAIN, "--generate-only", cfg)
    assert rc == 0, err
    assert not (out / "old").exists()
    assert (out / "weights" / "weights_e_to_e.txt").read_text().startswith("pre_neuron_id, post_neuron_id, weight\n")
