"""Network descriptions that can be built into any backend with the Simulation method names.

A `NetworkSpec` holds what the reference's main_buryn.cpp wires up (cpp_src/main_buryn.cpp:98-340):
two neuron groups, up to four connections, a stimulus, plasticities and monitors.  `build()`
replays those constructor calls on a backend -- libbsnn's `Simulation`, or the CPU oracle in the
tests -- so both see identical inputs.

`synthetic_network()` makes the workloads the benchmarks are quoted on: seeded synthetic inputs
with the reference example's shapes, sizes and parameter values (no dataset is involved).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import generation
from ._ffi import (PLASTICITY_ISTDP, PLASTICITY_STDP, PLASTICITY_TRIPLET, ConnectionParams, NeuronGroupParams,
                   PlasticityParams)


@dataclass
class ConnSpec:
    pre: int
    post: int
    weights: np.ndarray
    params: dict


@dataclass
class PlastSpec:
    kind: int
    conn: int
    params: dict


@dataclass
class MonSpec:
    kind: str  # "spikes" | "voltage"
    group: int
    ids: tuple = ()
    interval: int = 0


@dataclass
class NetworkSpec:
    num_excitatory: int
    num_inhibitory: int
    total_steps: int
    rng_seed: int = 314
    timestep: float = 1e-4
    recording_interval_steps: int = 10000
    groups: list = field(default_factory=list)  # NeuronGroupParams kwargs
    conns: list = field(default_factory=list)   # ConnSpec
    plasts: list = field(default_factory=list)  # PlastSpec
    stimulus: tuple | None = None               # (counts, ids, offsets, deltas)
    monitors: list = field(default_factory=list)
    name: str = "network"

    @property
    def num_neurons(self) -> int:
        return self.num_excitatory + self.num_inhibitory

    def synapse_entries(self) -> int:
        return int(sum(c.weights.size for c in self.conns))

    def sim_kwargs(self) -> dict:
        n_events = 0 if self.stimulus is None else len(self.stimulus[1])
        return dict(total_simulation_length=self.total_steps, num_stimulus_events=n_events,
                    num_plasticities=len(self.plasts), recording_interval_steps=self.recording_interval_steps,
                    rng_seed=self.rng_seed)

    def build(self, sim):
        """Adds every component to `sim` (a Simulation or an object with the same methods)."""
        for g in self.groups:
            sim.add_neuron_group(NeuronGroupParams.make(**g))
        for c in self.conns:
            sim.add_connection(c.pre, c.post, c.weights, ConnectionParams.make(**c.params))
        if self.stimulus is not None:
            sim.add_stimulus(*self.stimulus)
        for p in self.plasts:
            sim.add_plasticity(p.kind, p.conn, PlasticityParams.make(**p.params))
        for m in self.monitors:
            if m.kind == "spikes":
                sim.add_spike_recorder(m.group, m.interval)
            else:
                sim.add_voltage_recorder(m.group, m.ids, m.interval)
        return sim


# ---- the reference example's parameter values (configs_to_run/config01.json) -------------------
EXAMPLE = dict(
    timestep=1e-4, g_leak=0.05e-6, membrane_capacitance=100.0e-12, depolarization_slope_factor=0.0065625,
    v_effective_spike_threshold=-0.060625, v_excitatory_reversal=0.0, v_inhibitory_reversal=-0.08,
    v_threshold=-0.04, v_reset=-0.06, v_rest=-0.07, refractory_steps=50,
    mean_background_excitatory_spikes=0.02, mean_background_inhibitory_spikes=1.5,
    background_excitatory_postsynaptic_r_trace_decay=0.71653,
    background_excitatory_postsynaptic_d_trace_decay=0.95122,
    background_inhibitory_postsynaptic_r_trace_decay=0.71653,
    background_inhibitory_postsynaptic_d_trace_decay=0.96722,
    background_excitatory_scaling_factor=2.5e-9, background_inhibitory_scaling_factor=2.5e-12,
)
EXAMPLE_TRIPLET = dict(ltp_A=7.5e-22, ltd_A=7.0e-15, ltp_B=9.4e-15, ltd_B=2.3e-12, tau_ltp=33.7e-3, tau_ltd=16.8e-3,
                       triplet_tau_ltp=101e-3, triplet_tau_ltd=125e-3, weight_min=0.0, weight_max=3.0e-9)
EXAMPLE_ISTDP = dict(ltp_A=1.0e-12, ltd_A=1.0e-12, ltd_B=1.2e-3, tau_ltp=20e-3, tau_ltd=20e-3, weight_min=0.0,
                     weight_max=3.0e-9)


def decay(dt: float, tau: float) -> float:
    """std::exp(-1.0f * timestep / tau) evaluated in float (cpp_src/main_buryn.cpp:295-298)."""
    return float(np.float32(math.exp(float(np.float32(-1.0) * np.float32(dt) / np.float32(tau)))))


def triplet_params(dt: float, p: dict = EXAMPLE_TRIPLET, offset: int = 0) -> dict:
    return dict(ltp_A=p["ltp_A"], ltd_A=p["ltd_A"], ltp_B=p["ltp_B"], ltd_B=p["ltd_B"],
                pre_trace_decay=decay(dt, p["tau_ltp"]), post_trace_decay=decay(dt, p["tau_ltd"]),
                triplet_pre_trace_decay=decay(dt, p["triplet_tau_ltp"]),
                triplet_post_trace_decay=decay(dt, p["triplet_tau_ltd"]),
                weight_min=p["weight_min"], weight_max=p["weight_max"], plasticity_offset=offset)


def istdp_params(dt: float, p: dict = EXAMPLE_ISTDP, offset: int = 0) -> dict:
    return dict(ltp_A=p["ltp_A"], ltd_A=p["ltd_A"], ltd_B=p["ltd_B"], pre_trace_decay=decay(dt, p["tau_ltp"]),
                post_trace_decay=decay(dt, p["tau_ltd"]), weight_min=p["weight_min"], weight_max=p["weight_max"],
                plasticity_offset=offset)


WORKLOADS = {
    # 400 E (20x20) + 100 I (10x10), 9 grid points = 100 um, g_leak 10 nS, C 200 pF, 2 ms refractory,
    # Poisson background 5 kHz (0.5 per 0.1 ms step), triplet + iSTDP, one pulse into 20 E neurons.
    "small_plastic_500": dict(
        num_e=400, num_i=100, e_side=20, i_side=10, e_spacing=1.0, i_spacing=2.0, side=20.0, spread=81.0,
        steps=10001, seed=0, plastic=True, neuron=dict(g_leak=10e-9, membrane_capacitance=200e-12, refractory_steps=20,
                                                       mean_background_excitatory_spikes=0.5),
        tau=dict(rise_e=0.3e-3, decay_e=2e-3, rise_i=0.3e-3, decay_i=3e-3),
        stim=dict(n_ids=20, starts=[5000], ends=[6000], amp=0.25e-9), voltages=20),
    # The reference example network: 2,500 E (50x50) + 625 I (25x25), ~9.8 M dense FP32 synapse
    # entries, triplet STDP + iSTDP, 4 pulses of 0.5 nA, all spikes and 50 voltages recorded.
    "example_plastic_3125": dict(
        num_e=2500, num_i=625, e_side=50, i_side=25, e_spacing=1.0, i_spacing=2.0, side=50.0, spread=81.0,
        i_spread=324.0, steps=100001, seed=751, plastic=True, neuron={},
        tau=dict(rise_e=1e-3, decay_e=5e-3, rise_i=0.5e-3, decay_i=10e-3),
        stim=dict(n_ids=10, starts=[20000, 40000, 60000, 80000], ends=[22000, 42000, 62000, 82000], amp=0.5e-9),
        voltages=50),
    # Large network: 8,100 E (90x90) + 2,025 I (45x45), ~102 M dense synapse entries, plastic.
    "large_plastic_10125": dict(
        num_e=8100, num_i=2025, e_side=90, i_side=45, e_spacing=1.0, i_spacing=2.0, side=90.0, spread=81.0,
        i_spread=324.0, steps=50001, seed=751, plastic=True, neuron={},
        tau=dict(rise_e=1e-3, decay_e=5e-3, rise_i=0.5e-3, decay_i=10e-3),
        stim=dict(n_ids=10, starts=[20000], ends=[22000], amp=0.5e-9), voltages=50),
}


def synthetic_network(workload: str = "example_plastic_3125", *, steps: int | None = None, plastic: bool | None = None,
                      weight_values: str = "uniform", noise: bool = True, seed: int | None = None,
                      recording_interval_steps: int = 10000, scale_e: int | None = None) -> NetworkSpec:
    """Builds one of WORKLOADS (optionally resized with scale_e E neurons on a square grid)."""
    w = dict(WORKLOADS[workload])
    num_e, num_i = w["num_e"], w["num_i"]
    e_side, i_side, side = w["e_side"], w["i_side"], w["side"]
    if scale_e is not None:
        e_side = max(2, int(round(math.sqrt(scale_e))))
        i_side = max(1, e_side // 2)
        num_e, num_i, side = e_side * e_side, i_side * i_side, float(e_side)
    steps = w["steps"] if steps is None else steps
    plastic = w["plastic"] if plastic is None else plastic
    seed = w["seed"] if seed is None else seed
    dt = 1e-4
    spec = NetworkSpec(num_e, num_i, steps, rng_seed=seed, timestep=dt, recording_interval_steps=recording_interval_steps,
                       name=workload)
    neuron = dict(EXAMPLE)
    neuron.update(w["neuron"])
    if not noise:
        neuron.update(mean_background_excitatory_spikes=0.0, mean_background_inhibitory_spikes=0.0)
    spec.groups.append(dict(neuron, offset=0, num_neurons=num_e, is_inhibitory=False))
    spec.groups.append(dict(neuron, offset=num_e, num_neurons=num_i, is_inhibitory=True))
    e_loc = generation.generate_2d_grid_locations(num_e, w["e_spacing"], e_side, e_side)
    i_loc = generation.generate_2d_grid_locations(num_i, w["i_spacing"], i_side, i_side)
    e_spread = w["spread"]
    i_spread = w.get("i_spread", w["spread"])
    gen = [  # (pre, post, pre_loc, post_loc, max_w, prob, spread, no_diag)
        (0, 0, e_loc, e_loc, 1.5e-9, 0.2, e_spread, True),
        (0, 1, e_loc, i_loc, 1.5e-9, 0.6, e_spread, False),
        (1, 0, i_loc, e_loc, 5.0e-9, 0.6, i_spread, False),
        (1, 1, i_loc, i_loc, 5.0e-9, 0.6, i_spread, True),
    ]
    tau = w["tau"]
    for idx, (pre, post, pl, ql, max_w, prob, spread, no_diag) in enumerate(gen):
        wts = generation.distance_2d_weights(
            pl, ql, max_weight_value=max_w, max_distance=45.0, spread_scale=spread, weight_value_normal_dropoff=False,
            probabilistic_normal_not_uniform=True, probability_multiplier=prob, no_diagonal_connections=no_diag,
            x_location_length=side, y_location_length=side, rng_seed=seed + idx, value_mode=weight_values)
        rise, dec = (tau["rise_e"], tau["decay_e"]) if pre == 0 else (tau["rise_i"], tau["decay_i"])
        spec.conns.append(ConnSpec(pre, post, wts, dict(timestep=dt, decay_time=dec, rise_time=rise,
                                                        postsynaptic_kernel_normalization_value=1.7,
                                                        weight_matrix_idx=idx)))
    if plastic:
        spec.plasts.append(PlastSpec(PLASTICITY_TRIPLET, 0, triplet_params(dt, offset=0)))
        spec.plasts.append(PlastSpec(PLASTICITY_ISTDP, 2, istdp_params(dt, offset=1)))
    st = w["stim"]
    rng = np.random.default_rng(seed + 101)
    ids = np.sort(rng.choice(num_e, size=min(st["n_ids"], num_e), replace=False)).tolist()
    spec.stimulus = generation.partial_group_multiple_square_waves(
        steps, ids, [0] * len(ids), st["starts"], st["ends"], [st["amp"]])
    spec.monitors.append(MonSpec("spikes", 0))
    spec.monitors.append(MonSpec("spikes", 1))
    vids = tuple(np.sort(rng.choice(num_e, size=min(w["voltages"], num_e), replace=False)).tolist())
    spec.monitors.append(MonSpec("voltage", 0, vids))
    return spec


def random_network(num_e: int, num_i: int, *, steps: int = 200, seed: int = 0, density: float = 0.2,
                   plasticity=("triplet", "istdp"), noise: bool = True, stim_events: int = 6,
                   weight_scale: float = 1.0) -> NetworkSpec:
    """Small randomised networks for parity tests: random sparse-ish weights, the example's neuron
    parameters, strong enough drive that neurons spike within a few hundred steps."""
    rng = np.random.default_rng(seed)
    dt = 1e-4
    spec = NetworkSpec(num_e, num_i, steps, rng_seed=seed, timestep=dt, recording_interval_steps=64,
                       name=f"random_{num_e}_{num_i}")
    neuron = dict(EXAMPLE, mean_background_excitatory_spikes=0.3 if noise else 0.0,
                  mean_background_inhibitory_spikes=1.5 if noise else 0.0, refractory_steps=20)
    spec.groups.append(dict(neuron, offset=0, num_neurons=num_e, is_inhibitory=False))
    spec.groups.append(dict(neuron, offset=num_e, num_neurons=num_i, is_inhibitory=True))
    sizes = [num_e, num_i]
    taus = [(0.3e-3, 2e-3), (0.3e-3, 3e-3)]
    scales = [1.5e-9, 5e-9]
    idx = 0
    for pre in (0, 1):
        for post in (0, 1):
            w = (rng.random((sizes[pre], sizes[post]), dtype=np.float32) * np.float32(scales[pre] * weight_scale))
            w *= (rng.random(w.shape) < density).astype(np.float32)
            if pre == post:
                np.fill_diagonal(w, 0.0)
            rise, dec = taus[pre]
            spec.conns.append(ConnSpec(pre, post, w.astype(np.float32), dict(
                timestep=dt, decay_time=dec, rise_time=rise, postsynaptic_kernel_normalization_value=1.7,
                weight_matrix_idx=idx)))
            idx += 1
    off = 0
    if "triplet" in plasticity:
        spec.plasts.append(PlastSpec(PLASTICITY_TRIPLET, 0, triplet_params(
            dt, dict(EXAMPLE_TRIPLET, ltp_A=2e-12, ltp_B=4e-12, ltd_A=1e-12, ltd_B=1e-12), offset=off)))
        off += 1
    if "istdp" in plasticity:
        spec.plasts.append(PlastSpec(PLASTICITY_ISTDP, 2, istdp_params(dt, dict(EXAMPLE_ISTDP, ltd_B=0.2), offset=off)))
        off += 1
    if "stdp" in plasticity:
        spec.plasts.append(PlastSpec(PLASTICITY_STDP, 1, dict(
            ltp_A=2e-12, ltd_A=1e-12, pre_trace_decay=decay(dt, 20e-3), post_trace_decay=decay(dt, 20e-3),
            weight_min=0.0, weight_max=3e-9, plasticity_offset=off)))
        off += 1
    if stim_events:
        n_ids = max(1, min(num_e, stim_events))
        ids = np.sort(rng.choice(num_e, size=n_ids, replace=False)).tolist()
        spec.stimulus = generation.partial_group_multiple_square_waves(
            steps, ids, [0] * n_ids, [steps // 5], [steps // 2], [0.6e-9])
    spec.monitors.append(MonSpec("spikes", 0))
    spec.monitors.append(MonSpec("spikes", 1))
    spec.monitors.append(MonSpec("voltage", 0, tuple(range(0, num_e, max(1, num_e // 8)))))
    return spec
