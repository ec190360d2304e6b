"""Parity with the reference's own CUDA implementation on the bench's own networks: the example
network the headline is quoted on (2,500 E + 625 I, uniform[0, max_weight] weights, seed 751,
triplet STDP + iSTDP) and the large network (8,100 E + 2,025 I, ~102 M synapses) in the FP32
reference form.  oracle/_ref/ref_harness (the reference's cpp_src components built for sm_100a)
runs each for 1,000 steps and records the Poisson counts cuRAND drew; the CUDA path replays them,
so every input is identical.  Checked:

  * the spike rasters of all 1,000 steps: bit-identical;
  * at every 100th step, the background traces and conductances, refractory counters, stimulus
    current, connection traces x = d - r and plasticity traces: bit-identical;
  * membrane potentials and conductances at those steps, and the final weights, element by
    element: |a - b| <= 1e-5 (|b| + floor) with the floors of conftest.ELEMENT_FLOORS (the
    reference's cublasSgemv and its sequential row sums add in their own order, bsnn in a fixed
    order of its own, so only rounding separates them);
  * the same per-element figures are printed beside the bound."""
from __future__ import annotations

import numpy as np
import pytest

import bsnn
import refnet
from conftest import ELEMENT_FLOORS, assert_close_elementwise, elementwise_error

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refnet.HARNESS.exists(), reason="reference build (make -C oracle ref) absent")]

STEPS = 1000
EVERY = 100
RTOL = 1e-5
EXACT = ["i_stimulus", "refractory_counter", "background_g_excitatory", "background_g_inhibitory",
         "background_excitatory_r_traces", "background_excitatory_d_traces", "background_inhibitory_r_traces",
         "background_inhibitory_d_traces"]
CLOSE = ["membrane_potentials", "g_excitatory", "g_inhibitory"]


def raster_of(sim, spec, steps):
    out = np.zeros((steps, spec.num_neurons), np.uint8)
    for m, mon in enumerate(spec.monitors):
        if mon.kind == "spikes":
            off = spec.groups[mon.group]["offset"]
            hist = sim.read_spike_history(m)  # [neuron, slot]
            out[:, off:off + hist.shape[0]] = hist[:, :steps].T
    return out


@pytest.mark.parametrize("workload", ["example_plastic_3125", "large_plastic_10125"])
def test_bench_network_matches_reference_run(workload, tmp_path):
    spec = bsnn.synthetic_network(workload, steps=STEPS + 1, weight_values="uniform", recording_interval_steps=STEPS,
                                  seed=bsnn.network.WORKLOADS[workload]["seed"])
    states, ref_w, noise, ref_raster = refnet.run_dump(spec, STEPS, EVERY, tmp_path, raster=True)
    assert sorted(states) == list(range(EVERY - 1, STEPS, EVERY))
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    sim.set_noise_mode(bsnn.NOISE_REPLAY)
    sim.set_noise_replay(noise)
    worst = {f: 0.0 for f in CLOSE}
    done = 0
    for s in sorted(states):
        sim.run(done, s + 1 - done)
        done = s + 1
        want = states[s]
        for f in EXACT:
            got = sim.read(f)
            bad = np.flatnonzero(got != want[f])
            assert bad.size == 0, f"step {s} {f}: {bad.size} differ, first {bad[:5]}"
        for c in range(len(spec.conns)):
            assert np.array_equal(sim.read("connection_summed", c), want["summed"][c]), f"step {s} summed[{c}]"
        for p, pl in enumerate(spec.plasts):
            conn = spec.conns[pl.conn]
            pre_off, post_off = spec.groups[conn.pre]["offset"], spec.groups[conn.post]["offset"]
            n_pre, n_post = conn.weights.shape
            k = pl.params["plasticity_offset"]
            assert np.array_equal(sim.read("plasticity_pre_traces", p, count=n_pre),
                                  want["pre_traces"][k, pre_off:pre_off + n_pre]), f"step {s} pre traces[{p}]"
            assert np.array_equal(sim.read("plasticity_post_traces", p, count=n_post),
                                  want["post_traces"][k, post_off:post_off + n_post]), f"step {s} post traces[{p}]"
        for f in CLOSE:
            got = sim.read(f)
            worst[f] = max(worst[f], elementwise_error(got, want[f], ELEMENT_FLOORS[f])[0])
            assert_close_elementwise(got, want[f], RTOL, ELEMENT_FLOORS[f], f"step {s} {f}")
    got_raster = raster_of(sim, spec, STEPS)
    diff = np.argwhere(got_raster != ref_raster)
    assert diff.size == 0, f"{workload}: spike rasters differ at (step, neuron) {diff[:5].tolist()}"
    n_spikes = int(ref_raster.sum())
    wmax = 0.0
    for c in range(len(spec.conns)):
        got = sim.read_weights(c)
        wmax = max(wmax, elementwise_error(got, ref_w[c], ELEMENT_FLOORS["weights"])[0])
        assert_close_elementwise(got, ref_w[c], RTOL, ELEMENT_FLOORS["weights"], f"weights[{c}]")
    sim.close()
    print(f"{workload}: {n_spikes} spikes in {STEPS} steps, rasters identical; largest per-element relative "
          f"error: " + ", ".join(f"{f} {e:.2e}" for f, e in worst.items()) + f", weights {wmax:.2e}")
    assert n_spikes > 0
