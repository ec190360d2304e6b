"""Parity with the reference's own CUDA implementation, through the golden fixtures of
tests/golden/ (recorded by tests/golden/make_golden.py from the reference's cpp_src components
built for sm_100a).  Each fixture holds the Poisson counts the reference drew, so with the noise
replayed every input is identical and the comparison is step by step:

  * spike rasters: bit-identical at every one of the 1,000 recorded steps;
  * background traces and conductances, stimulus current, refractory counters, connection traces
    (x = d - r) and plasticity traces: bit-identical (they depend on spikes and noise only);
  * membrane potentials, conductances and the final weights: within 1e-5 x max|reference| of the
    field, and element by element within 1e-5 of each value (|a - b| <= 1e-5 (|b| + floor), the
    floors of conftest.ELEMENT_FLOORS) (the reference's cublasSgemv sums in float in its own
    order; the oracle sums in double, the CUDA path in float in a fixed order).

The CPU test pins the oracle to the reference; the GPU test runs the CUDA path through the C-ABI.
"""
from __future__ import annotations

import json
import sys

import numpy as np
import pytest

import bsnn
from conftest import ELEMENT_FLOORS, ROOT, assert_close, assert_close_elementwise

sys.path.insert(0, str(ROOT / "tests" / "golden"))
from specs import CHECK_STEPS, GOLDEN_STEPS, golden_specs, spec_digest  # noqa: E402

GOLDEN = ROOT / "tests" / "golden"
NAMES = ["small_plastic_500", "random_120_all_rules"]
RTOL = 1e-5
EXACT_FIELDS = ["i_stimulus", "refractory_counter", "background_g_excitatory", "background_g_inhibitory",
                "background_excitatory_r_traces", "background_excitatory_d_traces", "background_inhibitory_r_traces",
                "background_inhibitory_d_traces"]
CLOSE_FIELDS = ["membrane_potentials", "g_excitatory", "g_inhibitory"]


def load(name):
    fx = dict(np.load(GOLDEN / f"{name}.npz"))
    spec = golden_specs()[name]
    assert str(fx["digest"]) == spec_digest(spec), "network generators no longer reproduce the fixture's inputs"
    meta = json.loads(str(fx["meta"]))
    assert meta["steps"] == GOLDEN_STEPS and tuple(meta["check_steps"]) == CHECK_STEPS
    return fx, spec


def raster_from_monitors(sim, spec):
    """[steps, N] 0/1 from the two spike recorders (groups 0 and 1, one slot per step)."""
    cols = []
    for m, mon in enumerate(spec.monitors):
        if mon.kind == "spikes":
            cols.append((spec.groups[mon.group]["offset"], sim.read_spike_history(m)))
    raster = np.zeros((GOLDEN_STEPS, spec.num_neurons), np.uint8)
    for off, hist in cols:  # hist [neuron, slot]
        raster[:, off:off + hist.shape[0]] = hist[:, :GOLDEN_STEPS].T
    return raster


def compare(sim, spec, fx, name):
    """Runs the replayed network to each check step, compares the state, then the raster and weights."""
    done = 0
    for k, s in enumerate(CHECK_STEPS):
        sim.run(done, s + 1 - done)
        done = s + 1
        sim.synchronize()
        tag = f"{name} step {s}"
        for f in EXACT_FIELDS:
            got, want = sim.read(f), fx[f"state_{f}"][k]
            bad = np.flatnonzero(got != want)
            assert bad.size == 0, f"{tag} {f}: {bad.size} differ, first {bad[:5]}: {got[bad[:5]]} vs {want[bad[:5]]}"
        for f in CLOSE_FIELDS:
            assert_close(sim.read(f), fx[f"state_{f}"][k], RTOL, f"{tag} {f}")
            assert_close_elementwise(sim.read(f), fx[f"state_{f}"][k], RTOL, ELEMENT_FLOORS[f], f"{tag} {f}")
        for c in range(len(spec.conns)):
            got, want = sim.read("connection_summed", c), fx[f"summed_{c}"][k]
            assert np.array_equal(got, want), f"{tag} summed[{c}] differs"
        for p, pl in enumerate(spec.plasts):
            conn = spec.conns[pl.conn]
            pre_off, post_off = spec.groups[conn.pre]["offset"], spec.groups[conn.post]["offset"]
            n_pre, n_post = conn.weights.shape
            want_pre = fx["pre_traces"][k, pl.params["plasticity_offset"], pre_off:pre_off + n_pre]
            want_post = fx["post_traces"][k, pl.params["plasticity_offset"], post_off:post_off + n_post]
            assert np.array_equal(sim.read("plasticity_pre_traces", p, count=n_pre), want_pre), f"{tag} pre[{p}]"
            assert np.array_equal(sim.read("plasticity_post_traces", p, count=n_post), want_post), f"{tag} post[{p}]"
    want_raster = np.unpackbits(fx["spikes"], axis=1)[:, :spec.num_neurons]
    got_raster = raster_from_monitors(sim, spec)
    diff = np.argwhere(got_raster != want_raster)
    assert diff.size == 0, f"{name}: spike rasters differ at (step, neuron) {diff[:5].tolist()}"
    assert want_raster.sum() > 0, "fixture has no spikes"
    for c in range(len(spec.conns)):
        assert_close(sim.read_weights(c), fx[f"weights_{c}"], RTOL, f"{name} weights[{c}]")
        assert_close_elementwise(sim.read_weights(c), fx[f"weights_{c}"], RTOL, ELEMENT_FLOORS["weights"],
                                 f"{name} weights[{c}]")


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_run(oracle_mod, name):
    fx, spec = load(name)
    o = oracle_mod.OracleSimulation(spec.num_excitatory, spec.num_inhibitory, precision=32, **spec.sim_kwargs())
    spec.build(o)
    o.set_noise_mode(bsnn.NOISE_REPLAY)
    o.set_noise_replay(fx["noise"])
    compare(o, spec, fx, name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_path_matches_reference_run(name):
    fx, spec = load(name)
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    sim.set_noise_mode(bsnn.NOISE_REPLAY)
    sim.set_noise_replay(fx["noise"])
    compare(sim, spec, fx, name)
    sim.close()
