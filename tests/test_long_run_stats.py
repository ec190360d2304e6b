"""Long-run statistics against the reference's own CUDA implementation (oracle/_ref/ref_harness,
the reference's cpp_src components built for sm_100a), on the example network (2,500 E + 625 I,
the reference generator's weights, triplet STDP + iSTDP) over 20,001 clock steps (2 simulated
seconds), with the reference's Poisson counts replayed.  Individual spikes diverge once the
network's chaotic dynamics amplify last-bit differences, so the run is compared through:

  * the spike rows of the first 1,000 steps: identical, neuron for neuron;
  * per-population firing rates: within 10 % of the reference's;
  * the coefficient of variation of the inter-spike intervals (pooled per population): within 15 %;
  * the histogram of the final plastic weights (E->E, I->E): total-variation distance < 0.02 over
    50 bins, means and standard deviations within 1e-3 relative.

Both rasters come from the recorders' text files (SpikeRecorder format), written by
bsnn_run_system and by the reference's System::run loop."""
from __future__ import annotations

import sys

import numpy as np
import pytest

import bsnn
from conftest import ROOT

sys.path.insert(0, str(ROOT / "oracle"))
import refnet  # noqa: E402

pytestmark = pytest.mark.gpu
STEPS = 20001


def rates_and_cv(rows, n_neurons, steps, dt=1e-4):
    """Rate (Hz per neuron) and pooled ISI CV of one population from {step: [ids]}."""
    times = [[] for _ in range(n_neurons)]
    for step, ids in rows.items():
        for i in ids:
            times[i].append(step)
    n_spikes = sum(len(t) for t in times)
    isis = np.concatenate([np.diff(np.sort(t)) for t in times if len(t) > 1] or [np.zeros(0)])
    cv = float(isis.std() / isis.mean()) if isis.size > 1 else float("nan")
    return n_spikes / (n_neurons * (steps - 1) * dt), cv, n_spikes


@pytest.mark.skipif(not refnet.HARNESS.exists(), reason="reference build (make -C oracle ref) not present")
def test_long_run_statistics_match_reference(tmp_path):
    spec = bsnn.synthetic_network("example_plastic_3125", steps=STEPS + 1, weight_values="reference",
                                  recording_interval_steps=10000)
    ref_dir = tmp_path / "ref"
    noise, ref_w = refnet.run_record(spec, STEPS, ref_dir)

    ours = tmp_path / "ours"
    ours.mkdir()
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    sim.set_noise_mode(bsnn.NOISE_REPLAY)
    sim.set_noise_replay(noise)
    sim.set_monitor_output(0, ours / "spikes_m0.txt")
    sim.set_monitor_output(1, ours / "spikes_m1.txt")
    sim.run_system(STEPS)
    sim.flush_records()
    our_w = [sim.read_weights(c) for c in range(len(spec.conns))]
    sim.close()

    for m, n in ((0, spec.num_excitatory), (1, spec.num_inhibitory)):
        ref_rows = refnet.read_spike_rows(ref_dir / f"spikes_m{m}.txt")
        our_rows = refnet.read_spike_rows(ours / f"spikes_m{m}.txt")
        assert sorted(ref_rows) == sorted(our_rows) == list(range(STEPS - 1))
        # the first 1,000 steps spike for spike, before chaos can part the runs
        first = [t for t in range(1000) if ref_rows[t] != our_rows[t]]
        assert not first, f"population {m}: spike rows differ at steps {first[:5]}"
        assert sum(len(ref_rows[t]) for t in range(1000)) > 0
        r_ref, cv_ref, n_ref = rates_and_cv(ref_rows, n, STEPS)
        r_our, cv_our, n_our = rates_and_cv(our_rows, n, STEPS)
        print(f"population {m}: rate {r_our:.4f} Hz vs reference {r_ref:.4f} Hz ({n_our} vs {n_ref} spikes), "
              f"ISI CV {cv_our:.4f} vs {cv_ref:.4f}")
        assert n_ref > 100, f"population {m}: too few reference spikes ({n_ref}) for a rate comparison"
        assert abs(r_our - r_ref) <= 0.10 * r_ref, (m, r_our, r_ref)
        if np.isfinite(cv_ref):
            assert abs(cv_our - cv_ref) <= 0.15 * cv_ref, (m, cv_our, cv_ref)
    for p in spec.plasts:
        a, b = our_w[p.conn].ravel().astype(np.float64), ref_w[p.conn].ravel().astype(np.float64)
        hi = max(a.max(), b.max())
        ha, _ = np.histogram(a, bins=50, range=(0.0, hi))
        hb, _ = np.histogram(b, bins=50, range=(0.0, hi))
        tv = 0.5 * np.abs(ha / a.size - hb / b.size).sum()
        print(f"connection {p.conn}: weight histogram TV distance {tv:.5f}, mean {a.mean():.6e} vs {b.mean():.6e}, "
              f"std {a.std():.6e} vs {b.std():.6e}")
        assert tv < 0.02, (p.conn, tv)
        np.testing.assert_allclose(a.mean(), b.mean(), rtol=1e-3)
        np.testing.assert_allclose(a.std(), b.std(), rtol=1e-3)
