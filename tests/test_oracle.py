"""CPU tests of the oracle itself: Philox4x32-10 known-answer vectors, the Poisson sampler, and
semantic properties of the reference step that the oracle must reproduce."""
from __future__ import annotations

import math

import numpy as np
import pytest

import bsnn
from bsnn.network import EXAMPLE, NetworkSpec, ConnSpec, MonSpec


# Random123 known-answer vectors for philox4x32-10 (counter, key -> output).
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(oracle_mod, ctr, key, want):
    assert oracle_mod.philox4x32_10(ctr, key) == want


@pytest.mark.parametrize("mean", [0.02, 0.5, 1.5, 7.0])
def test_poisson_moments(oracle_mod, mean):
    L = float(np.float32(math.exp(-mean)))
    xs = np.array([oracle_mod.poisson(L, 751, n, s, 1) for n in range(200) for s in range(100)], dtype=np.float64)
    se = math.sqrt(mean / xs.size)
    assert abs(xs.mean() - mean) < 5 * se + 1e-3
    assert abs(xs.var() - mean) < 0.1 * mean + 0.01


def test_poisson_zero_probability(oracle_mod):
    # P(0) = exp(-mean)
    mean = 1.5
    L = float(np.float32(math.exp(-mean)))
    xs = np.array([oracle_mod.poisson(L, 3, n, s, 0) for n in range(300) for s in range(100)])
    assert abs((xs == 0).mean() - math.exp(-mean)) < 0.01


def test_poisson_streams_are_keyed(oracle_mod):
    L = float(np.float32(math.exp(-1.5)))
    a = [oracle_mod.poisson(L, 7, 5, s, 0) for s in range(64)]
    b = [oracle_mod.poisson(L, 7, 5, s, 1) for s in range(64)]
    c = [oracle_mod.poisson(L, 8, 5, s, 0) for s in range(64)]
    assert a != b and a != c
    assert a == [oracle_mod.poisson(L, 7, 5, s, 0) for s in range(64)]


def one_group_spec(n=4, steps=200, **neuron):
    spec = NetworkSpec(n, 0, steps, rng_seed=1, recording_interval_steps=16)
    p = dict(EXAMPLE, mean_background_excitatory_spikes=0.0, mean_background_inhibitory_spikes=0.0)
    p.update(neuron)
    spec.groups.append(dict(p, offset=0, num_neurons=n, is_inhibitory=False))
    return spec


def oracle_for(spec, precision=32):
    import oracle
    return spec.build(oracle.OracleSimulation(spec.num_excitatory, spec.num_inhibitory, precision=precision,
                                              **spec.sim_kwargs()))


def test_relaxes_to_eif_fixed_point_without_input():
    # From v_rest the exponential term alone drives v up to the EIF fixed point just above rest:
    # gL*(v - EL) = gL*dT*exp((v - VT)/dT), about 1.8 mV above EL for the example parameters.
    spec = one_group_spec()
    o = oracle_for(spec)
    vs = []
    for s in range(400):
        o.step(s)
        vs.append(o.read("membrane_potentials")[0])
    vs = np.array(vs, np.float64)
    assert np.all(np.diff(vs) >= 0) and o.read("spikes").sum() == 0
    el, vt, dT = EXAMPLE["v_rest"], EXAMPLE["v_effective_spike_threshold"], EXAMPLE["depolarization_slope_factor"]
    v = el
    for _ in range(200):  # fixed point by iteration
        v = el + dT * math.exp((v - vt) / dT)
    assert abs(vs[-1] - v) < 1e-5


def test_refractory_holds_reset_for_refractory_steps():
    spec = one_group_spec(n=1, refractory_steps=7)
    o = oracle_for(spec)
    o.write("membrane_potentials", [-0.030])  # above threshold: spikes at the first step
    o.step(0)
    assert o.read("spikes")[0] == 1 and o.read("refractory_counter")[0] == 7
    assert o.read("membrane_potentials")[0] == np.float32(EXAMPLE["v_threshold"])
    for k in range(7):
        o.step(1 + k)
        assert o.read("spikes")[0] == 0
        assert o.read("membrane_potentials")[0] == np.float32(EXAMPLE["v_reset"])
        assert o.read("refractory_counter")[0] == 6 - k


def test_stimulus_acts_from_the_next_step():
    steps = 40
    spec = one_group_spec(n=2, steps=steps)
    from bsnn import generation
    spec.stimulus = generation.partial_group_multiple_square_waves(steps, [1], [0], [10], [19], [0.5e-9])
    o = oracle_for(spec)
    istim = []
    v = []
    for s in range(steps):
        o.step(s)
        istim.append(o.read("i_stimulus")[1])
        v.append(o.read("membrane_potentials"))
    istim = np.array(istim)
    assert np.all(istim[:10] == 0) and np.all(istim[10:20] == np.float32(0.5e-9)) and np.all(istim[20:] == 0)
    v = np.array(v)
    assert np.all(v[:11, 1] == v[:11, 0])  # step 10 still integrates with I = 0
    assert v[11, 1] > v[11, 0]


def test_trace_impulse_response_is_difference_of_exponentials():
    # two E neurons, 0 -> 1; neuron 0 spikes once at step 0
    spec = one_group_spec(n=2, steps=100)
    w = np.zeros((2, 2), np.float32)
    w[0, 1] = 1e-9
    spec.conns.append(ConnSpec(0, 0, w, dict(timestep=1e-4, decay_time=2e-3, rise_time=0.3e-3,
                                            postsynaptic_kernel_normalization_value=1.7, weight_matrix_idx=0)))
    o = oracle_for(spec)
    o.write("membrane_potentials", [-0.030, np.float32(EXAMPLE["v_rest"])])
    rd = np.float32(math.exp(np.float32(-1e-4) / np.float32(0.3e-3)))
    dd = np.float32(math.exp(np.float32(-1e-4) / np.float32(2e-3)))
    r = d = np.float32(0.0)
    for s in range(60):
        o.step(s)
        r = np.float32(r * rd); d = np.float32(d * dd)
        r = np.float32(0) if r < np.float32(1e-30) else r
        d = np.float32(0) if d < np.float32(1e-30) else d
        if s == 0:
            r = np.float32(r + np.float32(1.7)); d = np.float32(d + np.float32(1.7))
        assert o.read("connection_r_traces", 0)[0] == r
        assert o.read("connection_d_traces", 0)[0] == d
        assert o.read("connection_summed", 0)[0] == np.float32(d - r)


def test_triplet_targets_are_initial_column_sums(oracle_mod):
    spec = bsnn.random_network(12, 4, steps=5, seed=3)
    o = oracle_for(spec)
    w = spec.conns[0].weights
    want = np.array([np.float32(sum(np.float32(w[i, q]) for i in range(w.shape[0]))) for q in range(w.shape[1])],
                    np.float32)
    # column sums accumulated in float in ascending pre order, used as targets for the rows
    np.testing.assert_array_equal(o.read("plasticity_pre_weight_sums", 0), want[:w.shape[0]])


def test_triplet_normalises_rows_to_targets():
    spec = bsnn.random_network(40, 10, steps=50, seed=4)
    o = oracle_for(spec)
    o.run(0, 50)
    w = o.read_weights(0).astype(np.float64)
    targets = o.read("plasticity_pre_weight_sums", 0).astype(np.float64)
    rows = w.sum(axis=1)
    ok = rows > 0
    np.testing.assert_allclose(rows[ok], targets[ok], rtol=2e-5)


def test_f32_and_f64_oracles_agree_short_horizon():
    spec = bsnn.random_network(60, 15, steps=40, seed=5)
    a = oracle_for(spec, 32)
    b = oracle_for(spec, 64)
    a.run(0, 40)
    b.run(0, 40)
    np.testing.assert_array_equal(a.read("spikes"), b.read("spikes"))
    np.testing.assert_allclose(a.read("membrane_potentials"), b.read_f64("membrane_potentials"), rtol=1e-5)


def test_stimulus_overflow_is_rejected(oracle_mod):
    spec = one_group_spec(n=2, steps=10)
    counts = np.zeros(10, np.uint32)
    counts[3] = 5
    o = oracle_mod.OracleSimulation(2, 0, total_simulation_length=10, num_stimulus_events=2, recording_interval_steps=16)
    spec.build(o)
    o.add_stimulus(counts, [0, 1], [0, 0], [1e-9, 1e-9])
    o.run(0, 3)
    with pytest.raises(RuntimeError):
        o.step(3)


def test_connection_propagate_restatement(oracle_mod):
    """or_connection_propagate against numpy: trace arithmetic bit-exact in float32, the GEMV
    within double-precision rounding of a float64 matrix-vector product."""
    rng = np.random.default_rng(11)
    n_pre, n_post = 37, 29
    w = rng.uniform(0, 2, (n_pre, n_post)).astype(np.float32)
    r = rng.uniform(0, 1, n_pre).astype(np.float32)
    d = rng.uniform(0, 1, n_pre).astype(np.float32)
    r[:3] = 1e-31  # decays below the 1e-30 flush threshold
    x = np.zeros(n_pre, np.float32)
    g = rng.uniform(0, 1, n_post).astype(np.float32)
    spikes = (rng.random(n_pre) < 0.3).astype(np.uint32)
    rd, dd, norm = np.float32(0.9), np.float32(0.97), np.float32(1.25)
    want_d = d * dd
    want_d[want_d < np.float32(1e-30)] = 0
    want_r = r * rd
    want_r[want_r < np.float32(1e-30)] = 0
    want_r = np.where(spikes == 1, want_r + norm, want_r).astype(np.float32)
    want_d = np.where(spikes == 1, want_d + norm, want_d).astype(np.float32)
    want_x = want_d - want_r
    want_g = (w.astype(np.float64).T @ want_x.astype(np.float64)).astype(np.float32) + g
    oracle_mod.connection_propagate(rd, dd, norm, w, r, d, x, g, spikes)
    assert np.array_equal(r, want_r) and np.array_equal(d, want_d) and np.array_equal(x, want_x)
    assert r[0] == 0 or spikes[0] == 1
    np.testing.assert_allclose(g, want_g, rtol=1e-6)
