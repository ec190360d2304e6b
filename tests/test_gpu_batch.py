"""GPU: the batched form (bsnn_batch_*) against the CPU oracle, instance by instance.

Each instance of a batch is an ordinary network whose weights are its class's weights rounded to
BF16 (`BatchSpec.instance_network`).  The batch computes the propagation on the tensor cores from
the BF16 weights and the traces split into BF16 high and low parts (x = hi + lo to about 2^-17)
with FP32 accumulation, so against the FP32 oracle run on the same BF16-valued weights it agrees
to within 2e-5 relative (to the field's largest magnitude) in g, v and the traces over the first
steps, with identical spikes and refractory counters.  Over longer runs (chaotic divergence), the
population spike counts are compared instead.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import bsnn
import oracle
from conftest import assert_close

pytestmark = pytest.mark.gpu

RTOL = 2e-5
FIELDS = ["membrane_potentials", "g_excitatory", "g_inhibitory", "i_stimulus", "background_g_excitatory",
          "background_g_inhibitory",
          "background_excitatory_r_traces", "background_excitatory_d_traces", "connection_summed"]


def oracle_for(spec, b, precision=oracle.PREC_F32):
    net = spec.instance_network(b)
    o = oracle.OracleSimulation(net.num_excitatory, net.num_inhibitory, precision=precision, **net.sim_kwargs())
    net.build(o)
    return o, net


def oracle_field(o, net, name):
    if name == "connection_summed":  # the neuron's own presynaptic trace: E from conn 0, I from conn 2
        return np.concatenate([o.read(name, 0), o.read(name, 2)])
    return o.read(name)


def compare_instance(g, b, o, net, tag):
    np.testing.assert_array_equal(g.read(b, "spikes"), o.read("spikes"), err_msg=f"{tag} spikes")
    np.testing.assert_array_equal(g.read(b, "refractory_counter"), o.read("refractory_counter"), err_msg=f"{tag} refrac")
    for f in FIELDS:
        assert_close(g.read(b, f), oracle_field(o, net, f), RTOL, f"{tag} {f}")


@pytest.mark.parametrize("noise", [True, False])
def test_batch_matches_the_oracle_over_the_first_steps(noise):
    spec = bsnn.config4_batch(n_instances=5, steps=400, seed=3, sizes=(400, 900), stim_window=(5, 300))
    g = bsnn.BatchSimulation(spec, noise=noise)
    info = g.info()
    assert info.num_instances == 5 and info.num_classes == len(spec.classes)
    oracles = []
    for b in range(len(spec.instances)):
        o, net = oracle_for(spec, b)
        if not noise:
            o.set_noise_mode(bsnn.NOISE_OFF)
        oracles.append((o, net))
    done = 0
    for block in (1, 9, 30):
        g.run(block)
        for o, _ in oracles:
            o.run(done, block)
        done += block
        for b, (o, net) in enumerate(oracles):
            compare_instance(g, b, o, net, f"instance {b} after {done} steps")
    g.close()


def test_batch_launch_split_and_spike_counts():
    """The same batch in one launch and in launches of 7 steps gives the same state bit for bit;
    the spike counter agrees with the oracle's spike history."""
    spec = bsnn.config4_batch(n_instances=4, steps=300, seed=5, sizes=(400, 900), stim_window=(10, 200))
    a = bsnn.BatchSimulation(spec)
    a.run(120)
    b = bsnn.BatchSimulation(spec)
    b.set_steps_per_launch(7)
    b.run(120)
    for k in range(4):
        for f in ("membrane_potentials", "g_excitatory", "connection_summed"):
            np.testing.assert_array_equal(a.read(k, f), b.read(k, f), err_msg=f)
    np.testing.assert_array_equal(a.spike_counts(), b.spike_counts())
    counts = a.spike_counts()
    for k in range(2):
        o, net = oracle_for(spec, k)
        total = np.zeros(2, np.int64)
        for t in range(60):  # spike counts over the first 60 steps, step by step
            o.step(t)
            s = o.read("spikes")
            total += [int(s[: net.num_excitatory].sum()), int(s[net.num_excitatory:].sum())]
        c = bsnn.BatchSimulation(spec)
        c.run(60)
        np.testing.assert_array_equal(c.spike_counts()[k], total)
        c.close()
    assert counts.sum() > 0
    a.close()
    b.close()


def test_batch_rates_against_fp64():
    """Population rates over 2,000 steps against the FP64 oracle for a few instances; the bound is
    stated per instance and population (relative, or 2 spikes for near-silent populations)."""
    spec = bsnn.config4_batch(n_instances=6, steps=2000, seed=7, sizes=(400, 900, 1600), stim_window=(200, 1500))
    g = bsnn.BatchSimulation(spec)
    g.run(2000)
    counts = g.spike_counts().astype(np.int64)
    worst = 0.0
    for b in range(3):
        o, net = oracle_for(spec, b, precision=oracle.PREC_F64)
        o.run(0, 2000)
        ref = np.array([int(o.read_spike_history(0).sum()), int(o.read_spike_history(1).sum())])
        for p in range(2):
            err = abs(counts[b, p] - ref[p]) / max(ref[p], 1)
            print(f"instance {b} pop {p}: {counts[b, p]} spikes vs FP64 {ref[p]}")
            assert abs(counts[b, p] - ref[p]) <= max(2, 0.05 * ref[p]), (b, p, counts[b, p], ref[p])
            if ref[p] > 100:
                worst = max(worst, err)
    print(f"largest relative rate error (populations with > 100 spikes): {worst:.2e}")
    g.close()


@pytest.mark.parametrize("env", [{"BSNN_BATCH_STATE": "global"}, {"BSNN_BATCH_STAGES": "2"},
                                 {"BSNN_BATCH_STATE": "global", "BSNN_BATCH_STAGES": "4"},
                                 {"BSNN_BATCH_STAGES": "8"}, {"BSNN_BATCH_CLASSWAIT": "0"}])
def test_batch_placements_are_bit_exact(env):
    """Neuron state in shared memory (the default when it fits) or in global memory, the operand
    ring's depth, and per-class waits (the default) or grid barriers between the phases change
    where data lives and when work starts, not the arithmetic: the states are identical."""
    spec = bsnn.config4_batch(n_instances=6, steps=200, seed=9, sizes=(400, 900, 1600), stim_window=(10, 150))
    a = bsnn.BatchSimulation(spec)
    ia = a.info()
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        b = bsnn.BatchSimulation(spec)
        ib = b.info()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    assert ia.state_in_smem == 1
    assert ib.state_in_smem == (0 if env.get("BSNN_BATCH_STATE") == "global" else 1)
    if "BSNN_BATCH_STAGES" in env:
        assert ib.operand_stages == int(env["BSNN_BATCH_STAGES"])
    for sim in (a, b):
        sim.set_steps_per_launch(37)
        sim.run(150)
    for k in range(len(spec.instances)):
        for f in FIELDS + ["spikes", "refractory_counter"]:
            np.testing.assert_array_equal(a.read(k, f), b.read(k, f), err_msg=f"instance {k} {f}")
    np.testing.assert_array_equal(a.spike_counts(), b.spike_counts())
    a.close()
    b.close()


@pytest.mark.parametrize("env", [{}, {"BSNN_BATCH_STATE": "global"}, {"BSNN_BATCH_STAGES": "2"}])
def test_batch_forms_are_bit_exact(env):
    """The flow form (each size class its own chain of neuron updates and GEMM units, no grid
    barriers) and the phased form do the same arithmetic in another order of work: states and
    spike counts are identical, over launches that end in the middle of the classes' chains."""
    spec = bsnn.config4_batch(n_instances=9, steps=200, seed=10, sizes=(400, 900, 1600), stim_window=(10, 150))
    assert len({i.cls for i in spec.instances}) == 3
    a = bsnn.BatchSimulation(spec, form="phased")
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        b = bsnn.BatchSimulation(spec, form="flow")
        ib = b.info()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    assert a.info().form == 1 and ib.form == 0
    for sim, per in ((a, 150), (b, 23)):
        sim.set_steps_per_launch(per)
        sim.run(150)
    for k in range(len(spec.instances)):
        for f in FIELDS + ["spikes", "refractory_counter"]:
            np.testing.assert_array_equal(a.read(k, f), b.read(k, f), err_msg=f"instance {k} {f}")
    np.testing.assert_array_equal(a.spike_counts(), b.spike_counts())
    assert b.spike_counts().sum() > 0
    a.close()
    b.close()


def test_batch_rate_error_over_a_simulated_second():
    """10,000 clock steps (1 simulated second) of four instances against the FP64 oracle on the same
    BF16-valued weights: the aggregate spike count of the populations is within 1e-3 relative,
    each population within 5e-3.  For scale, the FP32 oracle (the reference's arithmetic) on one
    instance is printed beside it: trajectories of this chaotic network separate after a few
    hundred steps in any precision, so a per-population difference of this order is the floor."""
    T = 10000
    spec = bsnn.config4_batch(n_instances=4, steps=T, seed=7, sizes=(400, 900), stim_window=(1000, 4000))
    g = bsnn.BatchSimulation(spec)
    g.run(T)
    counts = g.spike_counts().astype(np.int64)
    g.close()
    tot_b = tot_r = 0
    for b in range(len(spec.instances)):
        o, _ = oracle_for(spec, b, precision=oracle.PREC_F64)
        o.run(0, T)
        ref = [int(o.read_spike_history(0).sum()), int(o.read_spike_history(1).sum())]
        for p in range(2):
            err = abs(counts[b, p] - ref[p]) / max(ref[p], 1)
            print(f"instance {b} pop {p}: {counts[b, p]} spikes vs FP64 {ref[p]} (relative {err:.1e})")
            assert err <= 5e-3, (b, p, counts[b, p], ref[p])
            tot_b += counts[b, p]
            tot_r += ref[p]
        if b == 0:
            o32, _ = oracle_for(spec, b, precision=oracle.PREC_F32)
            o32.run(0, T)
            f32 = [int(o32.read_spike_history(0).sum()), int(o32.read_spike_history(1).sum())]
            print(f"  FP32 oracle on instance 0: {f32} (relative {abs(f32[0] - ref[0]) / ref[0]:.1e}, "
                  f"{abs(f32[1] - ref[1]) / ref[1]:.1e})")
    agg = abs(tot_b - tot_r) / tot_r
    print(f"aggregate: {tot_b} vs FP64 {tot_r} (relative {agg:.1e})")
    assert agg <= 1e-3


def test_autotune_keeps_a_valid_choice():
    """The autotuner times its candidates, leaves the batch at step 0 with the fastest shapes, and
    the tuned batch still matches the oracle; it refuses to run after the first step."""
    spec = bsnn.config4_batch(n_instances=5, steps=400, seed=3, sizes=(400, 900), stim_window=(5, 300))
    g = bsnn.BatchSimulation(spec)
    r = g.autotune(40)
    print(r)
    assert r["candidates"] >= 3 and 0 < r["us_per_step"] <= r["default_us_per_step"]
    assert 2 <= r["operand_stages"] <= 8 and r["k_tiles_per_unit"] >= 1
    assert g.info().steps_done == 0
    oracles = [oracle_for(spec, b) for b in range(len(spec.instances))]
    g.run(30)
    for o, _ in oracles:
        o.run(0, 30)
    for b, (o, net) in enumerate(oracles):
        compare_instance(g, b, o, net, f"tuned instance {b}")
    with pytest.raises(bsnn.StateError):
        g.autotune(40)
    h = bsnn.BatchSimulation(spec)
    h.set_tuning(r)
    h.run(30)
    for b in range(len(spec.instances)):
        np.testing.assert_array_equal(g.read(b, "membrane_potentials"), h.read(b, "membrane_potentials"))
    g.close()
    h.close()
