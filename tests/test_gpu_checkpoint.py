"""GPU: checkpoint / resume of the single-network engine (bsnn_save_checkpoint /
bsnn_load_checkpoint).

A run that is checkpointed, continued in a fresh simulation built from the same description and
compared with the uninterrupted run is bit-identical: every state field, every connection's
weights and traces, every plasticity trace and the monitor rings.  Loading into a differently
built simulation is refused.
"""
from __future__ import annotations

import numpy as np
import pytest

import bsnn
from conftest import FLOAT_FIELDS

pytestmark = pytest.mark.gpu


def build(spec, weight_format=None):
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    if weight_format:
        sim.set_weight_format(weight_format)
    return sim


def snapshot(sim, spec):
    out = {f: sim.read(f) for f in FLOAT_FIELDS + ["refractory_counter", "spikes"]}
    for c in range(len(spec.conns)):
        out[f"w{c}"] = sim.read_weights(c)
        for f in ("connection_r_traces", "connection_d_traces"):
            out[f"{f}{c}"] = sim.read(f, c)
    for k, p in enumerate(spec.plasts):
        n_pre, n_post = spec.conns[p.conn].weights.shape
        out[f"pre{k}"] = sim.read("plasticity_pre_traces", k, count=n_pre)
        out[f"post{k}"] = sim.read("plasticity_post_traces", k, count=n_post)
    for m in range(len(spec.monitors)):
        if spec.monitors[m].kind == "spikes":
            out[f"mon{m}"] = sim.read_spike_history(m)
    return out


@pytest.mark.parametrize("weight_format", [None, "bf16"])
def test_resume_is_bit_identical(tmp_path, weight_format):
    spec = bsnn.random_network(96, 24, steps=500, seed=21, plasticity=("triplet", "istdp", "stdp"))
    a = build(spec, weight_format)
    a.run(0, 230)
    path = tmp_path / "run.ckpt"
    a.save_checkpoint(path)
    a.run(230, 170)
    ref = snapshot(a, spec)
    b = build(spec, weight_format)
    b.load_checkpoint(path)
    assert b.info().steps_done == 230
    b.run(230, 170)
    got = snapshot(b, spec)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    a.close()
    b.close()


def test_load_refuses_a_different_network(tmp_path):
    spec = bsnn.random_network(96, 24, steps=300, seed=21)
    a = build(spec)
    a.run(0, 50)
    path = tmp_path / "run.ckpt"
    a.save_checkpoint(path)
    other = build(bsnn.random_network(64, 16, steps=300, seed=21))
    with pytest.raises(bsnn.InvalidArgument):
        other.load_checkpoint(path)
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(b"not a checkpoint at all")
    with pytest.raises(bsnn.InvalidArgument):
        a.load_checkpoint(bad)
    a.close()
    other.close()
