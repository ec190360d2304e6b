"""Shared pytest set-up: the `gpu` marker, import paths, and helpers that build one network into
both libbsnn (the product) and the CPU oracle (the checker)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "example-cuda-spiking-nn_b200"
sys.path.insert(0, str(PKG))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a library)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.load()
    return oracle


def make_pair(spec, precision=32, noise_mode=None, replay=None, steps_per_launch=None):
    """(gpu Simulation, OracleSimulation) built from one NetworkSpec."""
    import bsnn
    import oracle
    g = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    o = oracle.OracleSimulation(spec.num_excitatory, spec.num_inhibitory, precision=precision, **spec.sim_kwargs())
    for sim in (g, o):
        spec.build(sim)
        if noise_mode is not None:
            sim.set_noise_mode(noise_mode)
        if replay is not None:
            sim.set_noise_replay(replay)
    if steps_per_launch is not None:
        g.set_steps_per_launch(steps_per_launch)
    return g, o


FLOAT_FIELDS = ["membrane_potentials", "g_excitatory", "g_inhibitory", "i_stimulus", "background_g_excitatory",
                "background_g_inhibitory", "background_excitatory_r_traces", "background_excitatory_d_traces",
                "background_inhibitory_r_traces", "background_inhibitory_d_traces"]


def assert_close(a, b, rtol, what, scale=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = scale if scale is not None else max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-300)
    err = np.abs(a - b) / s
    bad = np.flatnonzero(err > rtol)
    assert bad.size == 0, (f"{what}: {bad.size} of {a.size} differ beyond {rtol:g} x max|ref|; first {bad[:5]}, "
                           f"got {a[bad[:5]]}, want {b[bad[:5]]}")


def compare_state(g, o, spec, rtol=1e-5, weights=True, tag=""):
    """Compares every per-neuron field, the connection and plasticity traces and the weights."""
    np.testing.assert_array_equal(g.read("spikes"), o.read("spikes"), err_msg=f"{tag} spikes")
    np.testing.assert_array_equal(g.read("refractory_counter"), o.read("refractory_counter"), err_msg=f"{tag} refrac")
    for f in FLOAT_FIELDS:
        assert_close(g.read(f), o.read(f), rtol, f"{tag} {f}")
    for c in range(len(spec.conns)):
        for f in ("connection_r_traces", "connection_d_traces", "connection_summed"):
            assert_close(g.read(f, c), o.read(f, c), rtol, f"{tag} {f}[{c}]")
    for k, p in enumerate(spec.plasts):
        n_pre = spec.conns[p.conn].weights.shape[0]
        n_post = spec.conns[p.conn].weights.shape[1]
        assert_close(g.read("plasticity_pre_traces", k, count=n_pre), o.read("plasticity_pre_traces", k), rtol,
                     f"{tag} pre traces[{k}]")
        assert_close(g.read("plasticity_post_traces", k, count=n_post), o.read("plasticity_post_traces", k), rtol,
                     f"{tag} post traces[{k}]")
    if weights:
        for c in range(len(spec.conns)):
            assert_close(g.read_weights(c), o.read_weights(c), rtol, f"{tag} weights[{c}]")
