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


# Absolute floors of the per-element comparison |a - b| <= rtol (|b| + floor), one per quantity.
# Membrane potentials (|v| >= 0.04 V) and conductances (1e-10 .. 1e-8 S once driven, exactly 0
# before) are held relative to themselves: their floors are far below any value they take.  A
# weight is computed in steps of 1e-9 S scale (LTP and LTD increments, row rescaling), so one that
# plasticity drove towards 0 keeps an absolute error of a few 1e-16 S, the rounding unit of that
# arithmetic: weights are held relative to themselves down to 1e-11 S (1/150 of the smallest
# connection's largest weight) and to 1e-16 S absolute below it.
ELEMENT_FLOORS = {"membrane_potentials": 1e-9, "g_excitatory": 1e-16, "g_inhibitory": 1e-16, "weights": 1e-11}


def elementwise_error(a, b, floor):
    """The largest per-element relative error with an absolute floor, max |a - b| / (|b| + floor),
    and the index where it occurs."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    if a.size == 0:
        return 0.0, -1
    e = np.abs(a - b) / (np.abs(b) + floor)
    k = int(np.argmax(e))
    return float(e[k]), k


def assert_close_elementwise(a, b, rtol, floor, what):
    """Every element within rtol of itself: |a - b| <= rtol (|b| + floor)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    bad = np.flatnonzero(np.abs(a - b) > rtol * (np.abs(b) + floor))
    assert bad.size == 0, (f"{what}: {bad.size} of {a.size} differ beyond {rtol:g} relative (floor {floor:g}); "
                           f"first {bad[:5]}, got {a[bad[:5]]}, want {b[bad[:5]]}")


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
