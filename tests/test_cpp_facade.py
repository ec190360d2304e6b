"""The C++ component facade (include/bsnn.hpp): tests/cpp/facade_run builds a network the way the
reference's main does (GpuSimulationState, NeuronGroup, Connection, Stimulus, the plasticities,
SpikeRecorder / VoltageRecorder, System::run) and must produce exactly what the Python path
through the same C-ABI produces: byte-identical spike files and bit-identical final membrane
potentials, with and without step callbacks (batched launches vs one launch per step)."""
from __future__ import annotations

import json
import subprocess
import sys

import numpy as np
import pytest

import bsnn
from conftest import ROOT

sys.path.insert(0, str(ROOT / "oracle"))
import refnet  # noqa: E402

CPP = ROOT / "tests" / "cpp"


def build():
    subprocess.run(["make", "-C", str(CPP)], check=True, capture_output=True)
    return CPP / "facade_run"


def test_facade_compiles_and_links():
    assert build().exists()


@pytest.mark.gpu
@pytest.mark.parametrize("callbacks", [False, True])
def test_facade_matches_python_path(tmp_path, callbacks):
    exe = build()
    spec = bsnn.random_network(96, 24, steps=400, seed=9, plasticity=("triplet", "istdp", "stdp"))
    spec.recording_interval_steps = 100
    steps = 301
    net = tmp_path / "net.bin"
    refnet.write_network(spec, net)
    cdir = tmp_path / "cpp"
    cdir.mkdir()
    res = subprocess.run([str(exe), str(net), str(steps), str(cdir)] + (["callbacks"] if callbacks else []),
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    out = json.loads(res.stdout.strip().splitlines()[-1])
    assert out["callbacks"] == (steps if callbacks else 0)
    assert out["weights_ee"] == 96 * 96

    pdir = tmp_path / "py"
    pdir.mkdir()
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    for m, mon in enumerate(spec.monitors):
        sim.set_monitor_output(m, pdir / (f"spikes_m{m}.txt" if mon.kind == "spikes" else f"voltage_m{m}.txt"))
    sim.run_system(steps)
    sim.flush_records()
    v = sim.read("membrane_potentials")
    sim.close()

    for m in (0, 1):
        a = (cdir / f"spikes_m{m}.txt").read_bytes()
        assert a == (pdir / f"spikes_m{m}.txt").read_bytes()
        assert a.count(b"\n") == 1 + 3 * spec.recording_interval_steps
    assert sorted(p.name for p in cdir.glob("voltage_m2_step*.txt")) == sorted(p.name for p in pdir.glob("voltage_m2_step*.txt"))
    np.testing.assert_array_equal(np.fromfile(cdir / "v.bin", np.float32), v)
