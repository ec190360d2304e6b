"""The recorder text files (Monitor::record) against the files the reference's own SpikeRecorder,
VoltageRecorder and WeightRecorder wrote over the same run (tests/golden/record_random_120.npz,
made by tests/golden/make_golden.py with the reference's CUDA build; the Poisson counts are
replayed, so both runs see identical inputs).

Spike files must match byte for byte.  Voltage and weight files must have the same names (the
reference's step labels, including the wrap-around of the voltage record at clock step 0), the
same headers and ids, and values within 1e-5 relative of the reference's printed values: they are
printed with 6 significant digits, and the GEMV and row-normalisation summation orders differ in
the last bits (the step-0 weight record already holds step 0's plasticity update)."""
from __future__ import annotations

import json
import sys

import numpy as np
import pytest

import bsnn
from conftest import ROOT

sys.path.insert(0, str(ROOT / "tests" / "golden"))
from specs import RECORD_STEPS, record_spec, spec_digest  # noqa: E402

FIXTURE = ROOT / "tests" / "golden" / "record_random_120.npz"


def load():
    fx = dict(np.load(FIXTURE))
    spec = record_spec()
    assert str(fx["digest"]) == spec_digest(spec)
    meta = json.loads(str(fx["meta"]))
    assert meta["steps"] == RECORD_STEPS and meta["interval"] == spec.recording_interval_steps
    files = {k[5:]: bytes(v) for k, v in fx.items() if k.startswith("file:")}
    return fx, spec, files


def test_fixture_has_every_kind_of_file():
    fx, spec, files = load()
    assert "spikes_m0.txt" in files and "spikes_m1.txt" in files
    assert files["spikes_m0.txt"].startswith(b"clock_step, neuron_ids\n")
    vfiles = [n for n in files if n.startswith("voltage_m2_step")]
    # records at steps 0, 50, ..., 250, one file per ring slot; the record at step 0 is labelled
    # from 2**32 - 50 + 1 on (unsigned wrap-around in the reference)
    assert len(vfiles) == 6 * spec.recording_interval_steps
    assert "voltage_m2_step4294967247.txt" in files
    assert all(f"weights_c{c}_step0.txt" in files for c in range(4))


@pytest.mark.gpu
def test_recorder_files_match_the_reference(tmp_path):
    fx, spec, files = load()
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    sim.set_noise_mode(bsnn.NOISE_REPLAY)
    sim.set_noise_replay(fx["noise"])
    for m, mon in enumerate(spec.monitors):
        name = f"spikes_m{m}.txt" if mon.kind == "spikes" else f"voltage_m{m}.txt"
        sim.set_monitor_output(m, tmp_path / name)
    for c in range(len(spec.conns)):
        sim.add_weight_recorder(c, tmp_path / f"weights_c{c}.txt")
    sim.run_system(RECORD_STEPS)
    sim.flush_records()
    sim.close()
    ours = {p.name: p.read_bytes() for p in tmp_path.iterdir()}
    assert sorted(ours) == sorted(files)
    n_spike_rows = 0
    for name, want in files.items():
        got = ours[name]
        if name.startswith("spikes"):
            assert got == want, f"{name} differs"
            n_spike_rows += want.count(b"\n") - 1
            continue
        gl, wl = got.decode().splitlines(), want.decode().splitlines()
        assert gl[0] == wl[0] and len(gl) == len(wl), name
        scale = max(abs(float(line.rsplit(", ", 1)[1])) for line in wl[1:])
        for a, b in zip(gl[1:], wl[1:]):
            ka, va = a.rsplit(", ", 1)
            kb, vb = b.rsplit(", ", 1)
            assert ka == kb, (name, a, b)
            assert abs(float(va) - float(vb)) <= 1e-5 * scale, (name, a, b)
    assert n_spike_rows == 2 * 5 * spec.recording_interval_steps


@pytest.mark.gpu
def test_run_system_prints_the_progress_line_and_memory_report(capfd):
    """System::run's console line after each record (cpp_src/core/system.cpp:78-81) and
    GpuSimulationState::memory_report (cpp_src/gpu_core/gpu_simulation_state.cu:357-362)."""
    import re
    spec = bsnn.random_network(48, 12, steps=200, seed=3)
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    report = sim.memory_report()
    m = re.fullmatch(r"Total GPU Memory Allocated: (\d+) bytes \((\d+\.\d{6}) MB\)", report)
    assert m, report
    assert int(m.group(1)) == sim.info().device_bytes > 0
    assert abs(float(m.group(2)) - int(m.group(1)) / 2 ** 20) < 1e-6
    sim.run_system(10)  # progress off (the default): nothing printed
    assert "Completed clock step" not in capfd.readouterr().out
    sim.close()
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    sim.set_progress_output(True)
    interval = spec.recording_interval_steps  # 64
    sim.run_system(2 * interval + 5)
    sim.flush_records()
    sim.close()
    lines = [ln for ln in capfd.readouterr().out.splitlines() if ln.startswith("Completed clock step")]
    steps = [int(re.fullmatch(r"Completed clock step: (\d+) \| elapsed: ([0-9.e+-]+)s", ln).group(1)) for ln in lines]
    assert steps == [0, interval, 2 * interval], lines
