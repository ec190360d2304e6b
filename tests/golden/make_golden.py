"""Records the golden fixtures of tests/golden/ from the reference's own CUDA implementation.

    python tests/golden/make_golden.py [--out DIR] [--only state|record]

Needs a GPU and oracle/_ref/ref_harness (the reference's unmodified cpp_src components compiled
for sm_100a by `make -C oracle ref`, linked with a driver that builds the network of a spec, calls
System::step_the_clock and dumps the device state).  For each network of specs.golden_specs() it
runs GOLDEN_STEPS steps and stores, in <name>.npz:

  noise        uint8 [steps, N, 2]  the Poisson counts curand_poisson drew for every neuron and
                                    step (channel 0 excitatory, 1 inhibitory), read from a copy of
                                    each neuron's curand state just before the step
  spikes       uint8 [steps, ceil(N/8)]  np.packbits of every step's spike vector
  state_<f>    [len(CHECK_STEPS), ...]   full per-neuron fields after the check steps
  summed_<c>   float32 [len(CHECK_STEPS), n_pre]  x = d - r of connection c
  pre_traces / post_traces  float32 [len(CHECK_STEPS), n_plast, N]
  weights_<c>  float32 [n_pre, n_post]  every connection's weights after the last step
  digest       sha256 of the network's inputs (specs.spec_digest)

and, in record_random_120.npz, the text files the reference's SpikeRecorder, VoltageRecorder and
WeightRecorder write over a System::run-style loop of RECORD_STEPS steps (ref_harness record
mode), with that run's Poisson counts.

Replaying `noise` makes every other input deterministic, so the oracle and the CUDA path can be
compared with the reference step for step.
"""
from __future__ import annotations

import argparse
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "example-cuda-spiking-nn_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE))

import refnet  # noqa: E402
from specs import CHECK_STEPS, GOLDEN_STEPS, RECORD_STEPS, golden_specs, record_spec, spec_digest  # noqa: E402

STATE_FIELDS = ["membrane_potentials", "g_excitatory", "g_inhibitory", "i_stimulus", "refractory_counter",
                "background_g_excitatory", "background_g_inhibitory", "background_excitatory_r_traces",
                "background_excitatory_d_traces", "background_inhibitory_r_traces", "background_inhibitory_d_traces"]


def record_state(name, spec, out_dir: Path):
    with tempfile.TemporaryDirectory() as td:
        states, weights, noise = refnet.run_dump(spec, GOLDEN_STEPS, 1, td)
    steps = sorted(states)
    assert steps == list(range(GOLDEN_STEPS)), "dump must hold every step"
    arrays = {
        "noise": noise,
        "spikes": np.packbits(np.stack([states[s]["spikes"].astype(bool) for s in steps]), axis=1),
        "digest": np.array(spec_digest(spec)),
        "meta": np.array(json.dumps({"steps": GOLDEN_STEPS, "check_steps": list(CHECK_STEPS),
                                     "num_neurons": spec.num_neurons,
                                     "source": "reference cpp_src components (sm_100a build) via oracle/_ref/ref_harness"})),
    }
    for f in STATE_FIELDS:
        arrays[f"state_{f}"] = np.stack([states[s][f] for s in CHECK_STEPS])
    for c in range(len(spec.conns)):
        arrays[f"summed_{c}"] = np.stack([states[s]["summed"][c] for s in CHECK_STEPS])
    if spec.plasts:
        arrays["pre_traces"] = np.stack([states[s]["pre_traces"] for s in CHECK_STEPS])
        arrays["post_traces"] = np.stack([states[s]["post_traces"] for s in CHECK_STEPS])
    for c, w in enumerate(weights):
        arrays[f"weights_{c}"] = w
    path = out_dir / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    n_spk = int(np.unpackbits(arrays["spikes"], axis=1).sum())
    print(f"{name}: {path.stat().st_size / 1e6:.2f} MB, {n_spk} spikes in {GOLDEN_STEPS} steps", flush=True)


def record(spec, steps, out_dir: Path):
    """The reference's recorder files of a System::run-style loop (ref_harness record mode): every
    file's bytes as `file:<name>` (uint8) plus the Poisson counts of every step as `noise`."""
    import subprocess
    with tempfile.TemporaryDirectory() as td:
        net = Path(td) / "net.bin"
        files = Path(td) / "files"
        files.mkdir()
        refnet.write_network(spec, net)
        subprocess.run([str(refnet.HARNESS), str(net), "record", str(steps), str(files)], check=True,
                       stdout=subprocess.DEVNULL)
        noise = np.fromfile(files / "noise.bin", np.uint8).reshape(steps, spec.num_neurons, 2)
        arrays = {"noise": noise, "digest": np.array(spec_digest(spec)),
                  "meta": np.array(json.dumps({"steps": steps, "interval": spec.recording_interval_steps}))}
        for f in sorted(files.iterdir()):
            if f.name != "noise.bin":
                arrays["file:" + f.name] = np.frombuffer(f.read_bytes(), np.uint8)
    path = out_dir / "record_random_120.npz"
    np.savez_compressed(path, **arrays)
    print(f"record_random_120: {path.stat().st_size / 1e6:.2f} MB, {len(arrays) - 3} files", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE))
    ap.add_argument("--only", choices=["state", "record"], help="make one kind of fixture only")
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    if not refnet.HARNESS.exists():
        sys.exit(f"{refnet.HARNESS} is missing: build it with `make -C oracle ref`")
    if args.only != "record":
        for name, spec in golden_specs().items():
            record_state(name, spec, out)
    if args.only != "state":
        record(record_spec(), RECORD_STEPS, out)


if __name__ == "__main__":
    main()
