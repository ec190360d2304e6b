"""Writes a NetworkSpec as the binary description oracle/_ref/ref_harness reads, runs the harness,
and parses its dumps (TEST / BASELINE INFRASTRUCTURE ONLY).

Format "BSNNNET1": header (n_e, n_i, total_steps, n_events, n_plast, interval: u32; seed: i32;
timestep: f32), then groups (raw NeuronGroupParams), connections (pre, post, raw
ConnectionParams, row-major float weights), stimulus arrays, plasticities (kind, conn, raw
PlasticityParams) and monitors (kind, group, ids).  The raw structs are the reference's PODs,
whose layout include/bsnn.h repeats.
"""
from __future__ import annotations

import ctypes
import struct
import subprocess
from pathlib import Path

import numpy as np

HARNESS = Path(__file__).resolve().parent / "_ref" / "ref_harness"


def write_network(spec, path):
    import bsnn
    n_events = 0 if spec.stimulus is None else len(spec.stimulus[1])
    with open(path, "wb") as f:
        f.write(b"BSNNNET1")
        f.write(struct.pack("<6Iif", spec.num_excitatory, spec.num_inhibitory, spec.total_steps, n_events,
                            len(spec.plasts), spec.recording_interval_steps, spec.rng_seed, spec.timestep))
        f.write(struct.pack("<I", len(spec.groups)))
        for g in spec.groups:
            f.write(bytes(bsnn.NeuronGroupParams.make(**g)))
        f.write(struct.pack("<I", len(spec.conns)))
        for c in spec.conns:
            f.write(struct.pack("<II", c.pre, c.post))
            f.write(bytes(bsnn.ConnectionParams.make(**c.params)))
            f.write(np.ascontiguousarray(c.weights, np.float32).tobytes())
        if spec.stimulus is None:
            f.write(struct.pack("<II", 0, 0))
        else:
            counts, ids, offs, deltas = spec.stimulus
            f.write(struct.pack("<I", len(counts)))
            f.write(np.asarray(counts, np.uint32).tobytes())
            f.write(struct.pack("<I", len(ids)))
            f.write(np.asarray(ids, np.uint32).tobytes())
            f.write(np.asarray(offs, np.uint32).tobytes())
            f.write(np.asarray(deltas, np.float32).tobytes())
        f.write(struct.pack("<I", len(spec.plasts)))
        for p in spec.plasts:
            f.write(struct.pack("<iI", p.kind, p.conn))
            f.write(bytes(bsnn.PlasticityParams.make(**p.params)))
        f.write(struct.pack("<I", len(spec.monitors)))
        for m in spec.monitors:
            ids = np.asarray(m.ids, np.uint32)
            f.write(struct.pack("<iII", 0 if m.kind == "spikes" else 1, m.group, len(ids)))
            f.write(ids.tobytes())


def run_dump(spec, steps, every, workdir, raster=False):
    """ref_harness dump mode: (states by step tag, final weights, Poisson counts [steps][N][2]) and,
    with raster=True, also every step's spikes as uint8 [steps][N]."""
    workdir = Path(workdir)
    net, out = workdir / "net.bin", workdir / "dump.bin"
    write_network(spec, net)
    subprocess.run([str(HARNESS), str(net), "dump", str(steps), str(out), str(every)], check=True)
    return read_dump(out, spec, steps, raster=raster)


def run_time(spec, warmup, steps, workdir):
    import json
    net = Path(workdir) / "net_time.bin"
    write_network(spec, net)
    res = subprocess.run([str(HARNESS), str(net), "time", str(warmup), str(steps)], check=True, capture_output=True,
                         text=True)
    return json.loads(res.stdout.strip().splitlines()[-1])


def run_bench(spec, warm_steps, samples, steps_per_sample, workdir):
    """ref_harness bench mode: wall seconds of each sample of `steps_per_sample` consecutive
    System::step_the_clock calls after `warm_steps`, with the L2 flushed between samples."""
    import json
    net = Path(workdir) / "net_bench.bin"
    write_network(spec, net)
    res = subprocess.run([str(HARNESS), str(net), "bench", str(warm_steps), str(samples), str(steps_per_sample)],
                         check=True, capture_output=True, text=True)
    return json.loads(res.stdout.strip().splitlines()[-1])


def read_dump(path, spec, steps, raster=False):
    b = Path(path).read_bytes()
    assert b[:8] == b"BSNNDMP1"
    N, nsteps = struct.unpack_from("<II", b, 8)
    pos = 16
    n_e, n_i = spec.num_excitatory, spec.num_inhibitory
    n_pl = len(spec.plasts)
    names = ["membrane_potentials", "g_excitatory", "g_inhibitory", "i_stimulus", "refractory_counter", "spikes",
             "background_g_excitatory", "background_g_inhibitory", "background_excitatory_r_traces",
             "background_excitatory_d_traces", "background_inhibitory_r_traces", "background_inhibitory_d_traces"]
    states = {}
    while b[pos:pos + 4] == b"STEP":
        (tag,) = struct.unpack_from("<I", b, pos + 4)
        pos += 8
        st = {}
        for nm in names:
            dt = np.uint32 if nm in ("refractory_counter", "spikes") else np.float32
            st[nm] = np.frombuffer(b, dt, N, pos).copy()
            pos += 4 * N
        st["summed"] = []
        for n in (n_e, n_e, n_i, n_i):
            st["summed"].append(np.frombuffer(b, np.float32, n, pos).copy())
            pos += 4 * n
        st["pre_traces"] = np.frombuffer(b, np.float32, n_pl * N, pos).copy().reshape(n_pl, N) if n_pl else None
        pos += 4 * n_pl * N
        st["post_traces"] = np.frombuffer(b, np.float32, n_pl * N, pos).copy().reshape(n_pl, N) if n_pl else None
        pos += 4 * n_pl * N
        states[tag] = st
    assert b[pos:pos + 4] == b"WGTS"
    pos += 4
    weights = []
    for c in spec.conns:
        (n,) = struct.unpack_from("<I", b, pos)
        pos += 4
        weights.append(np.frombuffer(b, np.float32, n, pos).copy().reshape(c.weights.shape))
        pos += 4 * n
    assert b[pos:pos + 4] == b"NOIS"
    pos += 4
    noise = np.frombuffer(b, np.uint8, steps * N * 2, pos).copy().reshape(steps, N, 2)
    pos += steps * N * 2
    if not raster:
        return states, weights, noise
    assert b[pos:pos + 4] == b"SPKS"
    pos += 4
    packed = np.frombuffer(b, np.uint8, steps * ((N + 7) // 8), pos).reshape(steps, (N + 7) // 8)
    return states, weights, noise, np.unpackbits(packed, axis=1)[:, :N]


def run_record(spec, steps, outdir):
    """ref_harness record mode: the reference's recorder files, the Poisson counts of every step
    ([steps][N][2] uint8) and the final weights of every connection, all in `outdir`."""
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    net = outdir / "net.bin"
    write_network(spec, net)
    subprocess.run([str(HARNESS), str(net), "record", str(steps), str(outdir)], check=True,
                   stdout=subprocess.DEVNULL)
    noise = np.fromfile(outdir / "noise.bin", np.uint8).reshape(steps, spec.num_neurons, 2)
    weights = [np.fromfile(outdir / f"weights_final_c{c}.bin", np.float32).reshape(cn.weights.shape)
               for c, cn in enumerate(spec.conns)]
    return noise, weights


def read_spike_rows(path):
    """The rows of a SpikeRecorder file: {label: [neuron ids]}."""
    rows = {}
    with open(path) as f:
        next(f)
        for line in f:
            label, _, ids = line.partition(", ")
            rows[int(label)] = [int(x) for x in ids.split()]
    return rows
