"""Benchmark of the per-step hot path (System::step_the_clock) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bsnn|reference] [--workload NAME]
                    [--weight-format F] [--no-forms]

A bench "step" is one recording interval of simulation (--sim-steps clock steps, default 10,000
= 1 simulated second at dt = 0.1 ms) of the workload, run through libbsnn's C-ABI.  The default
workload is the reference example network (2,500 E + 625 I, ~9.8 M dense FP32 synapses, triplet
STDP on E->E and iSTDP on I->E, Poisson background, 4 stimulus pulses, all spikes and 50
voltages recorded), built from seeded synthetic inputs (no dataset is involved).

Metric: simulated seconds per wall second (whole job, all ranks); the line also carries dense
synaptic updates/s and spike-driven synaptic events/s.  With N > 1 every rank runs an
independent replica (the single-network path is not sharded): weak scaling, no collective on
the data path.  The batched workload shards its instances over the ranks instead.

On one GPU the default run adds the chosen forms under their own keys of the same JSON line, each
with its own CUDA-event timing, clock record, roofline and error against an FP64 run:
`small_plastic_500` (400 E + 100 I, FP32), `large_bf16` and `large_fp8` (8,100 E + 2,025 I with
BF16 / per-row-scaled FP8 weight copies), `batched` (192 networks in one persistent launch, with
the plain form beside it) and `adjoint` (one surrogate gradient over 2,000 steps).

--impl reference times the reference's own implementation of the path: its CUDA build
(oracle/_ref/ref_harness, the unmodified cpp_src components) driving the same network on this
GPU, or, when that binary is absent, the CPU oracle on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "example-cuda-spiking-nn_b200"))

DT = 1e-4
STEPS_PER_LAUNCH = 1000
PROFILE_TRAFFIC = ROOT / "profiles" / "traffic.json"
METRIC = "simulated-s per wall-s (and synaptic events/s) at 1 B200"
DEFAULT_WORKLOAD = "example_plastic_3125"
L2_BYTES = 126e6
# steps of the reference arm's bench step: a bounded sample of the same workload (about 0.45 s of
# the reference build on the example network), so K of them end within seconds
REFERENCE_SAMPLE_STEPS = 500


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bsnn", choices=["bsnn", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--weight-format", default="f32", choices=["f32", "f32_rowscaled", "bf16", "fp8_e4m3"],
                    help="weight storage form: f32 = the reference's arithmetic; the others keep FP32 masters with "
                         "a per-row normalisation scale and propagate from a copy in that type")
    ap.add_argument("--sim-steps", type=int, default=10000)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the chosen forms on the default workload")
    ap.add_argument("--form-steps", type=int, default=3, help="timed bench steps of each chosen form")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.lines:
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_tensor_peak():
    """Dense BF16 TFLOP/s: the burst figure (a kernel timed alone)."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def profiled_traffic(key):
    """DRAM bytes per launch of the step kernel from one ncu capture (profiles/traffic.json)."""
    if PROFILE_TRAFFIC.exists():
        tr = json.loads(PROFILE_TRAFFIC.read_text()).get(key)
        if tr:
            return tr["dram_bytes_per_launch"]
    return None


def timed_runs(run_one, stream, k, flush):
    """k calls of run_one(), each bracketed by CUDA events on `stream`, the L2 flushed (a 256 MB
    write) and the device synchronised before each; returns the times in ms."""
    import torch
    times = []
    for _ in range(k):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_one()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def reduce_over_ranks(t_ms: float, events: int, spikes: int, device):
    """Whole-job figures of N independent replicas: the slowest rank's device time (max) and the
    summed event and spike counts.  `device` is where the process group's backend keeps tensors
    (a CUDA device for NCCL, "cpu" for gloo)."""
    import torch
    t = torch.tensor([t_ms], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ev = torch.tensor([float(events), float(spikes)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(ev)
    return float(t.item()), int(ev[0].item()), int(ev[1].item())


# ---- the single-network engine -------------------------------------------------------------------

COPY_BYTES = {"f32_rowscaled": 4, "bf16": 2, "fp8_e4m3": 1}
FORM_NAMES = {"f32": "plain FP32 (reference arithmetic)",
              "f32_rowscaled": "FP32 masters, per-row normalisation scale, GEMV from an FP32 copy",
              "bf16": "FP32 masters, per-row normalisation scale, GEMV from a BF16 copy (FP32 accumulate)",
              "fp8_e4m3": "FP32 masters, per-row normalisation scale, GEMV from an FP8 E4M3 copy with per-row "
                          "scales (FP32 accumulate)"}
FORM_DTYPES = {"f32": "f32", "f32_rowscaled": "f32", "bf16": "bf16 weights, f32 accumulate",
               "fp8_e4m3": "fp8 e4m3 weights, f32 accumulate"}


def algorithmic_bytes_per_step(spec, form="f32") -> float:
    """f32: weight read of every connection once (FP32), read+write of the plastic matrices (the
    update and the row normalisation, counted once at 4 B), and ~100 B/neuron of state.
    Row-scaled forms: one read of every connection's GEMV copy (4, 2 or 1 B per entry) and the
    same state; the updates touch only the rows and columns of spiking neurons (not counted)."""
    if form != "f32":
        return float(sum(c.weights.size * COPY_BYTES[form] for c in spec.conns) + 100 * spec.num_neurons)
    b = sum(c.weights.size * 4 for c in spec.conns)
    plastic = {p.conn for p in spec.plasts}
    b += sum(2 * spec.conns[c].weights.size * 4 for c in plastic)
    return float(b + 100 * spec.num_neurons)


def weight_read_bytes(spec, form="f32") -> float:
    return float(sum(c.weights.size * (4 if form == "f32" else COPY_BYTES[form]) for c in spec.conns))


def nnz_out(spec):
    """Nonzero outgoing synapses per neuron (for spike-driven event counts)."""
    out = np.zeros(spec.num_neurons, np.int64)
    for c in spec.conns:
        off = spec.groups[c.pre]["offset"]
        out[off:off + c.weights.shape[0]] += (c.weights != 0).sum(axis=1)
    return out


def spike_events_from_bits(bits, group_offset, n, nnz):
    unpacked = ((bits[:, :, None] >> np.arange(32, dtype=np.uint32)) & 1).reshape(bits.shape[0], -1)[:, :n]
    per_neuron = unpacked.sum(axis=0)
    return int(per_neuron.sum()), int((per_neuron * nnz[group_offset:group_offset + n]).sum())


def single_roofline(sim, spec, form, us_per_step, clock_steps_per_launch, traffic_key):
    """The bound that applies to the step kernel.  When the weights it reads each step fit on chip
    (shared memory plus half the 126 MB L2), nothing streams from HBM and the step is bound by
    latency: the floor is the step's own communication skeleton (partial-sum exchange and grid
    barrier, bsnn_measure_exchange_floor) run alone on the same grid, and the fraction is floor /
    measured.  Otherwise the weight stream is HBM-bound: algorithmic bytes per step over the
    measured HBM copy peak.  Both views are printed; `bound` names the one that applies."""
    peak, peak_kind = measured_peaks()
    bytes_step = algorithmic_bytes_per_step(spec, form)
    hbm_achieved = bytes_step / (us_per_step * 1e-6) / 1e9
    traffic = profiled_traffic(traffic_key)
    hbm = {"achieved": hbm_achieved, "peak": peak, "unit": "GB/s", "frac": hbm_achieved / peak,
           "peak_source": peak_kind, "bytes_per_clock_step": bytes_step,
           "dram_bytes_per_clock_step": None if traffic is None else traffic / clock_steps_per_launch}
    on_chip = weight_read_bytes(spec, form) <= 0.5 * L2_BYTES
    if not on_chip:
        return {"bound": "hbm", "achieved": hbm_achieved, "peak": peak, "unit": "GB/s", "frac": hbm_achieved / peak,
                "traffic": traffic, "peak_source": peak_kind, "bytes_per_clock_step": bytes_step,
                "clock_steps_per_launch": clock_steps_per_launch,
                "note": "algorithmic bytes (weight copy read once per step, O(N) state) over the measured HBM "
                        "copy peak; traffic is DRAM bytes per launch from one ncu capture"}
    floor_us = sim.exchange_floor_us(2000)
    return {"bound": "latency", "achieved": 1e3 / us_per_step, "peak": 1e3 / floor_us, "unit": "clock steps/ms",
            "frac": floor_us / us_per_step, "traffic": traffic, "us_per_clock_step": us_per_step,
            "floor_us_per_clock_step": floor_us, "clock_steps_per_launch": clock_steps_per_launch,
            "floor": "the step's partial-sum exchange and grid barrier alone (bsnn_measure_exchange_floor: every "
                     "CTA stores its slots, crosses the barrier, gathers its columns; same grid and plan)",
            "hbm_view": dict(hbm, note="the weights stay in shared memory and L2 for the whole launch, so this "
                                       "ratio of algorithmic bytes to the HBM peak is not a bound")}


def run_single(spec, form, S, K, W, dev, world=1, workload=None, with_events=True):
    """K timed bench steps of S clock steps of one network (after W untimed ones) through the
    single-network engine; returns the line fields (timing, rates, clocks, roofline)."""
    import torch

    import bsnn
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, device=dev, **spec.sim_kwargs())
    spec.build(sim)
    if form != "f32":
        sim.set_weight_format(form)
    sim.set_steps_per_launch(STEPS_PER_LAUNCH)
    stream = torch.cuda.ExternalStream(sim.stream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    nnz = nnz_out(spec)
    spike_mons = [(m, mon.group) for m, mon in enumerate(spec.monitors) if mon.kind == "spikes"]
    volt_mons = [m for m, mon in enumerate(spec.monitors) if mon.kind == "voltage"]
    clock = 0
    for _ in range(W):
        sim.run(clock, S)
        clock += S
    sim.synchronize()

    def drain():
        s_ = e_ = 0
        for m, g in spike_mons:
            bits = sim.read_spike_bits(m, flush=True)
            if with_events:
                a, b = spike_events_from_bits(bits, spec.groups[g]["offset"], spec.groups[g]["num_neurons"], nnz)
                s_ += a
                e_ += b
        for m in volt_mons:
            sim.read_voltage_history(m, flush=True)
        return s_, e_

    drain()
    info0 = sim.info()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    spikes = events = 0
    with ClockSampler(dev) as clocks:
        times_ms = []
        for _ in range(K):
            times_ms += timed_runs(lambda: sim.run(clock, S), stream, 1, flush)
            clock += S
            s_, e_ = drain()
            spikes += s_
            events += e_
        sim.synchronize()
    info1 = sim.info()
    t_ms = float(sum(times_ms))
    if world > 1:
        t_ms, events, spikes = reduce_over_ranks(t_ms, events, spikes, dev)
    launches = int(info1.kernel_launches - info0.kernel_launches)
    sim_seconds = K * S * DT * world
    steps_per_s = K * S * world / (t_ms / 1e3)
    us_per_step = t_ms * 1e3 / (K * S)
    key = (workload or spec.name) if form == "f32" else f"{workload or spec.name}/{form}"
    roof = single_roofline(sim, spec, form, us_per_step, K * S / max(1, launches), key)
    out = {
        "value": sim_seconds / (t_ms / 1e3), "unit": "simulated-s/wall-s", "steps": K, "warmup": W,
        "ms_per_step": t_ms / K, "clock_steps_per_bench_step": S, "dtype": FORM_DTYPES[form],
        "us_per_clock_step": us_per_step,
        "dense_synaptic_updates_per_s": spec.synapse_entries() * steps_per_s,
        "spike_driven_events_per_s": events / (t_ms / 1e3),
        "spikes_per_s_simulated": spikes / max(sim_seconds, 1e-12),
        "clock_steps_per_s": steps_per_s, "gpu_launches": launches, "roofline": roof, "clocks": clocks.summary(),
    }
    sim.close()
    return out


def form_errors(spec, forms, steps, device, v_step=20):
    """Error of each weight form against an FP64 run of the same network, seed and Poisson draws
    (the oracle in double precision): the largest |v - v64| / max|v64| after `v_step` steps, the
    relative spike-count difference per population over `steps` steps, and the drift of each
    plastic matrix, mean |w - w64| / mean |w64|, at the end."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    import bsnn
    t0 = time.perf_counter()
    o = oracle.OracleSimulation(spec.num_excitatory, spec.num_inhibitory, precision=oracle.PREC_F64,
                                **spec.sim_kwargs())
    spec.build(o)
    o.run(0, v_step)
    v_ref = o.read_f64("membrane_potentials")
    o.run(v_step, steps - v_step)
    spike_mons = [m for m, mon in enumerate(spec.monitors) if mon.kind == "spikes"]
    n_ref = [int(o.read_spike_history(m).sum()) for m in spike_mons]
    plastic = sorted({p.conn for p in spec.plasts})
    w_ref = {c: o.read_weights_f64(c) for c in plastic}
    o.close()
    fp64_s = time.perf_counter() - t0
    vscale = float(np.max(np.abs(v_ref)))
    out = {"sample": f"{steps} clock steps from step 0 (voltages at step {v_step}), the FP64 oracle with the same "
                     f"seed and Philox draws ({fp64_s:.1f} s on the host)", "fp64_spikes": n_ref}
    for form in forms:
        g = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, device=device, **spec.sim_kwargs())
        spec.build(g)
        if form != "f32":
            g.set_weight_format(form)
        g.run(0, v_step)
        v = g.read("membrane_potentials").astype(np.float64)
        g.run(v_step, steps - v_step)
        n = [int(g.read_spike_history(m).sum()) for m in spike_mons]
        drift = {str(c): float(np.mean(np.abs(g.read_weights(c).astype(np.float64) - w_ref[c])) /
                               max(float(np.mean(np.abs(w_ref[c]))), 1e-300)) for c in plastic}
        g.close()
        out[form] = {"voltage_rel_err": float(np.max(np.abs(v - v_ref))) / vscale,
                     "spikes": n, "rate_rel_err": [abs(a - b) / max(b, 1) for a, b in zip(n, n_ref)],
                     "weight_drift": drift}
    return out


def run_bsnn(args, rank, world):
    import torch

    import bsnn
    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    S, K, W = args.sim_steps, args.steps, args.warmup
    spec = bsnn.synthetic_network(args.workload, steps=(W + K) * S + 1, weight_values="uniform",
                                  recording_interval_steps=S,
                                  seed=bsnn.network.WORKLOADS[args.workload]["seed"] + rank)
    r = run_single(spec, args.weight_format, S, K, W, dev, world, args.workload)
    line = {
        "metric": METRIC, "value": r["value"], "unit": "simulated-s/wall-s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": r["dtype"],
        "data": "synthetic (seeded; reference example shapes, uniform[0, max_weight] weights)",
        "config": single_config(spec, args.workload, args.weight_format, world),
        "clock_steps_per_bench_step": S,
    }
    for k in ("us_per_clock_step", "dense_synaptic_updates_per_s", "spike_driven_events_per_s",
              "spikes_per_s_simulated", "clock_steps_per_s", "gpu_launches", "roofline", "clocks"):
        line[k] = r[k]
    return line, spec


def single_config(spec, workload, form, world):
    return {"workload": workload, "neurons": spec.num_neurons, "synapse_entries": spec.synapse_entries(),
            "dt_s": DT, "plasticity": "triplet(E->E)+iSTDP(I->E)" if spec.plasts else "off",
            "form": FORM_NAMES[form], "parallelism": f"replicas x{world}",
            "l2": "flushed (256 MB write) between timed steps"}


def run_e2e(args, dev):
    """Same metric through the public API with host buffers: build from host arrays (H2D of
    weights, parameters, stimulus), run, drain the spike and voltage rings to host memory every
    bench step, read the plastic weights back at the end.  Wall clock around all of it."""
    import torch

    import bsnn
    S, K = args.sim_steps, args.steps
    spec = bsnn.synthetic_network(args.workload, steps=K * S + 1, weight_values="uniform", recording_interval_steps=S)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, device=dev, **spec.sim_kwargs())
    spec.build(sim)
    if args.weight_format != "f32":
        sim.set_weight_format(args.weight_format)
    sim.set_steps_per_launch(STEPS_PER_LAUNCH)
    d2h = 0
    for k in range(K):
        sim.run(k * S, S)
        for m in (0, 1):
            d2h += sim.read_spike_bits(m, flush=True).nbytes
        d2h += sim.read_voltage_history(2, flush=True).nbytes
    w = sim.read_weights(0)
    d2h += w.nbytes
    sim.synchronize()
    el = time.perf_counter() - t0
    h2d = sum(c.weights.nbytes for c in spec.conns) + sum(np.asarray(a).nbytes for a in spec.stimulus)
    sim.close()
    return {"value": K * S * DT / el, "unit": "simulated-s/wall-s", "h2d_bytes_per_step": h2d // K,
            "d2h_bytes_per_step": d2h // K, "includes": "create+upload, run, per-step ring drains, final weight read"}


def _oracle_rate(spec, seconds: float, precision: int):
    """Simulated-s per wall-s of the CPU oracle stepping `spec` for about `seconds`."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    o = oracle.OracleSimulation(spec.num_excitatory, spec.num_inhibitory, precision=precision,
                                **spec.sim_kwargs())
    spec.build(o)
    o.run(0, 2)
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds and n < 20000:
        o.run(2 + n, 10)
        n += 10
    el = time.perf_counter() - t0
    o.close()
    return n * DT / el, n, el


def cpu_baseline(spec, seconds: float):
    """The CPU oracle on a bounded sample of the same workload, on all host threads: the FP32
    restatement of the reference step (the line's value: the reference's arithmetic) and, beside
    it, the same step in FP64."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    threads = int(os.environ.get("ORACLE_THREADS", os.cpu_count() or 1))
    v32, n32, el32 = _oracle_rate(spec, seconds * 2 / 3, oracle.PREC_F32)
    v64, n64, el64 = _oracle_rate(spec, seconds / 3, oracle.PREC_F64)
    return {"value": v32, "unit": "simulated-s/wall-s", "cores": threads, "kind": "port",
            "sample": f"{n32} clock steps of {spec.name} (FP32 oracle, {threads} threads), {el32:.1f} s",
            "fp64": {"value": v64, "unit": "simulated-s/wall-s", "cores": threads,
                     "sample": f"{n64} clock steps of {spec.name} (FP64 oracle, {threads} threads), {el64:.1f} s"}}


# ---- chosen forms (one GPU, default workload) ----------------------------------------------------

def form_small(args, dev):
    """Configuration 1: 400 E + 100 I, triplet + iSTDP, Poisson background at 5 kHz, one pulse into
    20 E neurons, 10,001 clock steps (the configuration's length) of FP32 (the reference's
    arithmetic)."""
    import bsnn
    S, K = args.sim_steps, args.form_steps
    spec = bsnn.synthetic_network("small_plastic_500", steps=(1 + K) * S + 1, weight_values="uniform",
                                  recording_interval_steps=S)
    r = run_single(spec, "f32", S, K, 1, dev, workload="small_plastic_500")
    err_spec = bsnn.synthetic_network("small_plastic_500", weight_values="uniform")  # 10,001 steps
    r["error_vs_fp64"] = form_errors(err_spec, ["f32"], err_spec.total_steps, dev)
    r["config"] = single_config(spec, "small_plastic_500", "f32", 1)
    return r


def forms_large(args, dev):
    """Configuration 3: 8,100 E + 2,025 I (~102 M dense synapse entries), triplet + iSTDP, with the
    BF16 and the per-row-scaled FP8 E4M3 weight copies (FP32 masters, FP32 accumulation); their
    error against FP64 beside that of the FP32 forms."""
    import bsnn
    S, K = args.sim_steps, max(1, args.form_steps - 1)
    spec = bsnn.synthetic_network("large_plastic_10125", steps=(1 + K) * S + 1, weight_values="uniform",
                                  recording_interval_steps=S)
    out = {}
    for form in ("bf16", "fp8_e4m3"):
        r = run_single(spec, form, S, K, 1, dev, workload="large_plastic_10125")
        r["config"] = single_config(spec, "large_plastic_10125", form, 1)
        out[form] = r
    err = form_errors(spec, ["f32", "f32_rowscaled", "bf16", "fp8_e4m3"], 200, dev)
    for form in ("bf16", "fp8_e4m3"):
        out[form]["error_vs_fp64"] = {"sample": err["sample"], "fp64_spikes": err["fp64_spikes"],
                                      form: err[form], "f32 (reference form)": err["f32"],
                                      "f32_rowscaled": err["f32_rowscaled"]}
    return out["bf16"], out["fp8_e4m3"]


BATCH_WORKLOADS = {"config4_batch_192": 192}


def shard_of(n_inst, rank, world):
    """Instances of a batch run by `rank`: every index congruent to rank modulo world."""
    return [b for b in range(n_inst) if b % world == rank]


def gather_instance_counts(counts_mine, mine, n_inst, device):
    """The one collective of the sharded batch: every rank places its instances' [n, 2] spike
    counts at their global indices and an all-reduce (sum) gives every rank all n_inst rows."""
    import torch
    allc = torch.zeros((n_inst, 2), dtype=torch.float64, device=device)
    allc[torch.as_tensor(mine, dtype=torch.long, device=device)] = torch.as_tensor(
        np.asarray(counts_mine, dtype=np.float64), device=device)
    torch.distributed.all_reduce(allc)
    return allc.cpu().numpy().astype(np.int64)


def run_batch(args, rank, world, K=None, W=None, seed=0):
    """The batched form: 192 independent networks (E from {400, 900, 1600, 2500, 3600}, I = E/4,
    own seed, g_leak and stimulus amplitude, plasticity off) in one persistent launch per bench
    step (a captured CUDA graph of --sim-steps clock steps).  With N ranks the instances are
    sharded (rank r runs every instance whose index is r mod N, with the seeds of the one-GPU
    spec) and one all-reduce gathers the spike counts at the end."""
    import torch

    import bsnn
    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    S = args.sim_steps
    K = args.steps if K is None else K
    W = args.warmup if W is None else W
    n_inst = BATCH_WORKLOADS.get(args.workload, 192)
    full = bsnn.config4_batch(n_inst, steps=(W + K) * S + 1, seed=seed)
    mine = shard_of(n_inst, rank, world)
    spec = full.subset(mine) if world > 1 else full
    sim = bsnn.BatchSimulation(spec, device=dev)
    tuning = sim.autotune(200)  # GEMM unit size and operand ring depth, timed on this GPU
    sim.set_steps_per_launch(S)
    stream = torch.cuda.ExternalStream(sim.stream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    sim.run(S)  # the first warm-up bench step: clock steps 0 .. S-1, compared with FP64 below
    sim.synchronize()
    first = sim.spike_counts().astype(np.int64)
    for _ in range(W - 1):
        sim.run(S)
    sim.synchronize()
    info0 = sim.info()
    c0 = sim.spike_counts().astype(np.int64)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clocks:
        times_ms = timed_runs(lambda: sim.run(S), stream, K, flush)
        sim.synchronize()
    info1 = sim.info()
    counts = sim.spike_counts().astype(np.int64)
    spikes = int((counts - c0).sum())
    t_ms = float(sum(times_ms))
    gathered = None
    if world > 1:
        gathered = gather_instance_counts(counts - c0, mine, n_inst, dev)
        spikes = int(gathered.sum())
        t_ms, _, _ = reduce_over_ranks(t_ms, 0, 0, dev)
    launches = int(info1.kernel_launches - info0.kernel_launches)
    sim_seconds = n_inst * K * S * DT
    value = sim_seconds / (t_ms / 1e3)
    sizes = [full.classes[i.cls].num_e + full.classes[i.cls].num_i for i in full.instances]
    flops_step = 2.0 * sum(n * n for n in sizes)
    synapses = sum(n * n for n in sizes)
    step_s = t_ms / 1e3 / (K * S)
    achieved = flops_step / step_s / 1e12
    peak, peak_kind = measured_tensor_peak()
    weight_bytes = float(info1.weight_bytes)
    line = {
        "metric": METRIC, "value": value, "unit": "simulated-s/wall-s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "bf16 weights and traces (hi + lo), f32 accumulate",
        "data": "synthetic (seeded; reference example shapes, uniform[0, max_weight] weights)",
        "config": {"workload": args.workload if args.workload in BATCH_WORKLOADS else "config4_batch_192",
                   "instances": n_inst, "neurons": int(sum(sizes)), "synapse_entries": int(synapses),
                   "size_classes": len(full.classes), "dt_s": DT, "plasticity": "off",
                   "form": "batched: one persistent launch per bench step, shared-weight propagation as a "
                           "tcgen05 BF16 GEMM per size class",
                   "parallelism": f"instances sharded x{world}" if world > 1 else "one GPU",
                   "l2": "flushed (256 MB write) between timed steps",
                   "autotuned": {"k_tiles_per_unit": tuning["k_tiles_per_unit"],
                                 "operand_stages": tuning["operand_stages"],
                                 "candidates": tuning["candidates"],
                                 "default_us_per_step": tuning["default_us_per_step"],
                                 "tuned_us_per_step": tuning["us_per_step"]}},
        "clock_steps_per_bench_step": S,
        "us_per_clock_step": step_s * 1e6,
        "dense_synaptic_updates_per_s": synapses / step_s,
        "spikes_per_s_simulated": spikes / max(sim_seconds, 1e-12),
        "clock_steps_per_s": 1.0 / step_s,
        "gpu_launches": launches,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind, "flops_per_clock_step": flops_step,
                     "bf16_weight_bytes_per_clock_step": weight_bytes,
                     "weight_read_gbs": weight_bytes / step_s / 1e9,
                     "note": "a GEMV-shaped GEMM (N = instances of a class x 2): bound by the MMA thread's "
                             "issue chain and the neuron phase between the GEMMs, not by the tensor pipe"},
        "clocks": clocks.summary(),
    }
    if world > 1:
        line["instances_this_rank"] = len(mine)
    sim.close()
    return line, (full, spec, mine, tuning, first, gathered)


def batch_error_vs_fp64(full, first, S, n_check=4):
    """Spike counts of the smallest instances over the first bench step (clock steps 0 .. S-1)
    against the FP64 oracle on the same BF16-valued weights, seed and Philox draws."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    sizes = [full.classes[i.cls].num_e for i in full.instances]
    pick = sorted(range(len(sizes)), key=lambda b: (sizes[b], b))[:n_check]
    tot_b = tot_r = 0
    per = []
    t0 = time.perf_counter()
    for b in pick:
        net = full.instance_network(b)
        net.recording_interval_steps = S  # the spike ring holds the whole first bench step
        o = oracle.OracleSimulation(net.num_excitatory, net.num_inhibitory, precision=oracle.PREC_F64,
                                    **net.sim_kwargs())
        net.build(o)
        o.run(0, S)
        ref = [int(o.read_spike_history(0).sum()), int(o.read_spike_history(1).sum())]
        o.close()
        for p in range(2):
            per.append(abs(int(first[b, p]) - ref[p]) / max(ref[p], 1))
            tot_b += int(first[b, p])
            tot_r += ref[p]
    return {"aggregate_rate_rel_err": abs(tot_b - tot_r) / max(tot_r, 1), "max_population_rate_rel_err": max(per),
            "spikes": tot_b, "fp64_spikes": tot_r,
            "sample": f"instances {pick} (the smallest), first {S} clock steps, FP64 oracle on the same "
                      f"BF16-valued weights ({time.perf_counter() - t0:.1f} s on the host)"}


def plain_form_baseline(spec, steps=2000):
    """The plain form of the same batch: the single-network engine (FP32, the reference's
    arithmetic) stepping one instance at a time; the time per clock step of one instance of each
    size class, weighted by the class's instances."""
    import torch

    import bsnn
    per_class = {}
    for b, inst in enumerate(spec.instances):
        if inst.cls in per_class:
            continue
        net = spec.instance_network(b)
        sim = bsnn.Simulation(net.num_excitatory, net.num_inhibitory, **net.sim_kwargs())
        net.build(sim)
        sim.run(0, 200)
        sim.synchronize()
        stream = torch.cuda.ExternalStream(sim.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.run(200, steps)
        e1.record(stream)
        e1.synchronize()
        per_class[inst.cls] = e0.elapsed_time(e1) / 1e3 / steps
        sim.close()
    wall = sum(per_class[i.cls] for i in spec.instances)  # seconds per clock step of all instances
    return {"value": len(spec.instances) * DT / wall, "unit": "simulated-s/wall-s",
            "seconds_per_clock_step_by_class": {str(k): v for k, v in sorted(per_class.items())},
            "sample": f"{steps} clock steps of one instance per size class through the single-network engine, "
                      f"weighted by the class's instance count"}


def run_batch_e2e(args, spec, tuning, K):
    """The batch through its public API with host buffers: build (weights and stimulus uploaded from
    host memory) with the shapes the autotuner chose, run K bench steps, read the spike counts
    back each step."""
    import torch

    import bsnn
    S = args.sim_steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim = bsnn.BatchSimulation(spec)
    sim.set_tuning(tuning)
    sim.set_steps_per_launch(S)
    d2h = 0
    for _ in range(K):
        sim.run(S)
        d2h += sim.spike_counts().nbytes
    sim.synchronize()
    el = time.perf_counter() - t0
    h2d = sum(sum(w.nbytes for w in c.weights) for c in spec.classes)
    h2d += sum(sum(np.asarray(a).nbytes for a in i.stimulus) for i in spec.instances)
    sim.close()
    return {"value": len(spec.instances) * K * S * DT / el, "unit": "simulated-s/wall-s", "h2d_bytes_per_step": h2d // K,
            "d2h_bytes_per_step": d2h // K, "includes": "create + upload, run, per-step spike-count reads"}


def form_batched(args, dev):
    line, (full, _, _, tuning, first, _) = run_batch(args, dev, 1, K=args.form_steps, W=1)
    pf = plain_form_baseline(full)
    keep = ("value", "unit", "steps", "warmup", "ms_per_step", "clock_steps_per_bench_step", "us_per_clock_step",
            "dtype", "config", "dense_synaptic_updates_per_s", "spikes_per_s_simulated", "gpu_launches", "roofline",
            "clocks")
    out = {k: line[k] for k in keep}
    out["plain_form"] = pf
    out["batched_over_plain"] = line["value"] / pf["value"]
    out["error_vs_fp64"] = batch_error_vs_fp64(full, first, args.sim_steps)
    out["e2e"] = run_batch_e2e(args, full, tuning, args.form_steps)
    return out


ADJOINT_WORKLOADS = {"config5_adjoint_3125": 2000}
ADJOINT_CHECKPOINT = 2000  # one segment: the whole tape in HBM, no recomputation


def run_adjoint(args, rank, world, K=None, W=None):
    """The differentiation form: one bench step is one gradient of the rate loss with respect to
    W_EE and g_leak (forward pass over 2,000 clock steps, then the backward pass) on the example
    network (2,500 E + 625 I, plasticity off), the target rate trace made by the same network with
    perturbed W_EE.  One checkpoint segment: the forward pass keeps the whole run's tape in HBM
    (about 160 MB), so the backward pass recomputes nothing."""
    import torch

    import bsnn
    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    T = ADJOINT_WORKLOADS["config5_adjoint_3125"]
    K = args.steps if K is None else K
    W = args.warmup if W is None else W
    spec, w_target = bsnn.config5_network(steps=T, seed=11 + rank)
    net = bsnn.AdjointNetwork(spec, T, checkpoint=ADJOINT_CHECKPOINT, noise=True, beta=0.5e-3, rate_weight=1.0,
                              device=dev)
    net.set_params(w_target, None)
    _, target, _ = net.forward(np.zeros(T, np.float32))
    net.set_params(spec.conns[0].weights, None)
    stream = torch.cuda.ExternalStream(net.stream())
    for _ in range(W):
        net.forward(target)
        net.backward()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    fwd_ms, tot_ms = [], []
    launches0 = net.launches()
    with ClockSampler(dev) as clocks:
        for _ in range(K):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            loss, rho, _ = net.forward(target)
            e1.record(stream)
            dW, dgl = net.backward()
            e2.record(stream)
            e2.synchronize()
            fwd_ms.append(e0.elapsed_time(e1))
            tot_ms.append(e0.elapsed_time(e2))
    t_ms = float(sum(tot_ms))
    if world > 1:
        t_ms, _, _ = reduce_over_ranks(t_ms, 0, 0, dev)
    launches = net.launches() - launches0
    sim_s = T * DT
    value = K * world * sim_s / (t_ms / 1e3)
    N, E, I = spec.num_neurons, spec.num_excitatory, spec.num_inhibitory
    w_bytes = 4.0 * (E + I) * N
    # per gradient: the backward pass streams all of W once per clock step (the pull-back GEMV)
    grad_bytes = T * w_bytes
    achieved = grad_bytes / (t_ms / K / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    line = {
        "metric": METRIC, "value": value,
        "unit": "simulated-s/wall-s (forward + backward)", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_ms / K, "ms_per_gradient": t_ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; reference example shapes, uniform[0, max_weight] weights)",
        "config": {"workload": "config5_adjoint_3125", "neurons": N, "clock_steps": T, "checkpoint_interval": ADJOINT_CHECKPOINT,
                   "dt_s": DT, "plasticity": "off", "loss": "MSE of the 5 ms-smoothed E rate vs a target trace",
                   "surrogate": "fast sigmoid, beta 0.5 mV", "parallelism": f"replicas x{world}",
                   "l2": "W (39 MB) is L2-resident by design; no flush"},
        "gradients_per_s": K * world / (t_ms / 1e3),
        "forward_ms": float(np.mean(fwd_ms)), "backward_ms": float(np.mean(tot_ms) - np.mean(fwd_ms)),
        "forward_simulated_s_per_wall_s": sim_s / (float(np.mean(fwd_ms)) / 1e3),
        "loss": loss, "mean_rate_hz": float(rho.mean()), "target_mean_rate_hz": float(target.mean()),
        "grad_norm_w_ee": float(np.linalg.norm(dW)), "grad_g_leak": dgl,
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind, "bytes_per_gradient": grad_bytes,
                     "note": "algorithmic bytes: the pull-back GEMV's dense W stream, once per clock step; "
                             "W is L2-resident, so this is an L2-served stream measured against the HBM peak"},
        "clocks": clocks.summary(),
    }
    return line, (spec, w_target, target, net)


def adjoint_error_vs_fp64(dev):
    """The surrogate gradient (rate loss, fast sigmoid, beta 0.5 mV) of an 80 E + 20 I network over
    300 steps against the FP64 restatement of the same adjoint: relative Frobenius error of dL/dW_EE
    and relative error of dL/dg_leak."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import adjoint_ref

    import bsnn
    T = 300
    spec = bsnn.random_network(80, 20, steps=T + 1, seed=4, noise=False, plasticity=(), stim_events=30)
    RT = np.full(T, 5.0, dtype=np.float32)
    VT = np.full(T, -0.062, dtype=np.float32)
    kw = dict(beta=0.5e-3, rate_weight=1.0, voltage_weight=1e3)
    net = bsnn.AdjointNetwork(spec, T, checkpoint=100, noise=False, device=dev, **kw)
    net.forward(RT, VT)
    dW, dgl = net.backward()
    net.close()
    _, dW64, dgl64 = adjoint_ref.reference_gradient(spec, T, RT, VT, **kw)
    return {"grad_w_ee_rel_err": float(np.linalg.norm(dW.astype(np.float64) - dW64) / np.linalg.norm(dW64)),
            "grad_g_leak_rel_err": abs(dgl - dgl64) / abs(dgl64),
            "sample": "80 E + 20 I, 300 clock steps, noise off, rate + voltage loss; the FP64 numpy restatement of "
                      "the same surrogate adjoint"}


def run_adjoint_e2e(args, state, K):
    """The gradient through the public API with host buffers, as torch.autograd sees it: W_EE and
    g_leak uploaded (set_params), forward, backward, dW_EE read back, every bench step."""
    import bsnn
    spec, w_target, target, net = state
    SpikingLoss = bsnn.spiking_loss_function()
    import torch
    w = torch.tensor(spec.conns[0].weights, requires_grad=True)
    gl = torch.tensor(float(np.float32(spec.groups[0]["g_leak"])), requires_grad=True)
    t0 = time.perf_counter()
    for _ in range(K):
        w.grad = None
        loss = SpikingLoss.apply(w, gl, net, target)
        loss.backward()
    el = time.perf_counter() - t0
    T = ADJOINT_WORKLOADS["config5_adjoint_3125"]
    return {"value": K * T * DT / el, "unit": "simulated-s/wall-s (forward + backward)",
            "h2d_bytes_per_step": w.numel() * 4 + target.nbytes, "d2h_bytes_per_step": w.numel() * 4 + 8 + 4 * 2 * T,
            "includes": "torch.autograd.Function: W_EE upload, forward, backward, dW_EE download"}


def adjoint_cpu_baseline(spec, seconds: float):
    """The FP64 restatement of the same gradient (numpy, noise off) on the host cores, over a
    bounded number of clock steps."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import adjoint_ref
    steps = 20
    while True:
        t0 = time.perf_counter()
        adjoint_ref.reference_gradient(spec, steps, np.zeros(steps), beta=0.5e-3)
        el = time.perf_counter() - t0
        if el > seconds / 4 or steps >= 2000:
            break
        steps *= 2
    return {"value": steps * DT / el, "unit": "simulated-s/wall-s (forward + backward)", "cores": os.cpu_count(),
            "kind": "port", "sample": f"the FP64 numpy restatement of the gradient over {steps} clock steps "
                                      f"(noise off), BLAS threads as numpy sets them"}


def form_adjoint(args, dev):
    line, state = run_adjoint(args, dev, 1, K=args.form_steps, W=1)
    keep = ("value", "unit", "steps", "warmup", "ms_per_step", "ms_per_gradient", "dtype", "config", "gradients_per_s",
            "forward_ms", "backward_ms", "forward_simulated_s_per_wall_s", "gpu_launches", "roofline", "clocks")
    out = {k: line[k] for k in keep}
    out["error_vs_fp64"] = adjoint_error_vs_fp64(dev)
    out["e2e"] = run_adjoint_e2e(args, state, args.form_steps)
    state[3].close()
    return out


def add_forms(line, args, dev):
    """The chosen forms of the metric ("chosen form vs plain"), each under its own key."""
    t0 = time.perf_counter()
    line["small_plastic_500"] = form_small(args, dev)
    line["large_bf16"], line["large_fp8"] = forms_large(args, dev)
    line["batched"] = form_batched(args, dev)
    line["adjoint"] = form_adjoint(args, dev)
    line["forms_wall_s"] = time.perf_counter() - t0


# ---- the reference arm ---------------------------------------------------------------------------

def run_reference(args, rank, world):
    """The reference's own implementation: its CUDA build (oracle/_ref/ref_harness) on this GPU,
    timed over K bench steps of REFERENCE_SAMPLE_STEPS clock steps each (a bounded sample of the
    same workload, L2 flushed between them); falls back to the CPU oracle when the build is
    absent."""
    import bsnn
    sys.path.insert(0, str(ROOT / "oracle"))
    if args.workload in BATCH_WORKLOADS:
        return {"impl": "reference", "unavailable": "the reference has no batched form (it steps one network per "
                "process); its per-network speed is its line on the default workload"}
    if args.workload in ADJOINT_WORKLOADS:
        return {"impl": "reference", "unavailable": "the reference has no gradient of the simulation (forward only); "
                "its forward speed is its line on the default workload"}
    R, K, W = REFERENCE_SAMPLE_STEPS, args.steps, args.warmup
    spec = bsnn.synthetic_network(args.workload, steps=(W + K) * R + 101, weight_values="uniform",
                                  recording_interval_steps=args.sim_steps,
                                  seed=bsnn.network.WORKLOADS[args.workload]["seed"])
    harness = ROOT / "oracle" / "_ref" / "ref_harness"
    gpu_ok = False
    try:
        import torch
        gpu_ok = torch.cuda.is_available()
    except Exception:
        pass
    base = {"metric": METRIC, "unit": "simulated-s/wall-s", "n_gpus": world, "steps": K, "warmup": W,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "impl": "reference",
            "data": "synthetic (seeded; reference example shapes, uniform[0, max_weight] weights)",
            "config": single_config(spec, args.workload, "f32", world)}
    if harness.exists() and gpu_ok:
        import refnet
        with tempfile.TemporaryDirectory() as td:
            r = refnet.run_bench(spec, W * R, K, R, td)
        secs = r["seconds"]
        value = K * R * DT / sum(secs)
        ms_per_step = 1e3 * sum(secs) / K
        sample = (f"{K} samples of {R} clock steps of System::step_the_clock after {W * R} warm-up steps, reference "
                  f"CUDA build (cpp_src, sm_100a, cuBLAS) on this GPU, driven by 1 host thread, L2 flushed between "
                  f"samples")
        kind, cores, steps_per = "reference", 1, R
    else:
        cb = cpu_baseline(spec, args.cpu_seconds)
        value, sample, kind, cores = cb["value"], cb["sample"], "port", cb["cores"]
        steps_per = int(round(value * args.cpu_seconds / DT / max(K, 1)))
        ms_per_step = args.cpu_seconds * 1e3 / max(K, 1)
    line = dict(base, value=value, ms_per_step=ms_per_step, clock_steps_per_bench_step=steps_per,
                us_per_clock_step=DT / value * 1e6,
                cpu_baseline={"value": value, "unit": "simulated-s/wall-s", "cores": cores, "kind": kind,
                              "sample": sample},
                e2e={"value": value, "unit": "simulated-s/wall-s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                dense_synaptic_updates_per_s=spec.synapse_entries() * value / DT)
    return line


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, rank, world)), flush=True)
        return
    import torch
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload in ADJOINT_WORKLOADS:
        line, state = run_adjoint(args, local, world)
        if rank == 0:
            if not args.no_e2e:
                line["e2e"] = run_adjoint_e2e(args, state, args.steps)
            if not args.no_cpu_baseline and world == 1:
                line["cpu_baseline"] = adjoint_cpu_baseline(state[0], args.cpu_seconds)
            print(json.dumps(line), flush=True)
        state[3].close()
    elif args.workload in BATCH_WORKLOADS:
        line, (full, spec, mine, tuning, first, gathered) = run_batch(args, local, world)
        if rank == 0:
            if gathered is not None:
                line["instances_gathered"] = int(gathered.shape[0])
            if not args.no_e2e:
                line["e2e"] = run_batch_e2e(args, spec, tuning, args.steps)
            if world == 1:
                pf = plain_form_baseline(full)
                line["plain_form"] = pf
                line["batched_over_plain"] = line["value"] / pf["value"]
                line["error_vs_fp64"] = batch_error_vs_fp64(full, first, args.sim_steps)
            if not args.no_cpu_baseline and world == 1:
                cb = cpu_baseline(full.instance_network(0), args.cpu_seconds / 2)
                line["cpu_baseline"] = dict(cb, value=cb["value"], sample=cb["sample"] + " (one instance; the "
                                            "batch's aggregate is the instance count times slower per instance)")
            print(json.dumps(line), flush=True)
    else:
        line, spec = run_bsnn(args, local, world)
        if rank == 0:
            dev = torch.cuda.current_device()
            if not args.no_e2e:
                line["e2e"] = run_e2e(args, dev)
            if not args.no_cpu_baseline and world == 1:
                line["cpu_baseline"] = cpu_baseline(spec, args.cpu_seconds)
            if world == 1 and not args.no_forms and args.workload == DEFAULT_WORKLOAD and args.weight_format == "f32":
                add_forms(line, args, dev)
            print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
