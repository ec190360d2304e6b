"""Benchmark of the per-step hot path (System::step_the_clock) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bsnn|reference] [--workload NAME]

A bench "step" is one recording interval of simulation (--sim-steps clock steps, default 10,000
= 1 simulated second at dt = 0.1 ms) of the workload, run through libbsnn's C-ABI.  The default
workload is the reference example network (2,500 E + 625 I, ~9.8 M dense FP32 synapses, triplet
STDP on E->E and iSTDP on I->E, Poisson background, 4 stimulus pulses, all spikes and 50
voltages recorded), built from seeded synthetic inputs (no dataset is involved).

Metric: simulated seconds per wall second (whole job, all ranks); the line also carries dense
synaptic updates/s and spike-driven synaptic events/s.  With N > 1 every rank runs an
independent replica (the single-network path is not sharded): weak scaling, no collective on
the data path.

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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bsnn", choices=["bsnn", "reference"])
    ap.add_argument("--workload", default="example_plastic_3125")
    ap.add_argument("--weight-format", default="f32", choices=["f32", "f32_rowscaled", "bf16", "fp8_e4m3"],
                    help="weight storage form: f32 = the reference's arithmetic; the others keep FP32 masters with "
                         "a per-row normalisation scale and propagate from a copy in that type")
    ap.add_argument("--sim-steps", type=int, default=10000)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
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


BATCH_WORKLOADS = {"config4_batch_192": 192}


def run_batch(args, rank, world):
    """The batched form: 192 independent networks (E from {400, 900, 1600, 2500, 3600}, I = E/4,
    own seed, g_leak and stimulus amplitude, plasticity off) in one persistent launch per bench
    step (a captured CUDA graph of --sim-steps clock steps).  Beside it, the plain form: the
    single-network engine stepping one instance at a time, timed per size class."""
    import torch

    import bsnn
    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    S, K, W = args.sim_steps, args.steps, args.warmup
    n_inst = BATCH_WORKLOADS[args.workload]
    spec = bsnn.config4_batch(n_inst, steps=(W + K) * S + 1, seed=rank)
    sim = bsnn.BatchSimulation(spec, device=dev)
    tuning = sim.autotune(200)  # GEMM unit size and operand ring depth, timed on this GPU
    sim.set_steps_per_launch(S)
    stream = torch.cuda.ExternalStream(sim.stream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    for _ in range(W):
        sim.run(S)
    sim.synchronize()
    info0 = sim.info()
    c0 = sim.spike_counts().astype(np.int64)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    times_ms = []
    with ClockSampler(dev) as clocks:
        for _ in range(K):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.run(S)
            e1.record(stream)
            e1.synchronize()
            times_ms.append(e0.elapsed_time(e1))
        sim.synchronize()
    info1 = sim.info()
    spikes = int((sim.spike_counts().astype(np.int64) - c0).sum())
    t_ms = float(sum(times_ms))
    if world > 1:
        t_ms, _, spikes = reduce_over_ranks(t_ms, 0, spikes, dev)
    launches = int(info1.kernel_launches - info0.kernel_launches)
    sim_seconds = n_inst * K * S * DT * world
    value = sim_seconds / (t_ms / 1e3)
    # algorithmic work per clock step: the propagation 2 * sum N_pre * N_post over instances
    sizes = [spec.classes[i.cls].num_e + spec.classes[i.cls].num_i for i in spec.instances]
    flops_step = 2.0 * sum(n * n for n in sizes)
    synapses = sum(n * n for n in sizes)
    step_s = t_ms / 1e3 / (K * S)
    achieved = flops_step / step_s / 1e12
    peak, peak_kind = measured_tensor_peak()
    weight_bytes = float(info1.weight_bytes)
    line = {
        "metric": "simulated-s per wall-s (and synaptic events/s) at 1 B200", "value": value,
        "unit": "simulated-s/wall-s", "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": t_ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 weights and traces (hi + lo), f32 accumulate",
        "data": "synthetic (seeded; reference example shapes, uniform[0, max_weight] weights)",
        "config": {"workload": args.workload, "instances": n_inst, "neurons": int(sum(sizes)),
                   "synapse_entries": int(synapses), "size_classes": len(spec.classes),
                   "clock_steps_per_bench_step": S, "dt_s": DT, "plasticity": "off",
                   "form": "batched: one persistent launch per bench step, shared-weight propagation as a "
                           "tcgen05 BF16 GEMM per size class", "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MB write) between timed steps",
                   "autotuned": {"k_tiles_per_unit": tuning["k_tiles_per_unit"],
                                 "operand_stages": tuning["operand_stages"],
                                 "candidates": tuning["candidates"],
                                 "default_us_per_step": tuning["default_us_per_step"],
                                 "tuned_us_per_step": tuning["us_per_step"]}},
        "dense_synaptic_updates_per_s": synapses / step_s * world,
        "spikes_per_s_simulated": spikes / max(sim_seconds, 1e-12),
        "clock_steps_per_s": 1.0 / step_s,
        "gpu_launches": launches,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind, "flops_per_clock_step": flops_step,
                     "bf16_weight_bytes_per_clock_step": weight_bytes,
                     "weight_read_gbs": weight_bytes / step_s / 1e9,
                     "note": "a GEMV-shaped GEMM (N = instances of a class x 2): bound by the weight stream "
                             "from L2 and the step's two grid barriers, not by the tensor pipe"},
        "clocks": clocks.summary(),
    }
    sim.close()
    return line, (spec, tuning)


ADJOINT_WORKLOADS = {"config5_adjoint_3125": 2000}


def run_adjoint(args, rank, world):
    """The differentiation form: one bench step is one gradient of the rate loss with respect to
    W_EE and g_leak (forward pass over 2,000 clock steps with checkpoints every 100, then the
    checkpointed backward pass) on the example network (2,500 E + 625 I, plasticity off), the
    target rate trace made by the same network with perturbed W_EE."""
    import torch

    import bsnn
    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    T, K, W = ADJOINT_WORKLOADS[args.workload], args.steps, args.warmup
    spec, w_target = bsnn.config5_network(steps=T, seed=11 + rank)
    net = bsnn.AdjointNetwork(spec, T, checkpoint=100, noise=True, beta=0.5e-3, rate_weight=1.0, device=dev)
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
    # per gradient: the forward pass and the replay each stream the rows of spiking neurons (x != 0),
    # the backward pass streams all of W once per clock step (the pull-back GEMV)
    grad_bytes = T * w_bytes
    achieved = grad_bytes / (t_ms / K / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    line = {
        "metric": "simulated-s per wall-s (and synaptic events/s) at 1 B200", "value": value,
        "unit": "simulated-s/wall-s (forward + backward)", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; reference example shapes, uniform[0, max_weight] weights)",
        "config": {"workload": args.workload, "neurons": N, "clock_steps": T, "checkpoint_interval": 100,
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


def run_adjoint_e2e(args, state):
    """The gradient through the public API with host buffers, as torch.autograd sees it: W_EE and
    g_leak uploaded (set_params), forward, backward, dW_EE read back, every bench step."""
    import bsnn
    spec, w_target, target, net = state
    SpikingLoss = bsnn.spiking_loss_function()
    import torch
    w = torch.tensor(spec.conns[0].weights, requires_grad=True)
    gl = torch.tensor(float(np.float32(spec.groups[0]["g_leak"])), requires_grad=True)
    K = args.steps
    t0 = time.perf_counter()
    for _ in range(K):
        w.grad = None
        loss = SpikingLoss.apply(w, gl, net, target)
        loss.backward()
    el = time.perf_counter() - t0
    T = ADJOINT_WORKLOADS[args.workload]
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


COPY_BYTES = {"f32_rowscaled": 4, "bf16": 2, "fp8_e4m3": 1}
FORM_NAMES = {"f32": "plain FP32 (reference arithmetic)",
              "f32_rowscaled": "FP32 masters, per-row normalisation scale, GEMV from an FP32 copy",
              "bf16": "FP32 masters, per-row normalisation scale, GEMV from a BF16 copy (FP32 accumulate)",
              "fp8_e4m3": "FP32 masters, per-row normalisation scale, GEMV from an FP8 E4M3 copy with per-row "
                          "scales (FP32 accumulate)"}


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


def run_bsnn(args, rank, world):
    import torch

    import bsnn
    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    S, K, W = args.sim_steps, args.steps, args.warmup
    total = (W + K) * S + 1
    spec = bsnn.synthetic_network(args.workload, steps=total, weight_values="uniform", recording_interval_steps=S,
                                  seed=bsnn.network.WORKLOADS[args.workload]["seed"] + rank)
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, device=dev, **spec.sim_kwargs())
    spec.build(sim)
    if args.weight_format != "f32":
        sim.set_weight_format(args.weight_format)
    sim.set_steps_per_launch(STEPS_PER_LAUNCH)
    stream = torch.cuda.ExternalStream(sim.stream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    nnz = nnz_out(spec)
    clock = 0
    for _ in range(W):
        sim.run(clock, S)
        clock += S
    sim.synchronize()
    for m in (0, 1):
        sim.read_spike_bits(m, flush=True)
    sim.read_voltage_history(2, flush=True)
    info0 = sim.info()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    times_ms = []
    spikes = events = 0
    with ClockSampler(dev) as clocks:
        for _ in range(K):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.run(clock, S)
            e1.record(stream)
            e1.synchronize()
            clock += S
            times_ms.append(e0.elapsed_time(e1))
            for m, g in ((0, 0), (1, 1)):
                bits = sim.read_spike_bits(m, flush=True)
                s_, e_ = spike_events_from_bits(bits, spec.groups[g]["offset"], spec.groups[g]["num_neurons"], nnz)
                spikes += s_
                events += e_
        sim.synchronize()
    info1 = sim.info()
    t_ms = float(sum(times_ms))
    if world > 1:
        t_ms, events, spikes = reduce_over_ranks(t_ms, events, spikes, dev)
    launches = int(info1.kernel_launches - info0.kernel_launches)
    sim_seconds = K * S * DT * world
    value = sim_seconds / (t_ms / 1e3)
    steps_per_s = K * S * world / (t_ms / 1e3)
    per_launch_ms = t_ms / max(1, launches)
    clock_steps_per_launch = K * S / max(1, launches)
    bytes_step = algorithmic_bytes_per_step(spec, args.weight_format)
    achieved = bytes_step * clock_steps_per_launch / (per_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    if PROFILE_TRAFFIC.exists():
        key = args.workload if args.weight_format == "f32" else f"{args.workload}/{args.weight_format}"
        tr = json.loads(PROFILE_TRAFFIC.read_text()).get(key)
        if tr:
            traffic = tr["dram_bytes_per_launch"]
    line = {
        "metric": "simulated-s per wall-s (and synaptic events/s) at 1 B200",
        "value": value,
        "unit": "simulated-s/wall-s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": t_ms / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"f32": "f32", "f32_rowscaled": "f32", "bf16": "bf16 weights, f32 accumulate",
                  "fp8_e4m3": "fp8 e4m3 weights, f32 accumulate"}[args.weight_format],
        "data": "synthetic (seeded; reference example shapes, uniform[0, max_weight] weights)",
        "config": {"workload": args.workload, "neurons": spec.num_neurons, "synapse_entries": spec.synapse_entries(),
                   "clock_steps_per_bench_step": S, "dt_s": DT, "plasticity": "triplet(E->E)+iSTDP(I->E)",
                   "form": FORM_NAMES[args.weight_format], "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MB write) between timed steps"},
        "dense_synaptic_updates_per_s": spec.synapse_entries() * steps_per_s,
        "spike_driven_events_per_s": events / (t_ms / 1e3),
        "spikes_per_s_simulated": spikes / max(sim_seconds, 1e-12),
        "clock_steps_per_s": steps_per_s,
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "bytes_per_clock_step": bytes_step, "clock_steps_per_launch": clock_steps_per_launch,
                     "launch_ms": per_launch_ms,
                     "note": ("working set is L2-resident, so frac of HBM peak can exceed 1"
                              if bytes_step < 100e6 else "working set exceeds L2: streamed from HBM")},
        "clocks": clocks.summary(),
    }
    sim.close()
    return line, spec


def run_batch_e2e(args, spec, tuning):
    """The batch through its public API with host buffers: build (weights and stimulus uploaded from
    host memory) with the shapes the autotuner chose, run K bench steps, read the spike counts
    back each step."""
    import torch

    import bsnn
    S, K = args.sim_steps, args.steps
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


def run_reference(args, rank, world):
    """The reference's own implementation: its CUDA build (oracle/_ref/ref_harness) on this GPU,
    timed over a bounded sample; falls back to the CPU oracle when the build is absent."""
    import bsnn
    sys.path.insert(0, str(ROOT / "oracle"))
    if args.workload in BATCH_WORKLOADS:
        return {"impl": "reference", "unavailable": "the reference has no batched form (it steps one network per "
                "process); its per-network speed is its line on the default workload"}
    if args.workload in ADJOINT_WORKLOADS:
        return {"impl": "reference", "unavailable": "the reference has no gradient of the simulation (forward only); "
                "its forward speed is its line on the default workload"}
    spec_steps = 3000
    spec = bsnn.synthetic_network(args.workload, steps=spec_steps + 1, weight_values="uniform",
                                  recording_interval_steps=args.sim_steps)
    harness = ROOT / "oracle" / "_ref" / "ref_harness"
    base = {"metric": "simulated-s per wall-s (and synaptic events/s) at 1 B200", "unit": "simulated-s/wall-s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "impl": "reference", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "neurons": spec.num_neurons,
                       "synapse_entries": spec.synapse_entries(), "dt_s": DT}}
    gpu_ok = False
    try:
        import torch
        gpu_ok = torch.cuda.is_available()
    except Exception:
        pass
    if harness.exists() and gpu_ok:
        import refnet
        with tempfile.TemporaryDirectory() as td:
            r = refnet.run_time(spec, 100, 2000, td)
        value = r["steps"] * DT / r["seconds"]
        sample = (f"{r['steps']} clock steps of System::step_the_clock after 100 warm-up steps, reference CUDA build "
                  f"(cpp_src, sm_100a, cuBLAS) on this GPU, driven by 1 host thread")
        kind, cores = "reference", 1
    else:
        cb = cpu_baseline(spec, args.cpu_seconds)
        value, sample, kind, cores = cb["value"], cb["sample"], "port", cb["cores"]
    line = dict(base, value=value, ms_per_step=args.sim_steps * DT / value * 1e3,
                cpu_baseline={"value": value, "unit": "simulated-s/wall-s", "cores": cores, "kind": kind,
                              "sample": sample},
                e2e={"value": value, "unit": "simulated-s/wall-s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                dense_synaptic_updates_per_s=spec.synapse_entries() * value / DT)
    return line


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, rank, world)), flush=True)
        return
    import torch
    if world > 1:
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload in ADJOINT_WORKLOADS:
        line, state = run_adjoint(args, int(os.environ.get("LOCAL_RANK", "0")), world)
        if rank == 0:
            if not args.no_e2e:
                line["e2e"] = run_adjoint_e2e(args, state)
            if not args.no_cpu_baseline and world == 1:
                line["cpu_baseline"] = adjoint_cpu_baseline(state[0], args.cpu_seconds)
            print(json.dumps(line), flush=True)
        state[3].close()
    elif args.workload in BATCH_WORKLOADS:
        line, (spec, tuning) = run_batch(args, int(os.environ.get("LOCAL_RANK", "0")), world)
        if rank == 0:
            if not args.no_e2e:
                line["e2e"] = run_batch_e2e(args, spec, tuning)
            if world == 1:
                pf = plain_form_baseline(spec)
                line["plain_form"] = pf
                line["batched_over_plain"] = line["value"] / pf["value"]
            if not args.no_cpu_baseline and world == 1:
                cb = cpu_baseline(spec.instance_network(0), args.cpu_seconds / 2)
                line["cpu_baseline"] = dict(cb, value=cb["value"], sample=cb["sample"] + " (one instance; the "
                                            "batch's aggregate is the instance count times slower per instance)")
            print(json.dumps(line), flush=True)
    else:
        line, spec = run_bsnn(args, int(os.environ.get("LOCAL_RANK", "0")), world)
        if rank == 0:
            if not args.no_e2e:
                line["e2e"] = run_e2e(args, torch.cuda.current_device())
            if not args.no_cpu_baseline and world == 1:
                line["cpu_baseline"] = cpu_baseline(spec, args.cpu_seconds)
            print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
