"""The batched form: many independent networks of uneven size stepped by one persistent launch
(bsnn_batch_* in include/bsnn.h).

`config4_batch()` builds the batched-form workload: instances with E drawn uniformly from
{400, 900, 1600, 2500, 3600} (E on a square grid, I = E / 4 on a grid half as wide), each with its
own seed, g_leak drawn from U[8, 12] nS and stimulus amplitude from U[0.2, 1.0] nA, plasticity off.
Instances of one size share one weight set (seeded synthetic distance-dependent connectivity with
uniform[0, max_weight] values), which the library stores in BF16.

`BatchSpec.instance_network(b)` is instance b as an ordinary single network (weights rounded to
BF16 as the batch stores them), so any single-network backend -- the CPU oracle in the tests --
can run it alone.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import generation
from ._ffi import FIELD, UINT_FIELDS, ConnectionParams, NeuronGroupParams, error_for, load_library
from .network import EXAMPLE, ConnSpec, MonSpec, NetworkSpec

CONFIG4_SIZES = (400, 900, 1600, 2500, 3600)


def bf16_round(w: np.ndarray) -> np.ndarray:
    """float32 -> nearest BF16 value (ties to even), as float32."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


@dataclass
class BatchClass:
    num_e: int
    num_i: int
    weights: tuple          # (w_ee, w_ei, w_ie, w_ii), row-major [pre][post] float32
    e_conn: dict            # ConnectionParams of the E-presynaptic connections
    i_conn: dict            # ... of the I-presynaptic connections


@dataclass
class BatchInstance:
    cls: int
    e_group: dict           # NeuronGroupParams kwargs
    i_group: dict
    seed: int
    stimulus: tuple         # (counts[T], instance-local neurons, deltas)


@dataclass
class BatchSpec:
    total_steps: int
    classes: list = field(default_factory=list)
    instances: list = field(default_factory=list)

    def subset(self, indices) -> "BatchSpec":
        """The instances at `indices` (in that order) as a batch of their own: the same weight sets,
        parameters, seeds and stimuli, so each runs exactly as it does in the full batch.  Classes
        no listed instance uses are dropped."""
        used = sorted({self.instances[b].cls for b in indices})
        remap = {c: k for k, c in enumerate(used)}
        out = BatchSpec(total_steps=self.total_steps, classes=[self.classes[c] for c in used])
        for b in indices:
            inst = self.instances[b]
            out.instances.append(BatchInstance(remap[inst.cls], inst.e_group, inst.i_group, inst.seed, inst.stimulus))
        return out

    def instance_network(self, b: int) -> NetworkSpec:
        inst = self.instances[b]
        c = self.classes[inst.cls]
        spec = NetworkSpec(c.num_e, c.num_i, self.total_steps, rng_seed=inst.seed, name=f"instance_{b}")
        spec.groups = [dict(inst.e_group, offset=0, is_inhibitory=False),
                       dict(inst.i_group, offset=c.num_e, is_inhibitory=True)]
        for k, (pre, post) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
            spec.conns.append(ConnSpec(pre, post, bf16_round(c.weights[k]), dict(c.e_conn if pre == 0 else c.i_conn,
                                                                                 weight_matrix_idx=k)))
        counts, neurons, deltas = inst.stimulus
        spec.stimulus = (counts, neurons, np.zeros_like(neurons), deltas)
        spec.monitors = [MonSpec("spikes", 0), MonSpec("spikes", 1)]
        return spec


NEURON = dict(EXAMPLE, g_leak=10e-9, membrane_capacitance=200e-12, refractory_steps=20,
              mean_background_excitatory_spikes=0.5)
TAU = dict(rise_e=0.3e-3, decay_e=2e-3, rise_i=0.3e-3, decay_i=3e-3)


def config4_batch(n_instances: int = 192, steps: int = 10000, seed: int = 0, sizes=CONFIG4_SIZES,
                  stim_window=(1000, 4000), n_stim_ids: int = 20) -> BatchSpec:
    rng = np.random.default_rng(seed)
    dt = 1e-4
    spec = BatchSpec(total_steps=steps)
    draws = rng.choice(len(sizes), size=n_instances)
    used = sorted(set(int(d) for d in draws))
    cls_of_size = {}
    for k in used:
        num_e = int(sizes[k])
        side = int(round(np.sqrt(num_e)))
        i_side = side // 2
        num_i = i_side * i_side
        e_loc = generation.generate_2d_grid_locations(num_e, 1.0, side, side)
        i_loc = generation.generate_2d_grid_locations(num_i, 2.0, i_side, i_side)
        gen = [(e_loc, e_loc, 1.5e-9, 0.2, True), (e_loc, i_loc, 1.5e-9, 0.6, False),
               (i_loc, e_loc, 5.0e-9, 0.6, False), (i_loc, i_loc, 5.0e-9, 0.6, True)]
        ws = []
        for q, (pl, ql, wmax, prob, no_diag) in enumerate(gen):
            ws.append(generation.distance_2d_weights(
                pl, ql, max_weight_value=wmax, max_distance=45.0, spread_scale=81.0, weight_value_normal_dropoff=False,
                probabilistic_normal_not_uniform=True, probability_multiplier=prob, no_diagonal_connections=no_diag,
                x_location_length=float(side), y_location_length=float(side), rng_seed=seed * 1000 + k * 10 + q,
                value_mode="uniform").astype(np.float32))
        e_conn = dict(timestep=dt, decay_time=TAU["decay_e"], rise_time=TAU["rise_e"],
                      postsynaptic_kernel_normalization_value=1.7)
        i_conn = dict(timestep=dt, decay_time=TAU["decay_i"], rise_time=TAU["rise_i"],
                      postsynaptic_kernel_normalization_value=1.7)
        cls_of_size[k] = len(spec.classes)
        spec.classes.append(BatchClass(num_e, num_i, tuple(ws), e_conn, i_conn))
    for b in range(n_instances):
        c = cls_of_size[int(draws[b])]
        C = spec.classes[c]
        g_leak = float(np.float32(rng.uniform(8e-9, 12e-9)))
        amp = float(np.float32(rng.uniform(0.2e-9, 1.0e-9)))
        ids = np.sort(rng.choice(C.num_e, size=min(n_stim_ids, C.num_e), replace=False)).tolist()
        counts, sel, _, deltas = generation.partial_group_multiple_square_waves(
            steps, ids, [0] * len(ids), [stim_window[0]], [stim_window[1]], [amp])
        e_group = dict(NEURON, g_leak=g_leak, num_neurons=C.num_e)
        i_group = dict(NEURON, g_leak=g_leak, num_neurons=C.num_i)
        spec.instances.append(BatchInstance(c, e_group, i_group, seed * 100003 + b + 1, (counts, sel, deltas)))
    return spec


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class BatchSimulation:
    """One batch on one GPU, built from a BatchSpec."""

    FORMS = {"flow": 0, "phased": 1}

    def __init__(self, spec: BatchSpec, device: int = 0, noise: bool = True, library=None, form: str = "phased"):
        self._lib = library if library is not None else load_library()
        self._h = ctypes.c_void_p()
        self._check(self._lib.bsnn_batch_create(device, ctypes.byref(self._h)), creating=True)
        self.spec = spec
        self._sizes = []
        for C in spec.classes:
            w = [np.ascontiguousarray(x, dtype=np.float32) for x in C.weights]
            ep, ip = ConnectionParams.make(**C.e_conn), ConnectionParams.make(**C.i_conn)
            out = ctypes.c_uint32()
            self._check(self._lib.bsnn_batch_add_class(self._h, C.num_e, C.num_i, *[_ptr(x, ctypes.c_float) for x in w],
                                                       ctypes.byref(ep), ctypes.byref(ip), ctypes.byref(out)))
        for inst in spec.instances:
            C = spec.classes[inst.cls]
            ge = NeuronGroupParams.make(**dict(inst.e_group, offset=0, is_inhibitory=False))
            gi = NeuronGroupParams.make(**dict(inst.i_group, offset=C.num_e, is_inhibitory=True))
            counts, neurons, deltas = (np.ascontiguousarray(inst.stimulus[0], dtype=np.uint32),
                                       np.ascontiguousarray(inst.stimulus[1], dtype=np.uint32),
                                       np.ascontiguousarray(inst.stimulus[2], dtype=np.float32))
            out = ctypes.c_uint32()
            self._check(self._lib.bsnn_batch_add_instance(
                self._h, inst.cls, ctypes.byref(ge), ctypes.byref(gi), int(inst.seed), _ptr(counts, ctypes.c_uint32),
                counts.size, _ptr(neurons, ctypes.c_uint32), _ptr(deltas, ctypes.c_float), neurons.size,
                ctypes.byref(out)))
            self._sizes.append(C.num_e + C.num_i)
        if not noise:
            self._check(self._lib.bsnn_batch_set_noise(self._h, 0))
        self.set_form(form)

    def set_form(self, form: str):
        """How the kernel orders a clock step's work, before the first step: "flow" (each size
        class its own chain of neuron updates and GEMM units, overlapping) or "phased" (all
        neurons, grid barrier, all GEMM units, grid barrier).  Results are bit-identical."""
        if form not in self.FORMS:
            raise ValueError(f"unknown batch form {form!r}")
        self._check(self._lib.bsnn_batch_set_form(self._h, self.FORMS[form]))

    def _check(self, st, creating=False):
        if st != 0:
            msg = self._lib.bsnn_batch_last_error(None if creating else self._h)
            raise error_for(st, msg.decode() if msg else "")

    def run(self, num_steps: int):
        self._check(self._lib.bsnn_batch_run(self._h, num_steps))

    def set_steps_per_launch(self, steps: int):
        self._check(self._lib.bsnn_batch_set_steps_per_launch(self._h, steps))

    def set_device_wait_limit(self, seconds: float):
        """Bound of every device-side wait of the batch kernel (default 2 s)."""
        self._check(self._lib.bsnn_batch_set_device_wait_limit(self._h, int(round(seconds * 1e9))))

    def synchronize(self):
        self._check(self._lib.bsnn_batch_synchronize(self._h))

    def stream(self) -> int:
        p = ctypes.c_void_p()
        self._check(self._lib.bsnn_batch_get_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    def read(self, instance: int, name: str) -> np.ndarray:
        out = np.empty(self._sizes[instance], dtype=np.uint32 if name in UINT_FIELDS else np.float32)
        self._check(self._lib.bsnn_batch_read_state(self._h, instance, FIELD[name], out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def spike_counts(self) -> np.ndarray:
        out = np.empty((len(self._sizes), 2), dtype=np.uint64)
        self._check(self._lib.bsnn_batch_read_spike_counts(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out

    def autotune(self, trial_steps: int = 200) -> dict:
        """Times candidate GEMM unit sizes and ring depths (before the first step) and keeps the
        fastest; returns the choice."""
        from ._ffi import BatchTuning
        r = BatchTuning()
        self._check(self._lib.bsnn_batch_autotune(self._h, trial_steps, ctypes.byref(r)))
        return {"k_tiles_per_unit": r.k_tiles_per_unit, "operand_stages": r.operand_stages,
                "candidates": r.candidates, "us_per_step": r.us_per_step,
                "default_us_per_step": r.default_us_per_step}

    def set_tuning(self, tuning: dict):
        """Applies shapes an earlier autotune() returned (before the first step)."""
        from ._ffi import BatchTuning
        r = BatchTuning(tuning.get("k_tiles_per_unit", 0), tuning.get("operand_stages", 0), 0, 0.0, 0.0)
        self._check(self._lib.bsnn_batch_set_tuning(self._h, ctypes.byref(r)))

    def info(self):
        from ._ffi import BatchInfo
        i = BatchInfo()
        self._check(self._lib.bsnn_batch_get_info(self._h, ctypes.byref(i)))
        return i

    def close(self):
        if self._h:
            self._lib.bsnn_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
