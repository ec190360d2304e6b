"""Python handle over one libbsnn simulation (the C-ABI of include/bsnn.h).

`Simulation` mirrors the reference's GpuSimulationState plus the component constructors and the
step loop: add_neuron_group / add_connection / add_stimulus / add_plasticity / add_*_recorder,
then step (System::step_the_clock) or run (System::run's step loop).  Every call goes through
the C-ABI; numpy arrays are passed as plain pointers.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _ffi
from ._ffi import (FIELD, UINT_FIELDS, ConnectionParams, ConnectionView, Info, NeuronGroupParams, PlasticityParams,
                   StateDesc, error_for)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class Simulation:
    """One network on one GPU, driven through libbsnn."""

    def __init__(self, num_excitatory_neurons: int, num_inhibitory_neurons: int, *, total_simulation_length: int = 0,
                 num_stimulus_events: int = 0, num_plasticities: int = 0, recording_interval_steps: int = 10000,
                 rng_seed: int = 314, device: int = 0, library=None):
        self._lib = library if library is not None else _ffi.load_library()
        self._h = ctypes.c_void_p()
        desc = StateDesc(total_simulation_length, num_excitatory_neurons, num_inhibitory_neurons, num_stimulus_events,
                         num_plasticities, recording_interval_steps, rng_seed, device)
        st = self._lib.bsnn_create(ctypes.byref(desc), ctypes.byref(self._h))
        if st != 0:
            raise error_for(st, self._lib.bsnn_last_error(None).decode())
        self.num_neurons = num_excitatory_neurons + num_inhibitory_neurons
        self.recording_interval_steps = recording_interval_steps
        self._groups: list[tuple[int, int]] = []
        self._conns: list[tuple[int, int]] = []
        self._mons: list[tuple[str, int, int, int]] = []

    # -- plumbing ---------------------------------------------------------------------------
    def _check(self, st: int):
        if st != 0:
            raise error_for(st, self._lib.bsnn_last_error(self._h).decode())

    def close(self):
        if self._h:
            self._lib.bsnn_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def info(self) -> Info:
        i = Info()
        self._check(self._lib.bsnn_get_info(self._h, ctypes.byref(i)))
        return i

    def stream(self) -> int:
        p = ctypes.c_void_p()
        self._check(self._lib.bsnn_get_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    # -- components -------------------------------------------------------------------------
    def add_neuron_group(self, params: NeuronGroupParams) -> int:
        out = ctypes.c_uint32()
        self._check(self._lib.bsnn_add_neuron_group(self._h, ctypes.byref(params), ctypes.byref(out)))
        self._groups.append((params.offset, params.num_neurons))
        return out.value

    def add_connection(self, pre_group: int, post_group: int, weights: np.ndarray, params: ConnectionParams) -> int:
        w = np.ascontiguousarray(weights, dtype=np.float32)
        n_pre, n_post = self._groups[pre_group][1], self._groups[post_group][1]
        if w.shape != (n_pre, n_post):
            # Connection::Connection (cpp_src/connections/connection.cpp:18-20)
            raise _ffi.InvalidArgument(
                "Weight matrix size does not match the number of connections between pre and post groups.")
        out = ctypes.c_uint32()
        self._check(self._lib.bsnn_add_connection(self._h, pre_group, post_group, _ptr(w, ctypes.c_float),
                                                  ctypes.byref(params), ctypes.byref(out)))
        self._conns.append((n_pre, n_post))
        return out.value

    def add_stimulus(self, timestep_event_count, neuron_ids, post_group_offsets, amplitude_changes):
        c = np.ascontiguousarray(timestep_event_count, dtype=np.uint32)
        i = np.ascontiguousarray(neuron_ids, dtype=np.uint32)
        o = np.ascontiguousarray(post_group_offsets, dtype=np.uint32)
        d = np.ascontiguousarray(amplitude_changes, dtype=np.float32)
        self._check(self._lib.bsnn_add_stimulus(self._h, _ptr(c, ctypes.c_uint32), len(c), _ptr(i, ctypes.c_uint32),
                                                _ptr(o, ctypes.c_uint32), _ptr(d, ctypes.c_float), len(i)))

    def add_plasticity(self, kind: int, connection: int, params: PlasticityParams) -> int:
        out = ctypes.c_uint32()
        self._check(self._lib.bsnn_add_plasticity(self._h, kind, connection, ctypes.byref(params), ctypes.byref(out)))
        return out.value

    def add_spike_recorder(self, group: int, interval: int = 0) -> int:
        out = ctypes.c_uint32()
        self._check(self._lib.bsnn_add_spike_recorder(self._h, group, interval, ctypes.byref(out)))
        self._mons.append(("spikes", group, interval or self.recording_interval_steps, self._groups[group][1]))
        return out.value

    def add_voltage_recorder(self, group: int, selected_neurons=(), interval: int = 0) -> int:
        ids = np.ascontiguousarray(selected_neurons, dtype=np.uint32)
        out = ctypes.c_uint32()
        self._check(self._lib.bsnn_add_voltage_recorder(self._h, group, _ptr(ids, ctypes.c_uint32), len(ids), interval,
                                                        ctypes.byref(out)))
        n_sel = len(ids) if len(ids) else self._groups[group][1]
        self._mons.append(("voltage", group, interval or self.recording_interval_steps, n_sel))
        return out.value

    def set_noise_mode(self, mode: int):
        self._check(self._lib.bsnn_set_noise_mode(self._h, mode))

    def set_noise_replay(self, counts: np.ndarray):
        c = np.ascontiguousarray(counts, dtype=np.uint8)
        n_steps = c.size // (2 * self.num_neurons)
        self._check(self._lib.bsnn_set_noise_replay(self._h, _ptr(c, ctypes.c_uint8), n_steps))

    def set_weight_format(self, form):
        """Weight storage form: "f32" (the reference's arithmetic), "f32_rowscaled", "bf16" or
        "fp8_e4m3" (FP32 masters with a per-row normalisation scale; the propagation reads a copy
        of the masters in that type).  Before the first step."""
        from ._ffi import WEIGHT_FORMATS
        code = WEIGHT_FORMATS[form] if isinstance(form, str) else int(form)
        self._check(self._lib.bsnn_set_weight_format(self._h, code))
        self._weight_format = code

    # -- hot path ---------------------------------------------------------------------------
    def step(self, clock_step: int):
        self._check(self._lib.bsnn_step(self._h, clock_step))

    def run(self, first_clock_step: int, num_steps: int):
        self._check(self._lib.bsnn_run(self._h, first_clock_step, num_steps))

    def synchronize(self):
        self._check(self._lib.bsnn_synchronize(self._h))

    def set_steps_per_launch(self, steps: int):
        self._check(self._lib.bsnn_set_steps_per_launch(self._h, steps))

    def set_device_wait_limit(self, seconds: float):
        """Bound of every device-side wait of the persistent kernel (default 2 s)."""
        self._check(self._lib.bsnn_set_device_wait_limit(self._h, int(round(seconds * 1e9))))

    def exchange_floor_us(self, steps: int = 2000) -> float:
        """Latency floor of one clock step (microseconds): the partial-sum exchange and grid barrier
        of the persistent kernel run alone, with this network's grid and plan."""
        out = ctypes.c_float()
        self._check(self._lib.bsnn_measure_exchange_floor(self._h, steps, ctypes.byref(out)))
        return float(out.value)

    def debug_skip_arrival(self, cta: int, step: int):
        """Test switch: CTA `cta` skips its arrival at the grid barrier ending internal step `step`."""
        self._check(self._lib.bsnn_debug_skip_arrival(self._h, cta, step))

    # -- state ------------------------------------------------------------------------------
    def _field_len(self, name: str, index: int) -> int:
        if name.startswith("connection_"):
            return self._conns[index][0]
        if name in ("plasticity_post_traces", "plasticity_triplet_post_traces"):
            raise KeyError("pass count explicitly for plasticity post traces")
        if name.startswith("plasticity_"):
            raise KeyError("pass count explicitly for plasticity fields")
        return self.num_neurons

    def read(self, name: str, index: int = 0, offset: int = 0, count: int | None = None) -> np.ndarray:
        if count is None:
            count = self._field_len(name, index) - offset
        out = np.empty(count, dtype=np.uint32 if name in UINT_FIELDS else np.float32)
        self._check(self._lib.bsnn_read_state(self._h, FIELD[name], index, offset, count, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def write(self, name: str, values, index: int = 0, offset: int = 0):
        a = np.ascontiguousarray(values, dtype=np.uint32 if name in UINT_FIELDS else np.float32)
        self._check(self._lib.bsnn_write_state(self._h, FIELD[name], index, offset, a.size, a.ctypes.data_as(ctypes.c_void_p)))

    def save_checkpoint(self, path):
        """Writes the whole device state and the clock cursor to `path` (binary)."""
        self._check(self._lib.bsnn_save_checkpoint(self._h, str(path).encode()))

    def load_checkpoint(self, path):
        """Restores a checkpoint written by a simulation built from the same components."""
        self._check(self._lib.bsnn_load_checkpoint(self._h, str(path).encode()))

    def read_weights(self, connection: int) -> np.ndarray:
        n_pre, n_post = self._conns[connection]
        out = np.empty((n_pre, n_post), dtype=np.float32)
        self._check(self._lib.bsnn_read_weights(self._h, connection, _ptr(out, ctypes.c_float)))
        return out

    def read_weight_copy(self, connection: int) -> np.ndarray:
        """Row-scaled forms: the propagation's copy of the masters as stored -- float32, BF16 bit
        patterns (uint16) or E4M3 bytes (uint8), [pre, post]."""
        from ._ffi import WEIGHTS_BF16, WEIGHTS_FP8_E4M3
        n_pre, n_post = self._conns[connection]
        fmt = getattr(self, "_weight_format", 0)
        dt = np.uint16 if fmt == WEIGHTS_BF16 else np.uint8 if fmt == WEIGHTS_FP8_E4M3 else np.float32
        out = np.empty((n_pre, n_post), dtype=dt)
        self._check(self._lib.bsnn_read_weight_copy(self._h, connection, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def read_spike_history(self, monitor: int, flush: bool = False) -> np.ndarray:
        """[neuron, slot] uint32 0/1, the reference's download_and_flush_spike_history layout."""
        kind, group, interval, n = self._mons[monitor]
        out = np.empty((n, interval), dtype=np.uint32)
        self._check(self._lib.bsnn_read_spike_history(self._h, monitor, _ptr(out, ctypes.c_uint32), int(flush)))
        return out

    def read_spike_bits(self, monitor: int, flush: bool = False) -> np.ndarray:
        kind, group, interval, n = self._mons[monitor]
        out = np.empty((interval, (n + 31) // 32), dtype=np.uint32)
        self._check(self._lib.bsnn_read_spike_bits(self._h, monitor, _ptr(out, ctypes.c_uint32), int(flush)))
        return out

    def read_voltage_history(self, monitor: int, flush: bool = False) -> np.ndarray:
        """[selected neuron, slot] float32."""
        kind, group, interval, n_sel = self._mons[monitor]
        out = np.empty((n_sel, interval), dtype=np.float32)
        self._check(self._lib.bsnn_read_voltage_history(self._h, monitor, _ptr(out, ctypes.c_float), int(flush)))
        return out

    # -- recording to text files (Monitor::record) ------------------------------------------------
    def set_monitor_output(self, monitor: int, path) -> None:
        """Output file of a spike or voltage recorder (the reference's output_filepath)."""
        self._check(self._lib.bsnn_set_monitor_output(self._h, monitor, str(path).encode()))

    def add_weight_recorder(self, connection: int, path) -> None:
        """WeightRecorder: weight triples at recorded clock steps that are multiples of 100,000."""
        self._check(self._lib.bsnn_add_weight_recorder(self._h, connection, str(path).encode()))

    def record(self, clock_step: int) -> None:
        """Monitor::record(clock_step) of every recorder with an output."""
        self._check(self._lib.bsnn_record(self._h, clock_step))

    def flush_records(self) -> None:
        """Waits until every queued record is written."""
        self._check(self._lib.bsnn_flush_records(self._h))

    def run_system(self, total_clock_steps: int) -> None:
        """System::run without callbacks: steps 0 .. total-1, recording at multiples of the interval."""
        self._check(self._lib.bsnn_run_system(self._h, total_clock_steps))

    def set_progress_output(self, enabled: bool) -> None:
        """run_system prints System::run's "Completed clock step: ... | elapsed: ...s" lines."""
        self._check(self._lib.bsnn_set_progress_output(self._h, 1 if enabled else 0))

    def memory_report(self) -> str:
        """GpuSimulationState::memory_report: "Total GPU Memory Allocated: <bytes> bytes (<MB> MB)".
        Finalises the network (allocates its device arena) when it has not run yet."""
        buf = ctypes.create_string_buffer(256)
        self._check(self._lib.bsnn_memory_report(self._h, buf, len(buf)))
        return buf.value.decode()

    def device_pointer(self, name: str, index: int = 0) -> int:
        p = ctypes.c_void_p()
        self._check(self._lib.bsnn_get_device_pointer(self._h, FIELD[name], index, ctypes.byref(p)))
        return p.value or 0


def connection_propagate(view: ConnectionView, stream: int = 0, library=None):
    """kernel_connection_propagate_launch (cpp_src/connections/kernel_connection_propagate.cu:64-111) on
    caller-owned device buffers described by `view`; queued on `stream` (a cudaStream_t address, 0 =
    legacy default stream).  Raises the BsnnError subclass of the returned status."""
    lib = library if library is not None else _ffi.load_library()
    st = lib.bsnn_connection_propagate(ctypes.byref(view), ctypes.c_void_p(stream or None))
    if st != 0:
        raise error_for(st, lib.bsnn_last_error(None).decode())
