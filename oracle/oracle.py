"""Python wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.  It
loads oracle/liboracle.so (built by oracle/Makefile) and exposes the same method names as
bsnn.Simulation so one NetworkSpec can be built into both.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "liboracle.so"

PREC_F32 = 32
PREC_F64 = 64

_FIELDS = {
    "membrane_potentials": 1, "g_excitatory": 2, "g_inhibitory": 3, "i_stimulus": 4, "refractory_counter": 5,
    "spikes": 6, "background_g_excitatory": 7, "background_g_inhibitory": 8, "background_excitatory_r_traces": 9,
    "background_excitatory_d_traces": 10, "background_inhibitory_r_traces": 11, "background_inhibitory_d_traces": 12,
    "connection_r_traces": 13, "connection_d_traces": 14, "connection_summed": 15, "plasticity_pre_traces": 16,
    "plasticity_post_traces": 17, "plasticity_triplet_pre_traces": 18, "plasticity_triplet_post_traces": 19,
    "plasticity_pre_weight_sums": 20,
}
_UINT = {"refractory_counter", "spikes"}

_lib = None


def build():
    subprocess.run(["make", "-C", str(ORACLE_DIR), "liboracle.so"], check=True, capture_output=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    lib = ctypes.CDLL(str(LIB_PATH))
    P, U32, I32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32
    sig = {
        "or_create": (P, [P, I32]), "or_destroy": (None, [P]), "or_last_error": (ctypes.c_char_p, [P]),
        "or_add_neuron_group": (I32, [P, P, P]), "or_add_connection": (I32, [P, U32, U32, P, P, P]),
        "or_add_stimulus": (I32, [P, P, U32, P, P, P, U32]), "or_add_plasticity": (I32, [P, I32, U32, P, P]),
        "or_add_spike_recorder": (I32, [P, U32, U32, P]), "or_add_voltage_recorder": (I32, [P, U32, P, U32, U32, P]),
        "or_set_noise_mode": (I32, [P, I32]), "or_set_noise_replay": (I32, [P, P, U32]),
        "or_step": (I32, [P, U32]), "or_run": (I32, [P, U32, U32]), "or_skip_steps": (I32, [P, U32]),
        "or_read_state": (I32, [P, I32, U32, U32, U32, P]), "or_read_state_f64": (I32, [P, I32, U32, U32, U32, P]),
        "or_write_state": (I32, [P, I32, U32, U32, U32, P]), "or_read_weights": (I32, [P, U32, P]),
        "or_read_weights_f64": (I32, [P, U32, P]), "or_write_weights": (I32, [P, U32, P]), "or_read_spike_history": (I32, [P, U32, P, I32]),
        "or_read_voltage_history": (I32, [P, U32, P, I32]), "or_last_noise_counts": (I32, [P, P]),
        "or_philox4x32_10": (None, [P, P, P]), "or_poisson": (U32, [ctypes.c_float, U32, U32, ctypes.c_uint64, U32]),
        "or_connection_propagate": (None, [ctypes.c_float, ctypes.c_float, ctypes.c_float, U32, U32, P, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def philox4x32_10(counter, key):
    lib = load()
    c = (ctypes.c_uint32 * 4)(*counter)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib.or_philox4x32_10(c, k, o)
    return list(o)


def poisson(exp_neg_mean, seed, neuron, step, channel):
    return load().or_poisson(exp_neg_mean, seed, neuron, step, channel)


def connection_propagate(r_decay, d_decay, norm, w, r, d, x, g, spikes):
    """One connection's propagation on numpy arrays, updated in place (r, d, x [n_pre] float32,
    g [n_post] float32, w [n_pre, n_post] float32, spikes [n_pre] uint32)."""
    n_pre, n_post = w.shape
    arrs = [np.ascontiguousarray(w, np.float32)]
    for a, dt in ((r, np.float32), (d, np.float32), (x, np.float32), (g, np.float32), (spikes, np.uint32)):
        assert a.dtype == dt and a.flags.c_contiguous
    load().or_connection_propagate(r_decay, d_decay, norm, n_pre, n_post, _vp(arrs[0]), _vp(r), _vp(d), _vp(x),
                                   _vp(g), _vp(spikes))


def _vp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleSimulation:
    """CPU restatement of the reference step (see oracle/bsnn_oracle.cpp)."""

    def __init__(self, num_excitatory_neurons, num_inhibitory_neurons, *, total_simulation_length=0,
                 num_stimulus_events=0, num_plasticities=0, recording_interval_steps=10000, rng_seed=314,
                 precision=PREC_F32, **_ignored):
        self._lib = load()
        from ctypes import Structure, c_int32, c_uint32

        class Desc(Structure):
            _fields_ = [("a", c_uint32), ("b", c_uint32), ("c", c_uint32), ("d", c_uint32), ("e", c_uint32),
                        ("f", c_uint32), ("g", c_int32), ("h", c_int32)]

        d = Desc(total_simulation_length, num_excitatory_neurons, num_inhibitory_neurons, num_stimulus_events,
                 num_plasticities, recording_interval_steps, rng_seed, 0)
        self._h = self._lib.or_create(ctypes.byref(d), precision)
        self.precision = precision
        self.num_neurons = num_excitatory_neurons + num_inhibitory_neurons
        self.recording_interval_steps = recording_interval_steps
        self._groups, self._conns, self._mons, self._plasts = [], [], [], []

    def _check(self, st):
        if st != 0:
            msg = self._lib.or_last_error(self._h).decode()
            exc = {1: ValueError, 2: IndexError}.get(st, RuntimeError)
            raise exc(f"[oracle status {st}] {msg}")

    def close(self):
        if self._h:
            self._lib.or_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_neuron_group(self, params):
        out = ctypes.c_uint32()
        self._check(self._lib.or_add_neuron_group(self._h, ctypes.byref(params), ctypes.byref(out)))
        self._groups.append((params.offset, params.num_neurons))
        return out.value

    def add_connection(self, pre, post, weights, params):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        out = ctypes.c_uint32()
        self._check(self._lib.or_add_connection(self._h, pre, post, _vp(w), ctypes.byref(params), ctypes.byref(out)))
        self._conns.append((self._groups[pre][1], self._groups[post][1]))
        return out.value

    def add_stimulus(self, counts, ids, offsets, deltas):
        c = np.ascontiguousarray(counts, dtype=np.uint32)
        i = np.ascontiguousarray(ids, dtype=np.uint32)
        o = np.ascontiguousarray(offsets, dtype=np.uint32)
        d = np.ascontiguousarray(deltas, dtype=np.float32)
        self._check(self._lib.or_add_stimulus(self._h, _vp(c), len(c), _vp(i), _vp(o), _vp(d), len(i)))

    def add_plasticity(self, kind, conn, params):
        out = ctypes.c_uint32()
        self._check(self._lib.or_add_plasticity(self._h, kind, conn, ctypes.byref(params), ctypes.byref(out)))
        self._plasts.append(conn)
        return out.value

    def add_spike_recorder(self, group, interval=0):
        out = ctypes.c_uint32()
        self._check(self._lib.or_add_spike_recorder(self._h, group, interval, ctypes.byref(out)))
        self._mons.append(("spikes", group, interval or self.recording_interval_steps, self._groups[group][1]))
        return out.value

    def add_voltage_recorder(self, group, selected_neurons=(), interval=0):
        ids = np.ascontiguousarray(selected_neurons, dtype=np.uint32)
        out = ctypes.c_uint32()
        self._check(self._lib.or_add_voltage_recorder(self._h, group, _vp(ids), len(ids), interval, ctypes.byref(out)))
        n_sel = len(ids) if len(ids) else self._groups[group][1]
        self._mons.append(("voltage", group, interval or self.recording_interval_steps, n_sel))
        return out.value

    def set_noise_mode(self, mode):
        self._check(self._lib.or_set_noise_mode(self._h, mode))

    def set_noise_replay(self, counts):
        c = np.ascontiguousarray(counts, dtype=np.uint8)
        self._check(self._lib.or_set_noise_replay(self._h, _vp(c), c.size // (2 * self.num_neurons)))

    def step(self, clock_step):
        self._check(self._lib.or_step(self._h, clock_step))

    def run(self, first_clock_step, num_steps):
        self._check(self._lib.or_run(self._h, first_clock_step, num_steps))

    def synchronize(self):
        pass

    def skip_steps(self, n):
        """Advances the step counter and stimulus cursors by n steps without simulating them."""
        self._check(self._lib.or_skip_steps(self._h, n))

    def _len(self, name, index):
        if name.startswith("connection_"):
            return self._conns[index][0]
        if name in ("plasticity_pre_traces", "plasticity_triplet_pre_traces", "plasticity_pre_weight_sums"):
            return self._conns[self._plasts[index]][0]
        if name in ("plasticity_post_traces", "plasticity_triplet_post_traces"):
            return self._conns[self._plasts[index]][1]
        return self.num_neurons

    def read(self, name, index=0, offset=0, count=None):
        if count is None:
            count = self._len(name, index) - offset
        out = np.empty(count, dtype=np.uint32 if name in _UINT else np.float32)
        self._check(self._lib.or_read_state(self._h, _FIELDS[name], index, offset, count, _vp(out)))
        return out

    def read_f64(self, name, index=0, offset=0, count=None):
        if count is None:
            count = self._len(name, index) - offset
        out = np.empty(count, dtype=np.float64)
        self._check(self._lib.or_read_state_f64(self._h, _FIELDS[name], index, offset, count, _vp(out)))
        return out

    def write(self, name, values, index=0, offset=0):
        a = np.ascontiguousarray(values, dtype=np.uint32 if name in _UINT else np.float32)
        self._check(self._lib.or_write_state(self._h, _FIELDS[name], index, offset, a.size, _vp(a)))

    def read_weights(self, conn):
        n_pre, n_post = self._conns[conn]
        out = np.empty((n_pre, n_post), dtype=np.float32)
        self._check(self._lib.or_read_weights(self._h, conn, _vp(out)))
        return out

    def write_weights(self, conn, weights):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        self._check(self._lib.or_write_weights(self._h, conn, _vp(w)))

    def read_weights_f64(self, conn):
        n_pre, n_post = self._conns[conn]
        out = np.empty((n_pre, n_post), dtype=np.float64)
        self._check(self._lib.or_read_weights_f64(self._h, conn, _vp(out)))
        return out

    def read_spike_history(self, monitor, flush=False):
        kind, group, interval, n = self._mons[monitor]
        out = np.empty((n, interval), dtype=np.uint32)
        self._check(self._lib.or_read_spike_history(self._h, monitor, _vp(out), int(flush)))
        return out

    def read_voltage_history(self, monitor, flush=False):
        kind, group, interval, n_sel = self._mons[monitor]
        out = np.empty((n_sel, interval), dtype=np.float32)
        self._check(self._lib.or_read_voltage_history(self._h, monitor, _vp(out), int(flush)))
        return out

    def last_noise_counts(self):
        out = np.empty(self.num_neurons * 2, dtype=np.uint8)
        self._check(self._lib.or_last_noise_counts(self._h, _vp(out)))
        return out.reshape(self.num_neurons, 2)
