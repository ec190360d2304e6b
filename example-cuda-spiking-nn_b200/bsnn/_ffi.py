"""ctypes bindings of include/bsnn.h (the C-ABI of libbsnn).

The structure layouts below are the C structs of include/bsnn.h, which in turn repeat the
reference's parameter PODs field by field:
  NeuronGroupParams  cpp_src/neuron_groups/neuron_group_params.h:7-31
  ConnectionParams   cpp_src/connections/connection_params.h:7-14
  PlasticityParams   cpp_src/plasticities/plasticity_params.h:7-20
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent.parent
LIBRARY_PATH = PACKAGE_DIR / "libbsnn.so"

# status codes
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_RANGE = 2
ERR_RUNTIME = 3
ERR_CUDA = 4
ERR_DEVICE_TIMEOUT = 5
ERR_STATE = 6

PLASTICITY_TRIPLET = 1
PLASTICITY_ISTDP = 2
PLASTICITY_STDP = 3

NOISE_PHILOX = 0
NOISE_OFF = 1
NOISE_REPLAY = 2

# Weight storage forms (bsnn_set_weight_format).
WEIGHTS_F32 = 0
WEIGHTS_F32_ROWSCALED = 1
WEIGHTS_BF16 = 2
WEIGHTS_FP8_E4M3 = 3
WEIGHT_FORMATS = {"f32": WEIGHTS_F32, "f32_rowscaled": WEIGHTS_F32_ROWSCALED, "bf16": WEIGHTS_BF16,
                  "fp8_e4m3": WEIGHTS_FP8_E4M3}

FIELD = {
    "membrane_potentials": 1,
    "g_excitatory": 2,
    "g_inhibitory": 3,
    "i_stimulus": 4,
    "refractory_counter": 5,
    "spikes": 6,
    "background_g_excitatory": 7,
    "background_g_inhibitory": 8,
    "background_excitatory_r_traces": 9,
    "background_excitatory_d_traces": 10,
    "background_inhibitory_r_traces": 11,
    "background_inhibitory_d_traces": 12,
    "connection_r_traces": 13,
    "connection_d_traces": 14,
    "connection_summed": 15,
    "plasticity_pre_traces": 16,
    "plasticity_post_traces": 17,
    "plasticity_triplet_pre_traces": 18,
    "plasticity_triplet_post_traces": 19,
    "plasticity_pre_weight_sums": 20,
    "connection_row_scale": 21,
    "connection_row_master_sum": 22,
    "connection_row_quant_scale": 23,
}
UINT_FIELDS = {"refractory_counter", "spikes"}


class BsnnError(RuntimeError):
    """Base of the errors raised for a non-zero bsnn_status."""


class InvalidArgument(BsnnError, ValueError):
    """std::invalid_argument in the reference."""


class OutOfRange(BsnnError, IndexError):
    """std::out_of_range in the reference."""


class CudaError(BsnnError):
    """A CUDA runtime call failed (cuda_check in the reference)."""


class DeviceTimeout(BsnnError, TimeoutError):
    """A bounded device-side wait gave up; the simulation state is invalid."""


class StateError(BsnnError):
    """A call was made in the wrong lifecycle state."""


_ERRORS = {
    ERR_INVALID_ARGUMENT: InvalidArgument,
    ERR_OUT_OF_RANGE: OutOfRange,
    ERR_RUNTIME: BsnnError,
    ERR_CUDA: CudaError,
    ERR_DEVICE_TIMEOUT: DeviceTimeout,
    ERR_STATE: StateError,
}


def error_for(status: int, message: str) -> BsnnError:
    return _ERRORS.get(status, BsnnError)(f"[bsnn status {status}] {message}")


class NeuronGroupParams(ctypes.Structure):
    _fields_ = [
        ("timestep", ctypes.c_float),
        ("g_leak", ctypes.c_float),
        ("membrane_capacitance", ctypes.c_float),
        ("depolarization_slope_factor", ctypes.c_float),
        ("v_effective_spike_threshold", ctypes.c_float),
        ("v_excitatory_reversal", ctypes.c_float),
        ("v_inhibitory_reversal", ctypes.c_float),
        ("v_threshold", ctypes.c_float),
        ("v_reset", ctypes.c_float),
        ("v_rest", ctypes.c_float),
        ("refractory_steps", ctypes.c_uint32),
        ("is_inhibitory", ctypes.c_bool),
        ("mean_background_excitatory_spikes", ctypes.c_float),
        ("mean_background_inhibitory_spikes", ctypes.c_float),
        ("background_excitatory_postsynaptic_r_trace_decay", ctypes.c_float),
        ("background_excitatory_postsynaptic_d_trace_decay", ctypes.c_float),
        ("background_inhibitory_postsynaptic_r_trace_decay", ctypes.c_float),
        ("background_inhibitory_postsynaptic_d_trace_decay", ctypes.c_float),
        ("background_excitatory_scaling_factor", ctypes.c_float),
        ("background_inhibitory_scaling_factor", ctypes.c_float),
        ("offset", ctypes.c_uint32),
        ("num_neurons", ctypes.c_uint32),
    ]

    # Defaults of the reference struct's member initialisers.
    DEFAULTS = dict(
        timestep=1e-4, g_leak=10.0, membrane_capacitance=0.1, depolarization_slope_factor=2.0,
        v_effective_spike_threshold=-50.0, v_excitatory_reversal=0.0, v_inhibitory_reversal=-80.0,
        v_threshold=-45.0, v_reset=-55.0, v_rest=-65.0, refractory_steps=0, is_inhibitory=False,
        mean_background_excitatory_spikes=0.0, mean_background_inhibitory_spikes=0.0,
        background_excitatory_postsynaptic_r_trace_decay=0.0,
        background_excitatory_postsynaptic_d_trace_decay=0.0,
        background_inhibitory_postsynaptic_r_trace_decay=0.0,
        background_inhibitory_postsynaptic_d_trace_decay=0.0,
        background_excitatory_scaling_factor=0.0, background_inhibitory_scaling_factor=0.0,
        offset=0, num_neurons=0,
    )

    @classmethod
    def make(cls, **kw):
        vals = dict(cls.DEFAULTS)
        unknown = set(kw) - set(vals)
        if unknown:
            raise TypeError(f"unknown NeuronGroupParams fields: {sorted(unknown)}")
        vals.update(kw)
        return cls(**vals)


class ConnectionParams(ctypes.Structure):
    _fields_ = [
        ("timestep", ctypes.c_float),
        ("decay_time", ctypes.c_float),
        ("rise_time", ctypes.c_float),
        ("postsynaptic_kernel_normalization_value", ctypes.c_float),
        ("weight_matrix_idx", ctypes.c_uint32),
    ]
    DEFAULTS = dict(timestep=0.0, decay_time=0.0, rise_time=0.0, postsynaptic_kernel_normalization_value=0.0,
                    weight_matrix_idx=0)

    @classmethod
    def make(cls, **kw):
        vals = dict(cls.DEFAULTS)
        vals.update(kw)
        return cls(**vals)


class PlasticityParams(ctypes.Structure):
    _fields_ = [
        ("ltp_A", ctypes.c_float),
        ("ltd_A", ctypes.c_float),
        ("ltp_B", ctypes.c_float),
        ("ltd_B", ctypes.c_float),
        ("pre_trace_decay", ctypes.c_float),
        ("post_trace_decay", ctypes.c_float),
        ("triplet_pre_trace_decay", ctypes.c_float),
        ("triplet_post_trace_decay", ctypes.c_float),
        ("weight_min", ctypes.c_float),
        ("weight_max", ctypes.c_float),
        ("plasticity_offset", ctypes.c_uint32),
    ]
    DEFAULTS = dict(ltp_A=0.0, ltd_A=0.0, ltp_B=0.0, ltd_B=0.0, pre_trace_decay=0.0, post_trace_decay=0.0,
                    triplet_pre_trace_decay=0.0, triplet_post_trace_decay=0.0, weight_min=0.0, weight_max=1.0,
                    plasticity_offset=0)

    @classmethod
    def make(cls, **kw):
        vals = dict(cls.DEFAULTS)
        vals.update(kw)
        return cls(**vals)


class StateDesc(ctypes.Structure):
    _fields_ = [
        ("total_simulation_length", ctypes.c_uint32),
        ("num_excitatory_neurons", ctypes.c_uint32),
        ("num_inhibitory_neurons", ctypes.c_uint32),
        ("num_stimulus_events", ctypes.c_uint32),
        ("num_plasticities", ctypes.c_uint32),
        ("recording_interval_steps", ctypes.c_uint32),
        ("rng_seed", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("total_neurons", ctypes.c_uint32),
        ("num_groups", ctypes.c_uint32),
        ("num_connections", ctypes.c_uint32),
        ("num_plasticities", ctypes.c_uint32),
        ("num_monitors", ctypes.c_uint32),
        ("grid_ctas", ctypes.c_uint32),
        ("block_threads", ctypes.c_uint32),
        ("steps_per_launch", ctypes.c_uint32),
        ("steps_done", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
        ("weight_bytes", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint64),
        ("smem_bytes", ctypes.c_uint64),
        ("resident_bytes", ctypes.c_uint64),
    ]


class ConnectionView(ctypes.Structure):
    """ConnectionView (cpp_src/connections/connection_view.h:8-31): device pointers of one connection."""
    _fields_ = [
        ("postsynaptic_r_trace_decay", ctypes.c_float),
        ("postsynaptic_d_trace_decay", ctypes.c_float),
        ("postsynaptic_kernel_normalization_value", ctypes.c_float),
        ("pre_group_is_inhibtory", ctypes.c_bool),
        ("weight_matrix_idx", ctypes.c_uint32),
        ("pre_group_offset", ctypes.c_uint32),
        ("post_group_offset", ctypes.c_uint32),
        ("pre_group_num_neurons", ctypes.c_uint32),
        ("post_group_num_neurons", ctypes.c_uint32),
        ("weight_matrix", ctypes.c_void_p),
        ("postsynaptic_r_traces", ctypes.c_void_p),
        ("postsynaptic_d_traces", ctypes.c_void_p),
        ("summed_postsynaptic_conductances", ctypes.c_void_p),
        ("post_group_g_excitatory", ctypes.c_void_p),
        ("post_group_g_inhibitory", ctypes.c_void_p),
        ("spikes", ctypes.c_void_p),
        ("cublas_handle", ctypes.c_void_p),
    ]


# Exported symbols and their signatures (every entry point declared in include/bsnn.h).
class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("num_classes", ctypes.c_uint32),
        ("num_instances", ctypes.c_uint32),
        ("num_neurons", ctypes.c_uint32),
        ("num_units", ctypes.c_uint32),
        ("grid_ctas", ctypes.c_uint32),
        ("block_threads", ctypes.c_uint32),
        ("steps_done", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
        ("weight_bytes", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint64),
        ("smem_bytes", ctypes.c_uint64),
        ("state_in_smem", ctypes.c_uint32),
        ("operand_stages", ctypes.c_uint32),
        ("form", ctypes.c_int32),
    ]


class AdjointDesc(ctypes.Structure):
    """bsnn_adjoint_desc."""
    _fields_ = [("num_excitatory", ctypes.c_uint32), ("num_inhibitory", ctypes.c_uint32),
                ("num_steps", ctypes.c_uint32), ("checkpoint_interval", ctypes.c_uint32),
                ("rng_seed", ctypes.c_int32), ("noise_on", ctypes.c_int32), ("rate_tau", ctypes.c_float),
                ("surrogate_beta", ctypes.c_float), ("rate_weight", ctypes.c_float), ("voltage_weight", ctypes.c_float)]


class BatchTuning(ctypes.Structure):
    """bsnn_batch_tuning."""
    _fields_ = [("k_tiles_per_unit", ctypes.c_uint32), ("operand_stages", ctypes.c_uint32),
                ("candidates", ctypes.c_uint32), ("us_per_step", ctypes.c_float),
                ("default_us_per_step", ctypes.c_float)]


class WeightGenerationParams(ctypes.Structure):
    """bsnn_weight_generation_params."""
    _fields_ = [("max_weight_value", ctypes.c_float), ("max_distance", ctypes.c_float),
                ("spread_scale", ctypes.c_float), ("probability_multiplier", ctypes.c_float),
                ("x_location_length", ctypes.c_float), ("y_location_length", ctypes.c_float),
                ("weight_value_normal_dropoff", ctypes.c_int32), ("probabilistic_normal_not_uniform", ctypes.c_int32),
                ("no_diagonal_connections", ctypes.c_int32), ("uniform_values", ctypes.c_int32)]


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_I32 = ctypes.c_int32
_FP = ctypes.POINTER(ctypes.c_float)
_UP = ctypes.POINTER(ctypes.c_uint32)
SIGNATURES = {
    "bsnn_version": (ctypes.c_char_p, []),
    "bsnn_create": (_I32, [ctypes.POINTER(StateDesc), ctypes.POINTER(_P)]),
    "bsnn_destroy": (_I32, [_P]),
    "bsnn_last_error": (ctypes.c_char_p, [_P]),
    "bsnn_batch_create": (_I32, [_I32, ctypes.POINTER(_P)]),
    "bsnn_batch_destroy": (_I32, [_P]),
    "bsnn_batch_last_error": (ctypes.c_char_p, [_P]),
    "bsnn_batch_add_class": (_I32, [_P, _U32, _U32, _FP, _FP, _FP, _FP, _P, _P, ctypes.POINTER(_U32)]),
    "bsnn_batch_add_instance": (_I32, [_P, _U32, _P, _P, _I32, ctypes.POINTER(_U32), _U32, ctypes.POINTER(_U32), _FP,
                                       _U32, ctypes.POINTER(_U32)]),
    "bsnn_batch_set_noise": (_I32, [_P, _I32]),
    "bsnn_batch_set_steps_per_launch": (_I32, [_P, _U32]),
    "bsnn_batch_set_form": (_I32, [_P, _I32]),
    "bsnn_batch_set_device_wait_limit": (_I32, [_P, ctypes.c_uint64]),
    "bsnn_batch_run": (_I32, [_P, _U32]),
    "bsnn_batch_synchronize": (_I32, [_P]),
    "bsnn_batch_get_stream": (_I32, [_P, ctypes.POINTER(_P)]),
    "bsnn_batch_read_state": (_I32, [_P, _U32, _I32, _P]),
    "bsnn_batch_read_spike_counts": (_I32, [_P, ctypes.POINTER(ctypes.c_uint64)]),
    "bsnn_batch_get_info": (_I32, [_P, ctypes.POINTER(BatchInfo)]),
    "bsnn_batch_autotune": (_I32, [_P, _U32, ctypes.POINTER(BatchTuning)]),
    "bsnn_batch_set_tuning": (_I32, [_P, ctypes.POINTER(BatchTuning)]),
    "bsnn_adjoint_create": (_I32, [ctypes.POINTER(AdjointDesc), _P, _P, _P, _P, _FP, _FP, _FP, _FP, _UP, _U32, _UP, _FP,
                                   _U32, _I32, ctypes.POINTER(_P)]),
    "bsnn_adjoint_destroy": (_I32, [_P]),
    "bsnn_adjoint_last_error": (ctypes.c_char_p, [_P]),
    "bsnn_adjoint_set_params": (_I32, [_P, _FP, ctypes.c_float]),
    "bsnn_adjoint_get_stream": (_I32, [_P, ctypes.POINTER(_P)]),
    "bsnn_adjoint_kernel_launches": (_I32, [_P, ctypes.POINTER(ctypes.c_uint64)]),
    "bsnn_adjoint_forward": (_I32, [_P, _FP, _FP, _FP, _FP, _FP]),
    "bsnn_adjoint_backward": (_I32, [_P, _FP, ctypes.POINTER(ctypes.c_double)]),
    "bsnn_get_info": (_I32, [_P, ctypes.POINTER(Info)]),
    "bsnn_generate_distance_weights": (_I32, [_FP, _U32, _FP, _U32, ctypes.POINTER(WeightGenerationParams),
                                              ctypes.c_uint64, _I32, _FP]),
    "bsnn_save_checkpoint": (_I32, [_P, ctypes.c_char_p]),
    "bsnn_load_checkpoint": (_I32, [_P, ctypes.c_char_p]),
    "bsnn_add_neuron_group": (_I32, [_P, ctypes.POINTER(NeuronGroupParams), _UP]),
    "bsnn_add_connection": (_I32, [_P, _U32, _U32, _FP, ctypes.POINTER(ConnectionParams), _UP]),
    "bsnn_add_stimulus": (_I32, [_P, _UP, _U32, _UP, _UP, _FP, _U32]),
    "bsnn_add_plasticity": (_I32, [_P, _I32, _U32, ctypes.POINTER(PlasticityParams), _UP]),
    "bsnn_add_spike_recorder": (_I32, [_P, _U32, _U32, _UP]),
    "bsnn_add_voltage_recorder": (_I32, [_P, _U32, _UP, _U32, _U32, _UP]),
    "bsnn_set_noise_mode": (_I32, [_P, _I32]),
    "bsnn_set_noise_replay": (_I32, [_P, ctypes.POINTER(ctypes.c_uint8), _U32]),
    "bsnn_set_weight_format": (_I32, [_P, _I32]),
    "bsnn_step": (_I32, [_P, _U32]),
    "bsnn_run": (_I32, [_P, _U32, _U32]),
    "bsnn_synchronize": (_I32, [_P]),
    "bsnn_get_stream": (_I32, [_P, ctypes.POINTER(_P)]),
    "bsnn_set_steps_per_launch": (_I32, [_P, _U32]),
    "bsnn_set_device_wait_limit": (_I32, [_P, ctypes.c_uint64]),
    "bsnn_debug_skip_arrival": (_I32, [_P, _U32, ctypes.c_uint64]),
    "bsnn_measure_exchange_floor": (_I32, [_P, _U32, ctypes.POINTER(ctypes.c_float)]),
    "bsnn_read_state": (_I32, [_P, _I32, _U32, _U32, _U32, _P]),
    "bsnn_write_state": (_I32, [_P, _I32, _U32, _U32, _U32, _P]),
    "bsnn_read_weights": (_I32, [_P, _U32, _FP]),
    "bsnn_read_weight_copy": (_I32, [_P, _U32, _P]),
    "bsnn_read_spike_history": (_I32, [_P, _U32, _UP, _I32]),
    "bsnn_read_spike_bits": (_I32, [_P, _U32, _UP, _I32]),
    "bsnn_read_voltage_history": (_I32, [_P, _U32, _FP, _I32]),
    "bsnn_get_device_pointer": (_I32, [_P, _I32, _U32, ctypes.POINTER(_P)]),
    "bsnn_set_monitor_output": (_I32, [_P, _U32, ctypes.c_char_p]),
    "bsnn_add_weight_recorder": (_I32, [_P, _U32, ctypes.c_char_p]),
    "bsnn_record": (_I32, [_P, _U32]),
    "bsnn_flush_records": (_I32, [_P]),
    "bsnn_run_system": (_I32, [_P, _U32]),
    "bsnn_set_progress_output": (_I32, [_P, _I32]),
    "bsnn_memory_report": (_I32, [_P, ctypes.c_char_p, ctypes.c_uint64]),
    "bsnn_connection_propagate": (_I32, [ctypes.POINTER(ConnectionView), _P]),
    "bsnn_connection_propagate_noalloc": (_I32, [ctypes.POINTER(ConnectionView), _P]),
}

_lib = None


def load_library(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Loads libbsnn.so (built in-tree by __graft_entry__.build / the package Makefile).

    There is no fallback: without the CUDA library nothing in this package can run.
    """
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIBRARY_PATH
    if not p.exists():
        raise ImportError(f"libbsnn.so not found at {p}; build it first (make -C {PACKAGE_DIR})")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
