"""C-ABI checks that need no GPU: the library loads, exports every entry point declared in
include/bsnn.h, and the product path fails loudly (no CPU fallback) when no GPU is present."""
from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT, gpu_available


def declared_entry_points():
    text = (ROOT / "include" / "bsnn.h").read_text()
    return sorted(set(re.findall(r"BSNN_API\s+[\w\s\*]+?\b(bsnn_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_entry_points()
    for must in ("bsnn_create", "bsnn_destroy", "bsnn_add_neuron_group", "bsnn_add_connection", "bsnn_add_stimulus",
                 "bsnn_add_plasticity", "bsnn_step", "bsnn_run", "bsnn_read_state", "bsnn_read_weights"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import bsnn
    lib = bsnn.load_library()
    missing = [n for n in declared_entry_points() if not hasattr(lib, n)]
    assert not missing, f"libbsnn.so does not export {missing}"
    # and the Python bindings cover them all
    from bsnn._ffi import SIGNATURES
    assert set(declared_entry_points()) <= set(SIGNATURES)


def test_version_string():
    import bsnn
    assert b"sm_100a" in bsnn.load_library().bsnn_version()


def test_struct_layouts_match_reference_field_order():
    # NeuronGroupParams: 10 floats, uint32, bool, 8 floats, 2 uint32 (neuron_group_params.h:7-31)
    from bsnn._ffi import ConnectionParams, NeuronGroupParams, PlasticityParams
    assert [f[0] for f in NeuronGroupParams._fields_][:12] == [
        "timestep", "g_leak", "membrane_capacitance", "depolarization_slope_factor", "v_effective_spike_threshold",
        "v_excitatory_reversal", "v_inhibitory_reversal", "v_threshold", "v_reset", "v_rest", "refractory_steps",
        "is_inhibitory"]
    assert NeuronGroupParams.is_inhibitory.offset == 44 and NeuronGroupParams.mean_background_excitatory_spikes.offset == 48
    assert ctypes.sizeof(NeuronGroupParams) == 88
    assert ctypes.sizeof(ConnectionParams) == 20
    assert ctypes.sizeof(PlasticityParams) == 44
    # ConnectionView: 3 floats, bool, 5 uint32, 8 pointers (connection_view.h:8-31)
    from bsnn._ffi import ConnectionView
    assert ConnectionView.pre_group_is_inhibtory.offset == 12 and ConnectionView.weight_matrix_idx.offset == 16
    assert ConnectionView.weight_matrix.offset == 40 and ConnectionView.cublas_handle.offset == 96
    assert ctypes.sizeof(ConnectionView) == 104


def test_connection_propagate_rejects_bad_views_before_touching_a_device():
    import bsnn
    lib = bsnn.load_library()
    assert lib.bsnn_connection_propagate(None, None) == 1  # BSNN_ERR_INVALID_ARGUMENT
    assert b"null view" in lib.bsnn_last_error(None)
    empty = bsnn.ConnectionView()
    with pytest.raises(bsnn.InvalidArgument, match="empty connection"):
        bsnn.connection_propagate(empty)
    nulls = bsnn.ConnectionView(pre_group_num_neurons=4, post_group_num_neurons=3)
    with pytest.raises(bsnn.InvalidArgument, match="null device pointer"):
        bsnn.connection_propagate(nulls)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU failure path")
def test_create_without_gpu_fails_loudly():
    import bsnn
    with pytest.raises(bsnn.BsnnError):
        bsnn.Simulation(10, 5)


def test_missing_library_raises_import_error(tmp_path):
    import bsnn
    with pytest.raises(ImportError):
        bsnn.load_library(tmp_path / "libbsnn.so")
