"""bsnn_connection_propagate_noalloc (fixed static scratch, no device allocation) against
bsnn_connection_propagate, both through the C-ABI, on two calls in a row.

Tolerance: traces bit-exact; conductances within 1e-5 relative to sum_i |w_iq x_i| + |g_q|."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import bsnn

RTOL = 1e-5
STATIC_SCRATCH_FLOATS = 1 << 20


def _lib():
    lib = bsnn.load_library()
    lib.bsnn_connection_propagate_noalloc.restype = ctypes.c_int32
    lib.bsnn_connection_propagate_noalloc.argtypes = [ctypes.POINTER(bsnn.ConnectionView), ctypes.c_void_p]
    return lib


def _case(n_pre, n_post, seed, inhibitory):
    rng = np.random.default_rng(seed)
    host = {
        "w": rng.uniform(0.0, 2.0, (n_pre, n_post)).astype(np.float32),
        "r": rng.uniform(0.0, 1.0, n_pre).astype(np.float32),
        "d": rng.uniform(0.0, 1.5, n_pre).astype(np.float32),
        "x": np.zeros(n_pre, np.float32),
        "ge": rng.uniform(0.0, 1.0, n_post).astype(np.float32),
        "gi": rng.uniform(0.0, 1.0, n_post).astype(np.float32),
        "spikes": (rng.random(n_pre) < 0.2).astype(np.int32),
    }
    return host, inhibitory


def _device(host, inhibitory):
    import torch
    t = {k: torch.from_numpy(v.copy()).cuda() for k, v in host.items()}
    n_pre, n_post = host["w"].shape
    view = bsnn.ConnectionView(
        postsynaptic_r_trace_decay=0.9048374, postsynaptic_d_trace_decay=0.9801987,
        postsynaptic_kernel_normalization_value=1.3, pre_group_is_inhibtory=inhibitory,
        pre_group_num_neurons=n_pre, post_group_num_neurons=n_post, weight_matrix=t["w"].data_ptr(),
        postsynaptic_r_traces=t["r"].data_ptr(), postsynaptic_d_traces=t["d"].data_ptr(),
        summed_postsynaptic_conductances=t["x"].data_ptr(), post_group_g_excitatory=t["ge"].data_ptr(),
        post_group_g_inhibitory=t["gi"].data_ptr(), spikes=t["spikes"].data_ptr())
    return t, view


@pytest.mark.gpu
@pytest.mark.parametrize("n_pre,n_post,inhibitory", [(1, 1, False), (300, 257, True), (2500, 2500, False),
                                                     (625, 2500, True), (10125, 301, False)])
def test_noalloc_matches_allocating_entry_point(n_pre, n_post, inhibitory):
    import torch
    lib = _lib()
    host, inh = _case(n_pre, n_post, seed=n_pre + 3 * n_post, inhibitory=inhibitory)
    ta, va = _device(host, inh)  # driven by bsnn_connection_propagate
    tb, vb = _device(host, inh)  # driven by bsnn_connection_propagate_noalloc
    stream = torch.cuda.current_stream().cuda_stream
    tgt = "gi" if inhibitory else "ge"
    for call in range(2):
        assert lib.bsnn_connection_propagate(ctypes.byref(va), ctypes.c_void_p(stream)) == 0, \
            lib.bsnn_last_error(None)
        assert lib.bsnn_connection_propagate_noalloc(ctypes.byref(vb), ctypes.c_void_p(stream)) == 0, \
            lib.bsnn_last_error(None)
        torch.cuda.synchronize()
        for k in ("r", "d", "x", "ge", "gi"):
            a, b = ta[k].cpu().numpy(), tb[k].cpu().numpy()
            if k != tgt:
                assert np.array_equal(a, b), f"call {call}: {k} differs"
                continue
            x = ta["x"].cpu().numpy().astype(np.float64)
            scale = np.abs(host["w"].astype(np.float64)).T @ np.abs(x) + np.abs(a.astype(np.float64))
            err = np.abs(a.astype(np.float64) - b.astype(np.float64))
            bad = np.flatnonzero(err > RTOL * scale + 1e-30)
            assert bad.size == 0, f"call {call}: {k} differs at {bad[:5]}: {a[bad[:5]]} vs {b[bad[:5]]}"


@pytest.mark.gpu
def test_noalloc_rejects_post_groups_beyond_the_static_scratch():
    import torch
    lib = _lib()
    n_post = STATIC_SCRATCH_FLOATS + 1
    # real buffers of the stated sizes (one presynaptic row), so nothing could read out of bounds
    t = {"w": torch.zeros(n_post, device="cuda"), "r": torch.zeros(1, device="cuda"),
         "d": torch.zeros(1, device="cuda"), "x": torch.zeros(1, device="cuda"),
         "ge": torch.zeros(n_post, device="cuda"), "gi": torch.zeros(n_post, device="cuda"),
         "spikes": torch.zeros(1, dtype=torch.int32, device="cuda")}
    view = bsnn.ConnectionView(pre_group_num_neurons=1, post_group_num_neurons=n_post,
                               weight_matrix=t["w"].data_ptr(), postsynaptic_r_traces=t["r"].data_ptr(),
                               postsynaptic_d_traces=t["d"].data_ptr(),
                               summed_postsynaptic_conductances=t["x"].data_ptr(),
                               post_group_g_excitatory=t["ge"].data_ptr(), post_group_g_inhibitory=t["gi"].data_ptr(),
                               spikes=t["spikes"].data_ptr())
    assert lib.bsnn_connection_propagate_noalloc(ctypes.byref(view), None) == 2  # BSNN_ERR_OUT_OF_RANGE
    assert b"static propagate scratch limit" in lib.bsnn_last_error(None)
