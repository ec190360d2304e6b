"""bsnn_connection_propagate_noalloc (fixed static scratch, no device allocation) against
bsnn_connection_propagate and against the oracle, all through the C-ABI, on two calls in a row.

Some callers cannot allocate device memory in the middle of a run: a step loop inside an
application whose device memory is held by its own caching allocator, where a per-call
cudaMallocAsync may fail or grow a pool.  The no-alloc entry point serves them with one fixed
4 MiB array per device.  These tests check that it gives the allocating entry point's result,
that it takes no device memory per call, and that it rejects connections too wide for the array.

Tolerances: traces bit-exact.  Conductances: bit-identical to the allocating path whenever both
split the rows into the same number of chunks (every size up to the limit on a 148-SM B200);
otherwise within 1e-5 relative to sum_i |w_iq x_i| + |g_q|, the bound the oracle comparison uses.

This file is collected last (test_zz_*) so that a run stopping at its first failure has run every
other test before it."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import bsnn

RTOL = 1e-5
STATIC_SCRATCH_FLOATS = 1 << 20
THREADS = 256  # columns per block of the split GEMV (csrc/propagate.cuh kThreads)


def _lib():
    lib = bsnn.load_library()
    lib.bsnn_connection_propagate_noalloc.restype = ctypes.c_int32
    lib.bsnn_connection_propagate_noalloc.argtypes = [ctypes.POINTER(bsnn.ConnectionView), ctypes.c_void_p]
    return lib


def _splits(n_pre, n_post, sms):
    """Row chunks of the allocating path (choose_splits) and of the no-alloc path (static_splits)."""
    col_blocks = (n_post + THREADS - 1) // THREADS
    s = min(max((4 * sms + col_blocks - 1) // col_blocks, 1), n_pre)
    return s, min(s, STATIC_SCRATCH_FLOATS // n_post)


def _case(n_pre, n_post, seed, inhibitory):
    rng = np.random.default_rng(seed)
    host = {
        "w": rng.uniform(0.0, 2.0, (n_pre, n_post)).astype(np.float32),
        "r": rng.uniform(0.0, 1.0, n_pre).astype(np.float32),
        "d": rng.uniform(0.0, 1.5, n_pre).astype(np.float32),
        "x": np.zeros(n_pre, np.float32),
        "ge": rng.uniform(0.0, 1.0, n_post).astype(np.float32),
        "gi": rng.uniform(0.0, 1.0, n_post).astype(np.float32),
        "spikes": (rng.random(n_pre) < 0.2).astype(np.uint32),
    }
    params = dict(r_decay=np.float32(0.9048374), d_decay=np.float32(0.9801987), norm=np.float32(1.3),
                  inhibitory=inhibitory)
    return host, params


def _device(host, params):
    import torch
    t = {k: torch.from_numpy((v.view(np.int32) if v.dtype == np.uint32 else v).copy()).cuda() for k, v in host.items()}
    n_pre, n_post = host["w"].shape
    view = bsnn.ConnectionView(
        postsynaptic_r_trace_decay=params["r_decay"], postsynaptic_d_trace_decay=params["d_decay"],
        postsynaptic_kernel_normalization_value=params["norm"], pre_group_is_inhibtory=params["inhibitory"],
        pre_group_num_neurons=n_pre, post_group_num_neurons=n_post, weight_matrix=t["w"].data_ptr(),
        postsynaptic_r_traces=t["r"].data_ptr(), postsynaptic_d_traces=t["d"].data_ptr(),
        summed_postsynaptic_conductances=t["x"].data_ptr(), post_group_g_excitatory=t["ge"].data_ptr(),
        post_group_g_inhibitory=t["gi"].data_ptr(), spikes=t["spikes"].data_ptr())
    return t, view


def _call_noalloc(lib, view, stream):
    st = lib.bsnn_connection_propagate_noalloc(ctypes.byref(view), ctypes.c_void_p(stream))
    assert st == 0, lib.bsnn_last_error(None)


@pytest.mark.gpu
@pytest.mark.parametrize("n_pre,n_post,inhibitory", [(1, 1, False), (300, 257, True), (2500, 2500, False),
                                                     (625, 2500, True), (10125, 301, False), (40, 151552, False),
                                                     (8, 600000, True)])
def test_noalloc_matches_allocating_entry_point(n_pre, n_post, inhibitory):
    import torch
    lib = _lib()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    same_chunks = _splits(n_pre, n_post, sms)[0] == _splits(n_pre, n_post, sms)[1]
    host, params = _case(n_pre, n_post, seed=n_pre + 3 * n_post, inhibitory=inhibitory)
    ta, va = _device(host, params)  # driven by bsnn_connection_propagate
    tb, vb = _device(host, params)  # driven by bsnn_connection_propagate_noalloc
    stream = torch.cuda.current_stream().cuda_stream
    tgt = "gi" if inhibitory else "ge"
    for call in range(2):
        assert lib.bsnn_connection_propagate(ctypes.byref(va), ctypes.c_void_p(stream)) == 0, \
            lib.bsnn_last_error(None)
        _call_noalloc(lib, vb, stream)
        torch.cuda.synchronize()
        for k in ("r", "d", "x", "ge", "gi"):
            a, b = ta[k].cpu().numpy(), tb[k].cpu().numpy()
            if k != tgt or same_chunks:
                assert np.array_equal(a, b), f"call {call}: {k} differs (same chunk count: {same_chunks})"
                continue
            x = ta["x"].cpu().numpy().astype(np.float64)
            scale = np.abs(host["w"].astype(np.float64)).T @ np.abs(x) + np.abs(a.astype(np.float64))
            err = np.abs(a.astype(np.float64) - b.astype(np.float64))
            bad = np.flatnonzero(err > RTOL * scale + 1e-30)
            assert bad.size == 0, f"call {call}: {k} differs at {bad[:5]}: {a[bad[:5]]} vs {b[bad[:5]]}"


@pytest.mark.gpu
@pytest.mark.parametrize("n_pre,n_post,inhibitory", [(625, 2500, True), (2500, 2500, False)])
def test_noalloc_matches_oracle(oracle_mod, n_pre, n_post, inhibitory):
    """Two calls in a row against the oracle's restatement of kernel_connection_propagate_launch
    (cpp_src/connections/kernel_connection_propagate.cu:64-111)."""
    import torch
    lib = _lib()
    host, params = _case(n_pre, n_post, seed=11 * n_pre + n_post, inhibitory=inhibitory)
    t, view = _device(host, params)
    stream = torch.cuda.current_stream().cuda_stream
    tgt, other = ("gi", "ge") if inhibitory else ("ge", "gi")
    for call in range(2):
        g = host[tgt]
        oracle_mod.connection_propagate(params["r_decay"], params["d_decay"], params["norm"], host["w"], host["r"],
                                        host["d"], host["x"], g, host["spikes"])
        scale = np.abs(host["w"].astype(np.float64)).T @ np.abs(host["x"].astype(np.float64))
        _call_noalloc(lib, view, stream)
        torch.cuda.synchronize()
        for k in ("r", "d", "x", other):
            assert np.array_equal(t[k].cpu().numpy(), host[k]), f"call {call}: {k} not bit-exact"
        got, want = t[tgt].cpu().numpy().astype(np.float64), host[tgt].astype(np.float64)
        bad = np.flatnonzero(np.abs(got - want) > RTOL * (scale + np.abs(want)) + 1e-30)
        assert bad.size == 0, f"call {call}: {tgt} differs at {bad[:5]}: got {got[bad[:5]]}, want {want[bad[:5]]}"


@pytest.mark.gpu
def test_noalloc_takes_no_device_memory_per_call():
    """After a first call (the per-device set-up), further calls leave the device's free memory
    and torch's allocator untouched."""
    import torch
    lib = _lib()
    host, params = _case(2500, 2500, seed=7, inhibitory=False)
    t, view = _device(host, params)
    stream = torch.cuda.current_stream().cuda_stream
    _call_noalloc(lib, view, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(3):
        _call_noalloc(lib, view, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0, f"free device memory fell by {free0 - free1} bytes over three calls"
    assert torch.cuda.memory_reserved() == reserved0


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
