"""bsnn_connection_propagate (kernel_connection_propagate_launch on caller-owned buffers) against the
oracle's restatement, through the C-ABI.

Tolerances: the trace arithmetic (decay, 1e-30 flush, +normalisation, x = d - r) is bit-exact; the
conductance g += W^T x is within 1e-5 relative to sum_i |w_iq x_i| + |g_q| (the oracle accumulates
in double, the kernel in float over row chunks)."""
from __future__ import annotations

import numpy as np
import pytest

import bsnn

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def make_case(n_pre, n_post, seed, spike_p=0.2, inhibitory=False):
    rng = np.random.default_rng(seed)
    host = {
        "w": rng.uniform(0.0, 2.0, (n_pre, n_post)).astype(np.float32),
        "r": rng.uniform(0.0, 1.0, n_pre).astype(np.float32),
        "d": rng.uniform(0.0, 1.5, n_pre).astype(np.float32),
        "x": np.zeros(n_pre, np.float32),
        "ge": rng.uniform(0.0, 1.0, n_post).astype(np.float32),
        "gi": rng.uniform(0.0, 1.0, n_post).astype(np.float32),
        "spikes": (rng.random(n_pre) < spike_p).astype(np.uint32),
    }
    host["r"][: min(4, n_pre)] = 1e-31  # below the flush threshold after the decay
    params = dict(r_decay=np.float32(0.9048374), d_decay=np.float32(0.9801987), norm=np.float32(1.3),
                  inhibitory=inhibitory)
    return host, params


class DeviceCase:
    """Device copies of a case plus the ConnectionView describing them."""

    def __init__(self, host, params):
        torch = _torch()
        self.t = {k: torch.from_numpy(v.view(np.int32) if v.dtype == np.uint32 else v).cuda()
                  for k, v in host.items()}
        n_pre, n_post = host["w"].shape
        t = self.t
        self.view = bsnn.ConnectionView(
            postsynaptic_r_trace_decay=params["r_decay"], postsynaptic_d_trace_decay=params["d_decay"],
            postsynaptic_kernel_normalization_value=params["norm"], pre_group_is_inhibtory=params["inhibitory"],
            pre_group_num_neurons=n_pre, post_group_num_neurons=n_post, weight_matrix=t["w"].data_ptr(),
            postsynaptic_r_traces=t["r"].data_ptr(), postsynaptic_d_traces=t["d"].data_ptr(),
            summed_postsynaptic_conductances=t["x"].data_ptr(), post_group_g_excitatory=t["ge"].data_ptr(),
            post_group_g_inhibitory=t["gi"].data_ptr(), spikes=t["spikes"].data_ptr())

    def host(self, k):
        return self.t[k].cpu().numpy()


def oracle_step(host, params, oracle_mod):
    """Advances the host copy by one oracle call; returns sum_i |w_iq x_i| per column."""
    g = host["gi"] if params["inhibitory"] else host["ge"]
    oracle_mod.connection_propagate(params["r_decay"], params["d_decay"], params["norm"], host["w"], host["r"],
                                    host["d"], host["x"], g, host["spikes"])
    return np.abs(host["w"].astype(np.float64)).T @ np.abs(host["x"].astype(np.float64))


def check(dev, host, params, scale, tag):
    for k in ("r", "d", "x"):
        assert np.array_equal(dev.host(k), host[k]), f"{tag}: {k} not bit-exact"
    tgt, other = ("gi", "ge") if params["inhibitory"] else ("ge", "gi")
    assert np.array_equal(dev.host(other), host[other]), f"{tag}: {other} must not change"
    got, want = dev.host(tgt).astype(np.float64), host[tgt].astype(np.float64)
    bound = RTOL * (scale + np.abs(want)) + 1e-30
    bad = np.flatnonzero(np.abs(got - want) > bound)
    assert bad.size == 0, f"{tag}: {tgt} differs at {bad[:5]}: got {got[bad[:5]]}, want {want[bad[:5]]}"


@pytest.mark.parametrize("n_pre,n_post,inhibitory,spike_p", [
    (1, 1, False, 1.0),
    (300, 257, False, 0.2),     # ragged column count
    (625, 2500, True, 0.1),     # I -> E of the example network
    (2500, 2500, False, 0.05),  # E -> E of the example network
    (10125, 301, False, 0.0),   # long columns, no spikes
    (64, 9000, True, 1.0),      # wide rows, every presynaptic neuron spikes
])
def test_propagate_matches_oracle(oracle_mod, n_pre, n_post, inhibitory, spike_p):
    torch = _torch()
    host, params = make_case(n_pre, n_post, seed=n_pre * 7 + n_post, spike_p=spike_p, inhibitory=inhibitory)
    dev = DeviceCase(host, params)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # the second call starts from the first call's traces and conductances
        scale = oracle_step(host, params, oracle_mod)
        bsnn.connection_propagate(dev.view, stream)
        torch.cuda.synchronize()
        check(dev, host, params, scale, f"call {call}")


def test_propagate_on_default_stream_and_side_stream(oracle_mod):
    torch = _torch()
    host, params = make_case(700, 333, seed=5)
    dev = DeviceCase(host, params)
    scale = oracle_step(host, params, oracle_mod)
    bsnn.connection_propagate(dev.view, 0)  # legacy default stream
    torch.cuda.synchronize()
    check(dev, host, params, scale, "default stream")
    side = torch.cuda.Stream()
    scale = oracle_step(host, params, oracle_mod)
    bsnn.connection_propagate(dev.view, side.cuda_stream)
    side.synchronize()
    check(dev, host, params, scale, "side stream")


def test_propagate_is_deterministic():
    torch = _torch()
    host, params = make_case(2500, 2500, seed=3)
    outs = []
    for _ in range(2):
        dev = DeviceCase(host, params)
        bsnn.connection_propagate(dev.view, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        outs.append(dev.host("ge"))
    assert np.array_equal(outs[0], outs[1])
