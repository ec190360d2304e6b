"""CPU: the FP64 restatement of the differentiation form (oracle/adjoint_ref.py), the checker of the
CUDA adjoint.

Its forward model is pinned to the FP64 oracle (same spike raster, voltages to 1e-9 V over 300
steps, plasticity and noise off), and its hand-derived gradient to central finite differences of
that forward model: with the surrogate off (beta = 0) and the voltage loss, the loss is smooth in
W_EE and g_leak wherever no spike time moves, and the backpropagated gradient is its exact
derivative (agreement to 1e-6 relative at h = 1e-6, with the spike raster checked unchanged).
"""
from __future__ import annotations

import numpy as np
import pytest

import adjoint_ref
import bsnn
import oracle

T = 300
E, I = 80, 20


def network(seed=4):
    return bsnn.random_network(E, I, steps=T + 1, seed=seed, noise=False, plasticity=(), stim_events=30)


def voltage_loss(spec, w=None, gl=None, vt=-0.062, weight=1e4):
    _, vbar, rec = adjoint_ref.reference_forward(spec, T, w_ee=w, g_leak=gl, tape=True)
    return weight * ((vbar - vt) ** 2).sum() / T, np.array(rec["s"])


def test_forward_matches_the_fp64_oracle(oracle_mod):
    spec = network()
    _, _, rec = adjoint_ref.reference_forward(spec, T, tape=True)
    o = oracle.OracleSimulation(E, I, precision=oracle.PREC_F64, **spec.sim_kwargs())
    spec.build(o)
    o.set_noise_mode(bsnn.NOISE_OFF)
    n_spikes = 0
    for t in range(T):
        o.step(t)
        s = o.read("spikes").astype(bool)
        np.testing.assert_array_equal(s, rec["s"][t], err_msg=f"step {t}")
        n_spikes += int(s.sum())
        if t + 1 < T:
            np.testing.assert_allclose(o.read_f64("membrane_potentials"), rec["v"][t + 1], rtol=0, atol=1e-9)
    assert n_spikes > 40


@pytest.mark.parametrize("seed", [4, 9])
def test_gradient_matches_central_differences(seed):
    spec = network(seed)
    vt = np.full(T, -0.062)
    _, dW, dgl = adjoint_ref.reference_gradient(spec, T, np.zeros(T), vt, beta=0.0, rate_weight=0.0, voltage_weight=1e4)
    W = spec.conns[0].weights.astype(np.float64)
    rng = np.random.default_rng(seed)
    h = 1e-6
    for k in range(3):
        D = rng.standard_normal(W.shape) * W
        lp, sp = voltage_loss(spec, W + h * D)
        lm, sm = voltage_loss(spec, W - h * D)
        np.testing.assert_array_equal(sp, sm)
        fd = (lp - lm) / (2 * h)
        adj = float((dW * D).sum())
        assert abs(fd - adj) <= 1e-6 * abs(adj) + 1e-12, (k, fd, adj)
    gl0 = float(np.float32(spec.groups[0]["g_leak"]))  # the value the forward model uses
    lp, sp = voltage_loss(spec, gl=gl0 * (1 + h))
    lm, sm = voltage_loss(spec, gl=gl0 * (1 - h))
    np.testing.assert_array_equal(sp, sm)
    fd = (lp - lm) / (2 * h * gl0)
    assert abs(fd - dgl) <= 1e-6 * abs(dgl), (fd, dgl)


def test_surrogate_adds_the_spike_paths():
    """With the surrogate on, the rate loss has a gradient (the hard threshold alone gives none), and
    beta -> 0 recovers the surrogate-free gradient."""
    spec = network()
    rt = np.full(T, 5.0)
    _, dW0, _ = adjoint_ref.reference_gradient(spec, T, rt, beta=0.0)
    assert not dW0.any()
    _, dW, dgl = adjoint_ref.reference_gradient(spec, T, rt, beta=0.5e-3)
    assert np.isfinite(dW).all() and np.abs(dW).max() > 0 and np.isfinite(dgl)
    vt = np.full(T, -0.062)
    _, a, _ = adjoint_ref.reference_gradient(spec, T, rt, vt, beta=0.0, rate_weight=0.0, voltage_weight=1e4)
    _, b, _ = adjoint_ref.reference_gradient(spec, T, rt, vt, beta=1e-12, rate_weight=0.0, voltage_weight=1e4)
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-9 * np.abs(a).max())
