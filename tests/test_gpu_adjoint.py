"""GPU: the differentiation form (bsnn_adjoint_*), the surrogate-gradient adjoint of the network.

* Its forward pass is the engine's step without plasticity: against the FP32 oracle (Philox noise
  on) the per-step excitatory spike counts are identical and the mean excitatory voltage agrees to
  1e-5 relative over 300 steps.
* With the surrogate off and the voltage loss, the FP32 gradient with respect to W_EE and g_leak
  is checked against FP64 central finite differences of the forward model (directional
  derivatives, spike raster unchanged) and against the FP64 reference adjoint: 1e-3 relative.
* With the fast-sigmoid surrogate (beta = 0.5 mV) and the rate loss, against the reference adjoint
  (same rule) in FP32 arithmetic to 1e-3 relative (Frobenius norm) and in FP64 to 1e-2, and
  independent of where the checkpoints fall.  The surrogate gradient is sensitive to the forward
  pass's rounding: a neuron that passes within 20 uV of threshold without spiking has its u
  amplified by the exponential upswing, and psi(u - v_th) then changes by parts in 1e3 between
  FP32 and FP64 forward passes (the FP32 restatement differs from FP64 by 5.1e-3 on this network,
  the GPU by the same amount).
* The torch.autograd.Function hands the same gradients to torch.
All on an 80 E + 20 I network, 300 steps, noise off unless stated.
"""
from __future__ import annotations

import numpy as np
import pytest

import adjoint_ref
import bsnn
import oracle

pytestmark = pytest.mark.gpu

T = 300
E, I = 80, 20
VT = np.full(T, -0.062, dtype=np.float32)
RT = np.full(T, 5.0, dtype=np.float32)


def network(seed=4, noise=False):
    return bsnn.random_network(E, I, steps=T + 1, seed=seed, noise=noise, plasticity=(), stim_events=30)


def rel_err(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def check_surrogate_gradient(dW, dgl, spec, **kw):
    _, dW32, dgl32 = adjoint_ref.reference_gradient(spec, T, RT, VT, dtype=np.float32, **kw)
    _, dW64, dgl64 = adjoint_ref.reference_gradient(spec, T, RT, VT, **kw)
    print(f"dW vs FP32 restatement {rel_err(dW, dW32):.2e}, vs FP64 {rel_err(dW, dW64):.2e}; "
          f"dg_leak {abs(dgl - dgl32) / abs(dgl32):.2e} / {abs(dgl - dgl64) / abs(dgl64):.2e}")
    assert rel_err(dW, dW32) <= 1e-3, rel_err(dW, dW32)
    assert abs(dgl - dgl32) <= 1e-3 * abs(dgl32), (dgl, dgl32)
    assert rel_err(dW, dW64) <= 1e-2, rel_err(dW, dW64)
    assert abs(dgl - dgl64) <= 1e-2 * abs(dgl64), (dgl, dgl64)


def reference_rho(spec, rate_tau=5e-3):
    counts, vbar, _ = adjoint_ref.reference_forward(spec, T)
    dt = 1e-4
    a = np.exp(-dt / rate_tau)
    rho = np.zeros(T)
    r = 0.0
    for t in range(T):
        r = a * r + (1 - a) * counts[t] / (E * dt)
        rho[t] = r
    return rho, vbar


def test_forward_matches_the_oracle_with_noise():
    spec = network(seed=6, noise=True)
    net = bsnn.AdjointNetwork(spec, T, checkpoint=64, noise=True, voltage_weight=1.0)
    _, rho, vbar = net.forward(RT, VT)
    o = oracle.OracleSimulation(E, I, precision=oracle.PREC_F32, **spec.sim_kwargs())
    spec.build(o)
    a = np.exp(-1e-4 / 5e-3)
    r = 0.0
    spikes = 0
    for t in range(T):
        o.step(t)
        n = int(o.read("spikes")[:E].sum())
        spikes += n
        r = a * r + (1 - a) * n / (E * 1e-4)
        assert abs(rho[t] - r) <= 1e-5 * max(r, 1.0), (t, rho[t], r)
        v = o.read("membrane_potentials")[:E].astype(np.float64).mean()
        assert abs(vbar[t] - v) <= 1e-5 * abs(v), (t, vbar[t], v)
    assert spikes > 20
    net.close()


@pytest.mark.parametrize("seed", [4, 9])
def test_voltage_gradient_matches_fd_and_fp64(seed):
    spec = network(seed)
    net = bsnn.AdjointNetwork(spec, T, checkpoint=100, noise=False, beta=0.0, rate_weight=0.0, voltage_weight=1e4)
    loss, rho, vbar = net.forward(RT, VT)
    dW, dgl = net.backward()
    rho_ref, vbar_ref = reference_rho(spec)
    np.testing.assert_allclose(rho, rho_ref, rtol=1e-5, atol=1e-3)  # same spikes
    L64, dW64, dgl64 = adjoint_ref.reference_gradient(spec, T, RT, VT, beta=0.0, rate_weight=0.0, voltage_weight=1e4)
    assert abs(loss - L64) <= 1e-4 * L64
    assert rel_err(dW, dW64) <= 1e-3, rel_err(dW, dW64)
    assert abs(dgl - dgl64) <= 1e-3 * abs(dgl64), (dgl, dgl64)
    # FP64 central differences of the forward model
    W = spec.conns[0].weights.astype(np.float64)
    rng = np.random.default_rng(seed)
    h = 1e-6

    def loss64(w=None, gl=None):
        _, vb, rec = adjoint_ref.reference_forward(spec, T, w_ee=w, g_leak=gl, tape=True)
        return 1e4 * ((vb - VT) ** 2).sum() / T, np.array(rec["s"])

    for k in range(3):
        D = rng.standard_normal(W.shape) * W
        lp, sp = loss64(W + h * D)
        lm, sm = loss64(W - h * D)
        np.testing.assert_array_equal(sp, sm)
        fd = (lp - lm) / (2 * h)
        got = float((dW.astype(np.float64) * D).sum())
        assert abs(got - fd) <= 1e-3 * abs(fd), (k, got, fd)
    gl0 = float(np.float32(spec.groups[0]["g_leak"]))
    lp, sp = loss64(gl=gl0 * (1 + h))
    lm, sm = loss64(gl=gl0 * (1 - h))
    np.testing.assert_array_equal(sp, sm)
    fd = (lp - lm) / (2 * h * gl0)
    assert abs(dgl - fd) <= 1e-3 * abs(fd), (dgl, fd)
    net.close()


def test_surrogate_rate_gradient_matches_fp64_and_checkpoints():
    spec = network(4)
    kw = dict(noise=False, beta=0.5e-3, rate_weight=1.0, voltage_weight=1e3)
    grads = []
    for ckpt in (64, 100, T):
        net = bsnn.AdjointNetwork(spec, T, checkpoint=ckpt, **kw)
        net.forward(RT, VT)
        grads.append(net.backward())
        net.close()
    check_surrogate_gradient(*grads[0], spec, beta=0.5e-3, rate_weight=1.0, voltage_weight=1e3)
    for dW, dgl in grads[1:]:
        assert rel_err(dW, grads[0][0]) <= 1e-5
        assert abs(dgl - grads[0][1]) <= 1e-5 * abs(grads[0][1])


@pytest.mark.parametrize("ckpt", [64, T])
def test_backward_twice_gives_the_same_gradient(ckpt):
    """The forward pass leaves the last segment's tape for the backward pass; a second backward
    pass of the same forward pass (after the first replayed the other segments over that tape)
    replays it again and gives the same bits."""
    spec = network(4)
    net = bsnn.AdjointNetwork(spec, T, checkpoint=ckpt, noise=True, beta=0.5e-3, rate_weight=1.0, voltage_weight=1e3)
    net.forward(RT, VT)
    dW1, dgl1 = net.backward()
    dW2, dgl2 = net.backward()
    np.testing.assert_array_equal(dW1, dW2)
    assert dgl1 == dgl2
    net.close()


def test_set_params_and_errors():
    spec = network(4)
    net = bsnn.AdjointNetwork(spec, T, checkpoint=50, noise=False, beta=0.5e-3, voltage_weight=1e3)
    with pytest.raises(bsnn.StateError):
        net.backward()
    with pytest.raises(bsnn.InvalidArgument):
        net.forward(RT, None)
    w2 = spec.conns[0].weights * np.float32(1.3)
    net.set_params(w2, 11e-9)
    loss, _, _ = net.forward(RT, VT)
    dW, dgl = net.backward()
    kw = dict(w_ee=w2, g_leak=float(np.float32(11e-9)), beta=0.5e-3, rate_weight=1.0, voltage_weight=1e3)
    L64, _, _ = adjoint_ref.reference_gradient(spec, T, RT, VT, **kw)
    assert abs(loss - L64) <= 1e-3 * L64
    check_surrogate_gradient(dW, dgl, spec, **kw)
    net.close()


def test_autograd_function():
    torch = pytest.importorskip("torch")
    spec = network(4)
    net = bsnn.AdjointNetwork(spec, T, checkpoint=100, noise=False, beta=0.5e-3, voltage_weight=1e3)
    SpikingLoss = bsnn.spiking_loss_function()
    w = torch.tensor(spec.conns[0].weights, requires_grad=True)
    gl = torch.tensor(float(np.float32(spec.groups[0]["g_leak"])), requires_grad=True)
    loss = SpikingLoss.apply(w, gl, net, RT, VT)
    (2.0 * loss).backward()
    net.forward(RT, VT)
    dW, dgl = net.backward()
    np.testing.assert_allclose(w.grad.numpy(), 2.0 * dW, rtol=1e-6)
    assert abs(float(gl.grad) - 2.0 * dgl) <= 1e-5 * abs(dgl)
    net.close()
