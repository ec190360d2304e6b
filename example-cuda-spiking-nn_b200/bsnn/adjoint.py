"""The differentiation form: a surrogate-gradient adjoint of the network (bsnn_adjoint_* in
include/bsnn.h), its torch.autograd.Function, and an FP64 reference of the same gradient.

The model is the reference's step without plasticity.  Gradients of

    L = rate_weight / T sum_t (rho_t - rho*_t)^2 + voltage_weight / T sum_t (vbar_{t+1} - v*_t)^2

(rho: the excitatory population rate in Hz smoothed with time constant rate_tau; vbar: the mean
excitatory membrane potential) are taken with respect to the E->E weights and the g_leak shared
by both groups, by backpropagation through time with the spike's derivative replaced by the fast
sigmoid psi(u - v_th) = 1 / (1 + |u - v_th| / beta)^2 (beta = 0 turns it off) and the reset not
differentiated.  With beta = 0 and only the voltage term the result is the exact derivative of
the hard-threshold forward pass wherever no spike time moves.
"""
from __future__ import annotations

import ctypes
import numpy as np

from ._ffi import AdjointDesc, ConnectionParams, NeuronGroupParams, error_for, load_library
from .network import NetworkSpec


def _fp(a):
    return np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class AdjointNetwork:
    """A NetworkSpec (groups E then I, connections E->E, E->I, I->E, I->I; plasticity ignored) as a
    differentiable simulation of `steps` steps on one GPU."""

    def __init__(self, spec: NetworkSpec, steps: int, *, checkpoint: int = 100, noise: bool = True,
                 rate_tau: float = 5e-3, beta: float = 0.5e-3, rate_weight: float = 1.0, voltage_weight: float = 0.0,
                 device: int = 0, library=None):
        self._lib = library if library is not None else load_library()
        self.spec = spec
        self.E, self.I, self.T = spec.num_excitatory, spec.num_inhibitory, steps
        d = AdjointDesc(self.E, self.I, steps, checkpoint, int(spec.rng_seed), 1 if noise else 0, rate_tau, beta,
                        rate_weight, voltage_weight)
        ge = NeuronGroupParams.make(**spec.groups[0])
        gi = NeuronGroupParams.make(**spec.groups[1])
        ce = ConnectionParams.make(**spec.conns[0].params)
        ci = ConnectionParams.make(**spec.conns[2].params)
        self._keep = [np.ascontiguousarray(c.weights, dtype=np.float32) for c in spec.conns]
        if spec.stimulus is not None:
            counts, ids, offsets, deltas = spec.stimulus
            counts = np.ascontiguousarray(counts, dtype=np.uint32)
            neurons = np.ascontiguousarray(np.asarray(ids) + np.asarray(offsets), dtype=np.uint32)
            deltas = np.ascontiguousarray(deltas, dtype=np.float32)
        else:
            counts = np.zeros(0, np.uint32)
            neurons = np.zeros(0, np.uint32)
            deltas = np.zeros(0, np.float32)
        self._stim = (counts, neurons, deltas)
        self._h = ctypes.c_void_p()
        st = self._lib.bsnn_adjoint_create(
            ctypes.byref(d), ctypes.byref(ge), ctypes.byref(gi), ctypes.byref(ce), ctypes.byref(ci),
            *[x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) for x in self._keep],
            counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), counts.size,
            neurons.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), deltas.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
            neurons.size, device, ctypes.byref(self._h))
        self._check(st, creating=True)

    def _check(self, st, creating=False):
        if st != 0:
            msg = self._lib.bsnn_adjoint_last_error(None if creating else self._h)
            raise error_for(st, msg.decode() if msg else "")

    def set_params(self, w_ee=None, g_leak=None):
        w = None if w_ee is None else np.ascontiguousarray(w_ee, dtype=np.float32)
        self._check(self._lib.bsnn_adjoint_set_params(self._h, None if w is None else _fp(w),
                                                      float("nan") if g_leak is None else float(g_leak)))

    def forward(self, rate_target, voltage_target=None):
        """(loss, rho[T], vbar[T])."""
        rt = np.ascontiguousarray(rate_target, dtype=np.float32)
        vt = None if voltage_target is None else np.ascontiguousarray(voltage_target, dtype=np.float32)
        loss = ctypes.c_float()
        rate = np.empty(self.T, np.float32)
        vbar = np.empty(self.T, np.float32)
        self._check(self._lib.bsnn_adjoint_forward(self._h, _fp(rt), None if vt is None else _fp(vt), ctypes.byref(loss),
                                                   _fp(rate), _fp(vbar)))
        return float(loss.value), rate, vbar

    def backward(self):
        """(dL/dW_EE [E, E] float32, dL/dg_leak)."""
        g = np.empty((self.E, self.E), np.float32)
        gl = ctypes.c_double()
        self._check(self._lib.bsnn_adjoint_backward(self._h, g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                    ctypes.byref(gl)))
        return g, float(gl.value)

    def stream(self) -> int:
        p = ctypes.c_void_p()
        self._check(self._lib.bsnn_adjoint_get_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    def launches(self) -> int:
        """Kernels run so far (those of the captured graphs included)."""
        n = ctypes.c_uint64()
        self._check(self._lib.bsnn_adjoint_kernel_launches(self._h, ctypes.byref(n)))
        return int(n.value)

    def close(self):
        if self._h:
            self._lib.bsnn_adjoint_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spiking_loss_function():
    """torch.autograd.Function: loss = SpikingLoss.apply(w_ee, g_leak, net, rate_target[, voltage_target]);
    w_ee an [E, E] float32 tensor, g_leak a 0-d tensor.  The forward and backward passes run on
    the network's GPU through the C-ABI (host tensors in and out)."""
    import torch

    class SpikingLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, w_ee, g_leak, net, rate_target, voltage_target=None):
            net.set_params(w_ee.detach().cpu().numpy(), float(g_leak.detach().cpu()))
            vt = None if voltage_target is None else np.asarray(voltage_target)
            loss, _, _ = net.forward(np.asarray(rate_target), vt)
            ctx.net = net
            ctx.dev = (w_ee.device, g_leak.device)
            return torch.tensor(loss, dtype=torch.float32, device=w_ee.device)

        @staticmethod
        def backward(ctx, grad):
            gw, gl = ctx.net.backward()
            s = float(grad)
            return (torch.from_numpy(gw * s).to(ctx.dev[0]), torch.tensor(gl * s, dtype=torch.float32, device=ctx.dev[1]),
                    None, None, None)

    return SpikingLoss


def config5_network(steps: int = 2000, perturb: float = 0.1, seed: int = 11):
    """The differentiation-form workload: the reference example network (2,500 E + 625 I, the
    example's neuron, synapse and noise parameters) with plasticity off, driven by one 0.5 nA pulse
    into 250 E neurons from step 200 to step 1400 (about 3 Hz mean E rate over 2,000 steps), and
    the E->E weights of the target network: W_EE perturbed by N(0, perturb * w), clipped at 0.
    Returns (spec, w_target)."""
    from . import generation
    from .network import synthetic_network
    spec = synthetic_network("example_plastic_3125", steps=steps + 1, plastic=False, weight_values="uniform")
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.choice(spec.num_excitatory, size=250, replace=False)).tolist()
    spec.stimulus = generation.partial_group_multiple_square_waves(steps + 1, ids, [0] * len(ids), [200], [1400],
                                                                   [0.5e-9])
    w = spec.conns[0].weights
    w_target = np.maximum(w + rng.standard_normal(w.shape).astype(np.float32) * np.float32(perturb) * w, 0.0)
    return spec, w_target.astype(np.float32)
