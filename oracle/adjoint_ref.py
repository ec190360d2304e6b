"""FP64 restatement of the differentiation form (TEST INFRASTRUCTURE ONLY): the forward model of
bsnn_adjoint_* (the reference's step without plasticity, noise off) and its surrogate-gradient
backpropagation through time, in numpy.

Only tests/ import this module.  The forward model follows the reference's per-step arithmetic:
kernel_neuron_group_evolve.cu:85-130 (conductance-EIF Euler step, refractoriness, threshold and
reset), kernel_stimulus_apply.cu:7-21 (stimulus events act from the next step),
kernel_connection_propagate.cu:8-46 (difference-of-exponentials traces) and :79-94 (g = W^T x,
used by the next step).  `reference_gradient` differentiates the same recursion by hand; with
beta = 0 and only the voltage term it is the exact derivative of the forward pass wherever no
spike time moves, which the CPU tests confirm against central finite differences.
"""
from __future__ import annotations

import math

import numpy as np


def _group_arrays(spec):
    E, I = spec.num_excitatory, spec.num_inhibitory
    keys = ["timestep", "g_leak", "membrane_capacitance", "depolarization_slope_factor", "v_effective_spike_threshold",
            "v_excitatory_reversal", "v_inhibitory_reversal", "v_threshold", "v_reset", "v_rest", "refractory_steps"]
    out = {}
    for k in keys:
        # the parameters cross the C-ABI as float32 (bsnn_neuron_group_params)
        out[k] = np.concatenate([np.full(E, float(np.float32(spec.groups[0][k]))),
                                 np.full(I, float(np.float32(spec.groups[1][k])))])
    return out


def reference_forward(spec, steps, w_ee=None, g_leak=None, dtype=np.float64, tape=False):
    """The adjoint's forward model in `dtype` with the noise off: (E spike counts[T], vbar[T], tape).
    Follows the reference step's arithmetic statement by statement (without plasticity)."""
    E, I = spec.num_excitatory, spec.num_inhibitory
    N = E + I
    P = _group_arrays(spec)
    f = lambda x: np.asarray(x, dtype=dtype)  # noqa: E731
    dt, C, dT, vT = f(P["timestep"]), f(P["membrane_capacitance"]), f(P["depolarization_slope_factor"]), f(P["v_effective_spike_threshold"])
    Ee, Ei, vth, vreset, vrest = (f(P[k]) for k in ("v_excitatory_reversal", "v_inhibitory_reversal", "v_threshold",
                                                   "v_reset", "v_rest"))
    gL = f(P["g_leak"]) if g_leak is None else f(np.full(N, g_leak))
    norm32 = [float(np.float32(p["postsynaptic_kernel_normalization_value"])) for p in (spec.conns[0].params, spec.conns[2].params)]
    R = P["refractory_steps"].astype(np.int64)
    W = [f(c.weights) for c in spec.conns]
    if w_ee is not None:
        W[0] = f(w_ee)
    WE = np.concatenate([W[0], W[1]], axis=1)  # [E, N]
    WI = np.concatenate([W[2], W[3]], axis=1)  # [I, N]
    cp = [spec.conns[0].params, spec.conns[2].params]
    dec = lambda p, k: f(np.float32(math.exp(float(np.float32(-1.0) * np.float32(p["timestep"]) / np.float32(p[k])))))  # noqa: E731
    rdec = np.concatenate([np.full(E, dec(cp[0], "rise_time")), np.full(I, dec(cp[1], "rise_time"))])
    ddec = np.concatenate([np.full(E, dec(cp[0], "decay_time")), np.full(I, dec(cp[1], "decay_time"))])
    norm = np.concatenate([np.full(E, norm32[0]), np.full(I, norm32[1])]).astype(dtype)
    counts_in, ids, offs, deltas = spec.stimulus if spec.stimulus is not None else (np.zeros(0), [], [], [])
    ev_n = np.asarray(ids, np.int64) + np.asarray(offs, np.int64)
    ev_d = f(deltas)
    ev_off = np.concatenate([[0], np.cumsum(np.asarray(counts_in, np.int64))])
    v = vrest.copy()
    ge = np.zeros(N, dtype)
    gi = np.zeros(N, dtype)
    istim = np.zeros(N, dtype)
    ref = np.zeros(N, np.int64)
    tr = np.zeros(N, dtype)
    td = np.zeros(N, dtype)
    x = np.zeros(N, dtype)
    counts = np.zeros(steps, np.int64)
    vbar = np.zeros(steps, dtype)
    rec = {k: [] for k in ("v", "u", "ge", "gi", "s", "ref", "x")} if tape else None
    for t in range(steps):
        refr = ref > 0
        lin = -gL * (v - vrest)
        ex = gL * dT * np.exp((v - vT) / dT)
        u = v + (dt / C) * (lin + ex - ge * (v - Ee) - gi * (v - Ei) + istim)
        u = np.where(refr, v, u)
        s = (~refr) & (u >= vth)
        if tape:
            for k, val in (("v", v), ("u", u), ("ge", ge), ("gi", gi), ("s", s), ("ref", refr), ("x", x)):
                rec[k].append(val.copy())
        v_new = np.where(refr, vreset, np.where(s, vth, u))
        ref = np.where(refr, ref - 1, np.where(s, R, 0))
        v = v_new
        counts[t] = int(s[:E].sum())
        vbar[t] = v[:E].mean()
        if t < len(ev_off) - 1:
            for k in range(ev_off[t], ev_off[t + 1]):
                istim[ev_n[k]] += ev_d[k]
        td = td * ddec + norm * s
        tr = tr * rdec + norm * s
        x = td - tr
        ge = x[:E] @ WE
        gi = x[E:] @ WI
    return counts, vbar, rec


def reference_gradient(spec, steps, rate_target, voltage_target=None, *, w_ee=None, g_leak=None, rate_tau=5e-3,
                       beta=0.5e-3, rate_weight=1.0, voltage_weight=0.0, dtype=np.float64):
    """(loss, dL/dW_EE [E, E], dL/dg_leak), noise off (the spec's background means must be 0).
    `dtype` is the arithmetic of the forward model and of the adjoint recursion (the loss and its
    sensitivities stay FP64): float64 for the reference gradient, float32 to measure how much of a
    difference the recursion's rounding alone makes."""
    E, I = spec.num_excitatory, spec.num_inhibitory
    N = E + I
    P = _group_arrays(spec)
    f = lambda x: np.asarray(x, dtype=dtype)  # noqa: E731
    counts, vbar, rec = reference_forward(spec, steps, w_ee, g_leak, dtype, tape=True)
    vbar = vbar.astype(np.float64)
    dt = float(P["timestep"][0])
    a = math.exp(-dt / rate_tau)
    rho = np.zeros(steps)
    r = 0.0
    for t in range(steps):
        r = a * r + (1 - a) * counts[t] / (E * dt)
        rho[t] = r
    rt = np.asarray(rate_target, np.float64)
    vt = np.zeros(steps) if voltage_target is None else np.asarray(voltage_target, np.float64)
    loss = (rate_weight * ((rho - rt) ** 2).sum() + voltage_weight * ((vbar - vt) ** 2).sum()) / steps
    W = [f(c.weights) for c in spec.conns]
    if w_ee is not None:
        W[0] = f(w_ee)
    WE = np.concatenate([W[0], W[1]], axis=1)
    WI = np.concatenate([W[2], W[3]], axis=1)
    gL = f(P["g_leak"]) if g_leak is None else f(np.full(N, g_leak))
    C, dT, vT = f(P["membrane_capacitance"]), f(P["depolarization_slope_factor"]), f(P["v_effective_spike_threshold"])
    Ee, Ei, vth, vrest = (f(P[kk]) for kk in ("v_excitatory_reversal", "v_inhibitory_reversal", "v_threshold", "v_rest"))
    k = f(P["timestep"]) / C
    cp = [spec.conns[0].params, spec.conns[2].params]
    dec = lambda p, kk: float(np.float32(math.exp(float(np.float32(-1.0) * np.float32(p["timestep"]) / np.float32(p[kk])))))  # noqa: E731
    rdec = np.concatenate([np.full(E, dec(cp[0], "rise_time")), np.full(I, dec(cp[1], "rise_time"))])
    ddec = np.concatenate([np.full(E, dec(cp[0], "decay_time")), np.full(I, dec(cp[1], "decay_time"))])
    n32 = [float(np.float32(p["postsynaptic_kernel_normalization_value"])) for p in cp]
    norm = f(np.concatenate([np.full(E, n32[0]), np.full(I, n32[1])]))
    rdec, ddec = f(rdec), f(ddec)
    lam_v = np.zeros(N, dtype)
    lam_d = np.zeros(N, dtype)
    lam_r = np.zeros(N, dtype)
    lam_x = np.zeros(N, dtype)
    dW = np.zeros((E, E), dtype)
    dgl = 0.0
    lrho = 0.0
    for t in range(steps - 1, -1, -1):
        lrho = a * lrho + rate_weight * 2.0 / steps * (rho[t] - rt[t])
        c_s = lrho * (1 - a) / (E * dt)
        c_v = voltage_weight * 2.0 / steps * (vbar[t] - vt[t]) / E
        v, u, ge, gi = rec["v"][t], rec["u"][t], rec["ge"][t], rec["gi"][t]
        s = rec["s"][t].astype(dtype)
        refr = rec["ref"][t]
        Ld = lam_d + lam_x
        Lr = lam_r - lam_x
        dLds = norm * (Ld + Lr)
        dLds[:E] += dtype(c_s)
        Lv_next = lam_v.copy()
        Lv_next[:E] += dtype(c_v)
        psi = 1.0 / (1.0 + np.abs(u - vth) / dtype(beta)) ** 2 if beta > 0 else np.zeros(N, dtype)
        lu = Lv_next * (1 - s) + dLds * psi
        lu = np.where(refr, dtype(0.0), lu)
        ex = np.exp((v - vT) / dT)
        lam_v = lu * (1 + k * (-gL + gL * ex - ge - gi))
        lge = lu * k * (Ee - v)
        lgi = lu * k * (Ei - v)
        dgl += float((lu.astype(np.float64) * (k * (-(v - vrest) + dT * ex)).astype(np.float64)).sum())
        lam_d = ddec * Ld
        lam_r = rdec * Lr
        dW += np.outer(rec["x"][t][:E], lge[:E])
        lam_x = np.concatenate([WE @ lge, WI @ lgi])
    return float(loss), dW, dgl
