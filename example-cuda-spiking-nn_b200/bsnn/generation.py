"""Host-side network generation (one-shot set-up, outside the per-step hot path).

Restates the reference's generators so networks of the reference's shape can be built without
its binary:
  grid locations            cpp_src/generation/generate_location.cpp:5-47
  distance-dependent weights cpp_src/generation/generate_weights.cpp:10-107 with
                            cpp_src/utils/math_functions.cpp:8-16 (periodic-boundary distance)
  square-wave stimulus       cpp_src/generation/generate_stimulus_schedules.cpp:20-228

The weight generator follows the reference's draw order with MT19937 seeded by rng_seed and
uniform floats formed as libstdc++'s uniform_real_distribution<float> forms them from one 32-bit
draw.  Its float arithmetic is numpy's, so a probability that lands within an ulp of a draw can
resolve differently than in the C++ build; parity runs therefore feed the same matrices to every
implementation instead of regenerating them.
"""
from __future__ import annotations

import numpy as np


def generate_2d_grid_locations(num_neurons: int, spacing: float, rows: int, cols: int) -> np.ndarray:
    """[num_neurons, 2] float32 (x, y); neuron id -> (col, row) * spacing, row-major."""
    if num_neurons == 0:
        return np.zeros((0, 2), np.float32)
    if rows == 0 or cols == 0:
        raise ValueError("rows and cols must be > 0")
    if rows < (num_neurons + cols - 1) // cols:
        raise ValueError("grid too small: need at least num_neurons cells")
    ids = np.arange(num_neurons)
    x = (ids % cols).astype(np.float32) * np.float32(spacing)
    y = (ids // cols).astype(np.float32) * np.float32(spacing)
    return np.stack([x, y], axis=1).astype(np.float32)


def pbc_distance(pre: np.ndarray, post: np.ndarray, lx: float, ly: float) -> np.ndarray:
    """[n_pre, n_post] float32 Euclidean distance on a periodic lattice (math_functions.cpp:8-16)."""
    f32 = np.float32
    dx = np.abs(pre[:, None, 0] - post[None, :, 0]).astype(f32)
    dy = np.abs(pre[:, None, 1] - post[None, :, 1]).astype(f32)
    dx = np.minimum(dx, f32(lx) - dx)
    dy = np.minimum(dy, f32(ly) - dy)
    return np.sqrt(dx * dx + dy * dy).astype(f32)


def _canonical_floats(raw: np.ndarray) -> np.ndarray:
    """uniform_real_distribution<float>(0, 1) from one 32-bit MT19937 output each (libstdc++
    generate_canonical<float, 24>): float(x) / 2^32, pulled below 1."""
    u = raw.astype(np.float32) / np.float32(4294967296.0)
    u[u >= np.float32(1.0)] = np.nextafter(np.float32(1.0), np.float32(0.0))
    return u


def distance_2d_weights(pre_loc: np.ndarray, post_loc: np.ndarray, *, max_weight_value: float, max_distance: float,
                        spread_scale: float, weight_value_normal_dropoff: bool, probabilistic_normal_not_uniform: bool,
                        probability_multiplier: float, no_diagonal_connections: bool, x_location_length: float,
                        y_location_length: float, rng_seed: int, value_mode: str = "reference") -> np.ndarray:
    """Row-major [pre, post] float32 weights.

    value_mode "reference": every accepted synapse gets max_weight_value (times the normal dropoff
    when enabled), as generate_weights.cpp:80-86 does.  "uniform": accepted synapses get
    U[0, max_weight_value) drawn from a separate numpy generator (used for synthetic benchmark
    inputs that ask for uniform weights); acceptance is unchanged.
    """
    f32 = np.float32
    n_pre, n_post = len(pre_loc), len(post_loc)
    if n_pre == 0 or n_post == 0:
        raise ValueError("Neuron groups must not be empty.")
    d = pbc_distance(pre_loc, post_loc, x_location_length, y_location_length)
    cand = np.abs(d) <= f32(max_distance)
    if no_diagonal_connections:
        k = min(n_pre, n_post)
        cand[np.arange(k), np.arange(k)] = False
    # One MT19937 draw per candidate pair, in row-major (pre, post) order.
    n_draw = int(cand.sum())
    rs = np.random.RandomState(rng_seed & 0xFFFFFFFF)
    raw = rs.randint(0, 2**32, size=n_draw, dtype=np.uint64).astype(np.uint32) if n_draw else np.zeros(0, np.uint32)
    u = np.full(d.shape, f32(2.0), dtype=f32)
    u[cand] = _canonical_floats(raw)
    prob = np.full(d.shape, f32(probability_multiplier), dtype=f32)
    if probabilistic_normal_not_uniform:
        prob = prob * np.exp(f32(-1.0) * (d * d) / f32(spread_scale)).astype(f32)
    accept = cand & (u < prob)
    if value_mode == "reference":
        val = np.full(d.shape, f32(max_weight_value), dtype=f32)
    elif value_mode == "uniform":
        g = np.random.default_rng(rng_seed + 7919)
        val = (g.random(d.shape, dtype=np.float32) * f32(max_weight_value)).astype(f32)
    else:
        raise ValueError(f"unknown value_mode {value_mode!r}")
    if weight_value_normal_dropoff:
        val = val * np.exp(f32(-1.0) * (d * d) / f32(spread_scale)).astype(f32)
    w = np.where(accept, val, f32(0.0)).astype(f32)
    if (w < 0).any():
        raise RuntimeError("generate_weights::distance_2d_weights_file: negative weight value calculated")
    return w


def partial_group_multiple_square_waves(max_timestep: int, selected_input_ids, selected_input_post_group_offsets,
                                        start_clock_steps, end_clock_steps, stimulus_input_values):
    """(timestep_event_counts[T], neuron_ids, post_group_offsets, amplitude_changes): +amp at each
    start, -amp at end+1, events sorted by (t, offset, id) (generate_stimulus_schedules.cpp:20-228)."""
    ids = list(selected_input_ids)
    offs = list(selected_input_post_group_offsets)
    starts, ends = list(start_clock_steps), list(end_clock_steps)
    vals = list(stimulus_input_values)
    empty = (np.zeros(max_timestep, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.float32))
    if len(ids) != len(offs) or len(starts) != len(ends):
        return empty
    if len(vals) != len(starts):
        if len(vals) == 1:
            vals = vals * len(starts)
        else:
            return empty
    if any(s > e for s, e in zip(starts, ends)) or max_timestep == 0:
        return empty
    seen, selected = set(), []
    for nid, off in zip(ids, offs):
        if (off, nid) not in seen:
            seen.add((off, nid))
            selected.append((off, nid))
    events = []
    for off, nid in selected:
        for s, e, a in zip(starts, ends, vals):
            if s < max_timestep:
                events.append((s, off, nid, np.float32(a)))
            if e + 1 < max_timestep:
                events.append((e + 1, off, nid, np.float32(-a)))
    events.sort(key=lambda ev: (ev[0], ev[1], ev[2]))
    for a, b in zip(events, events[1:]):
        if a[:3] == b[:3]:
            raise RuntimeError(f"duplicate events detected for time step {a[0]}, post_group_offset {a[1]}, neuron_id {a[2]}")
    counts = np.zeros(max_timestep, np.uint32)
    for ev in events:
        counts[ev[0]] += 1
    return (counts, np.array([e[2] for e in events], np.uint32), np.array([e[1] for e in events], np.uint32),
            np.array([e[3] for e in events], np.float32))


def distance_2d_weights_gpu(pre_loc: np.ndarray, post_loc: np.ndarray, *, max_weight_value: float, max_distance: float,
                            spread_scale: float, weight_value_normal_dropoff: bool,
                            probabilistic_normal_not_uniform: bool, probability_multiplier: float,
                            no_diagonal_connections: bool, x_location_length: float, y_location_length: float,
                            rng_seed: int, value_mode: str = "reference", device: int = 0, library=None) -> np.ndarray:
    """The same rule as distance_2d_weights, generated on the GPU with counter-based draws per
    (seed, pre, post) (bsnn_generate_distance_weights): identical candidate sets, equal in
    distribution, not bit for bit."""
    import ctypes

    from ._ffi import WeightGenerationParams, error_for, load_library
    lib = library if library is not None else load_library()
    pre = np.ascontiguousarray(pre_loc, dtype=np.float32).reshape(-1, 2)
    post = np.ascontiguousarray(post_loc, dtype=np.float32).reshape(-1, 2)
    if value_mode not in ("reference", "uniform"):
        raise ValueError(f"unknown value_mode {value_mode!r}")
    p = WeightGenerationParams(max_weight_value, max_distance, spread_scale, probability_multiplier,
                               x_location_length, y_location_length, int(weight_value_normal_dropoff),
                               int(probabilistic_normal_not_uniform), int(no_diagonal_connections),
                               int(value_mode == "uniform"))
    w = np.empty((len(pre), len(post)), dtype=np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    st = lib.bsnn_generate_distance_weights(pre.ctypes.data_as(fp), len(pre), post.ctypes.data_as(fp), len(post),
                                            ctypes.byref(p), int(rng_seed) & 0xFFFFFFFFFFFFFFFF, device,
                                            w.ctypes.data_as(fp))
    if st != 0:
        raise error_for(st, lib.bsnn_last_error(None).decode())
    return w
