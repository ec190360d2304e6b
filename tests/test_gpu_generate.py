"""GPU: distance-dependent weight generation on the GPU (bsnn_generate_distance_weights), the
flagged alternative to the reference's sequential mt19937 generator.

* The candidate sets are the reference's exactly: with every candidate accepted (multiplier 1,
  flat probability) the GPU matrix equals the host generator's bit for bit.
* With the example's settings, the number of synapses, overall and per distance bin, is within
  5 binomial standard deviations of the expectation, as is the host generator's.
* Values: constant max_weight (times the Gaussian with the normal drop-off), or U[0, max_weight)
  with the uniform mode; the same seed gives the same matrix, another seed another.
"""
from __future__ import annotations

import time

import numpy as np
import pytest

from bsnn import generation

pytestmark = pytest.mark.gpu


def grid(n_side, spacing=1.0):
    return generation.generate_2d_grid_locations(n_side * n_side, spacing, n_side, n_side)


def kw(**over):
    k = dict(max_weight_value=1.5e-9, max_distance=45.0, spread_scale=81.0, weight_value_normal_dropoff=False,
             probabilistic_normal_not_uniform=True, probability_multiplier=0.2, no_diagonal_connections=True,
             x_location_length=50.0, y_location_length=50.0, rng_seed=751)
    k.update(over)
    return k


def test_candidate_sets_are_the_references():
    e = grid(30)
    i = generation.generate_2d_grid_locations(15 * 15, 2.0, 15, 15)
    for pre, post, diag in ((e, e, True), (e, i, False), (i, e, False)):
        k = kw(probability_multiplier=1.0, probabilistic_normal_not_uniform=False, max_distance=9.5,
               no_diagonal_connections=diag, x_location_length=30.0, y_location_length=30.0)
        gpu = generation.distance_2d_weights_gpu(pre, post, **k)
        host = generation.distance_2d_weights(pre, post, **k)
        np.testing.assert_array_equal(gpu, host)
        assert 0 < (gpu > 0).mean() < 1


def expected_counts(pre, post, k, bins):
    d = generation.pbc_distance(pre, post, k["x_location_length"], k["y_location_length"]).astype(np.float64)
    cand = d <= k["max_distance"]
    if k["no_diagonal_connections"]:
        np.fill_diagonal(cand, False)
    p = k["probability_multiplier"] * np.exp(-(d * d) / k["spread_scale"])
    p = np.where(cand, p, 0.0)
    idx = np.digitize(d, bins)
    mean = np.bincount(idx.ravel(), weights=p.ravel(), minlength=len(bins) + 1)
    var = np.bincount(idx.ravel(), weights=(p * (1 - p)).ravel(), minlength=len(bins) + 1)
    return idx, mean, var


def test_synapse_counts_match_the_rule():
    e = grid(50)
    k = kw()
    bins = np.array([0.5, 2.5, 5, 10, 20, 45.5])
    idx, mean, var = expected_counts(e, e, k, bins)
    for name, w in (("gpu", generation.distance_2d_weights_gpu(e, e, **k)),
                    ("host", generation.distance_2d_weights(e, e, **k))):
        got = np.bincount(idx.ravel(), weights=(w > 0).ravel().astype(np.float64), minlength=len(bins) + 1)
        z = (got - mean) / np.sqrt(np.maximum(var, 1e-12))
        print(name, "synapses", int(got.sum()), "expected", round(mean.sum()), "z per bin", np.round(z, 2))
        assert np.all(np.abs(z[var > 0]) < 5), (name, z)
        assert abs(got.sum() - mean.sum()) < 5 * np.sqrt(var.sum())


def test_values_and_seeds():
    e = grid(40)
    k = kw(x_location_length=40.0, y_location_length=40.0)
    a = generation.distance_2d_weights_gpu(e, e, **k)
    np.testing.assert_array_equal(a, generation.distance_2d_weights_gpu(e, e, **k))
    b = generation.distance_2d_weights_gpu(e, e, **dict(k, rng_seed=752))
    assert not np.array_equal(a, b)
    assert set(np.unique(a)) == {np.float32(0.0), np.float32(1.5e-9)}
    u = generation.distance_2d_weights_gpu(e, e, **k, value_mode="uniform")
    np.testing.assert_array_equal(u > 0, a > 0)  # the same acceptance draw
    vals = u[u > 0] / np.float32(1.5e-9)
    assert vals.max() < 1.0 and abs(vals.mean() - 0.5) < 5 * np.sqrt(1 / 12 / vals.size)
    g = generation.distance_2d_weights_gpu(e, e, **dict(k, weight_value_normal_dropoff=True))
    d = generation.pbc_distance(e, e, 40.0, 40.0)
    want = np.float32(1.5e-9) * np.exp(np.float32(-1.0) * (d * d) / np.float32(81.0)).astype(np.float32)
    np.testing.assert_allclose(g[g > 0], want[g > 0], rtol=1e-6)


def test_large_matrix_speed():
    """The large network's E->E matrix (8,100 x 8,100) on the GPU against the host generator."""
    e = grid(90)
    k = kw(x_location_length=90.0, y_location_length=90.0)
    generation.distance_2d_weights_gpu(e[:100], e[:100], **k)  # context and module load
    t0 = time.perf_counter()
    w = generation.distance_2d_weights_gpu(e, e, **k)
    t_gpu = time.perf_counter() - t0
    t0 = time.perf_counter()
    h = generation.distance_2d_weights(e, e, **k)
    t_host = time.perf_counter() - t0
    print(f"8100 x 8100: GPU {t_gpu * 1e3:.0f} ms (host copy included), host generator {t_host * 1e3:.0f} ms; "
          f"synapses {int((w > 0).sum())} vs {int((h > 0).sum())}")
    assert abs(int((w > 0).sum()) - int((h > 0).sum())) < 0.01 * int((h > 0).sum())
