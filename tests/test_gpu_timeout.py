"""The device-side timeout path of the persistent step kernel, made to run out on purpose without a
fault or a hang: one CTA skips its arrival at one grid barrier (bsnn_debug_skip_arrival), and
every CTA's bounded wait (bsnn_set_device_wait_limit, here 1 ms) gives up, records the failure
and returns.  The error contract is the reference's cuda_check (cpp_src/gpu_core/cuda_utils.h:10-20)
turned into status codes: the synchronising call reports BSNN_ERR_DEVICE_TIMEOUT, later calls on
that simulation BSNN_ERR_STATE, and a fresh simulation on the same device runs normally."""
from __future__ import annotations

import numpy as np
import pytest

import bsnn
from conftest import make_pair

pytestmark = pytest.mark.gpu


def test_skipped_arrival_times_out_and_the_device_stays_usable():
    spec = bsnn.random_network(96, 24, steps=400, seed=1)
    sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
    spec.build(sim)
    sim.run(0, 20)
    sim.synchronize()
    grid = sim.info().grid_ctas
    assert grid > 1
    with pytest.raises(bsnn.OutOfRange):
        sim.debug_skip_arrival(grid, 25)
    sim.set_device_wait_limit(1e-3)
    sim.debug_skip_arrival(grid // 2, 25)  # internal step 25 lies inside the next launch
    sim.run(20, 20)
    with pytest.raises(bsnn.DeviceTimeout):
        sim.synchronize()
    with pytest.raises(bsnn.StateError):
        sim.run(40, 1)
    sim.close()

    # the device and a new simulation on it are unaffected; it still matches the oracle
    g, o = make_pair(spec)
    g.run(0, 60)
    o.run(0, 60)
    g.synchronize()
    np.testing.assert_array_equal(g.read("spikes"), o.read("spikes"))
    np.testing.assert_array_equal(g.read("refractory_counter"), o.read("refractory_counter"))
    v, w = g.read("membrane_potentials").astype(np.float64), o.read("membrane_potentials").astype(np.float64)
    assert np.max(np.abs(v - w)) <= 1e-5 * np.max(np.abs(w))
    g.close()
    o.close()


def test_a_skip_outside_the_run_changes_nothing():
    """A skip armed for a step the run never reaches leaves the run intact (bit-identical to one
    without the switch)."""
    spec = bsnn.random_network(96, 24, steps=400, seed=2)
    outs = []
    for arm in (False, True):
        sim = bsnn.Simulation(spec.num_excitatory, spec.num_inhibitory, **spec.sim_kwargs())
        spec.build(sim)
        if arm:
            sim.set_device_wait_limit(1e-3)
            sim.debug_skip_arrival(0, 10_000)
        sim.run(0, 50)
        sim.synchronize()
        outs.append({f: sim.read(f) for f in ("membrane_potentials", "g_excitatory", "spikes")})
        sim.close()
    for f in outs[0]:
        np.testing.assert_array_equal(outs[0][f], outs[1][f], err_msg=f)
