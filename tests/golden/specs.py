"""Networks of the reference-run golden fixtures, shared by make_golden.py (which runs the
reference build on a GPU to record them) and the parity tests (which rebuild the same networks
and compare).  Both sides build through bsnn.network, so the fixture stores a digest of every
input array to catch any drift of the generators."""
from __future__ import annotations

import hashlib

import numpy as np

GOLDEN_STEPS = 1000                  # clock steps recorded per fixture
CHECK_STEPS = (0, 9, 99, 499, 999)   # steps whose full state is stored


def _retime_stimulus(spec, n_ids, start, end, amp):
    """One pulse into the n_ids E neurons synthetic_network picks (same draw), from start to end."""
    from bsnn import generation
    rng = np.random.default_rng(spec.rng_seed + 101)
    ids = np.sort(rng.choice(spec.num_excitatory, size=n_ids, replace=False)).tolist()
    spec.stimulus = generation.partial_group_multiple_square_waves(
        spec.total_steps, ids, [0] * len(ids), [start], [end], [amp])
    return spec


def golden_specs():
    """name -> NetworkSpec.  `small_plastic_500` is the 400 E + 100 I example with the reference
    generator's weight values (max_weight on every accepted synapse) and its pulse moved inside
    the recorded steps; `random_120_all_rules` is a small random network with triplet, iSTDP and
    pair STDP all active, and stimulus."""
    import bsnn
    specs = {}
    s = bsnn.synthetic_network("small_plastic_500", steps=GOLDEN_STEPS + 1, weight_values="reference",
                               recording_interval_steps=GOLDEN_STEPS)
    specs["small_plastic_500"] = _retime_stimulus(s, 20, 300, 700, 0.25e-9)
    r = bsnn.random_network(96, 24, steps=GOLDEN_STEPS + 1, seed=5, plasticity=("triplet", "istdp", "stdp"),
                            stim_events=8)
    r.recording_interval_steps = GOLDEN_STEPS
    specs["random_120_all_rules"] = r
    return specs


def spec_digest(spec) -> str:
    """sha256 over every array and parameter the network is built from."""
    h = hashlib.sha256()
    h.update(repr((spec.num_excitatory, spec.num_inhibitory, spec.total_steps, spec.rng_seed,
                   spec.recording_interval_steps)).encode())
    for g in spec.groups:
        h.update(repr(sorted(g.items())).encode())
    for c in spec.conns:
        h.update(repr((c.pre, c.post, sorted(c.params.items()))).encode())
        h.update(np.ascontiguousarray(c.weights, np.float32).tobytes())
    for p in spec.plasts:
        h.update(repr((p.kind, p.conn, sorted(p.params.items()))).encode())
    if spec.stimulus is not None:
        for a, dt in zip(spec.stimulus, (np.uint32, np.uint32, np.uint32, np.float32)):
            h.update(np.asarray(a, dt).tobytes())
    for m in spec.monitors:
        h.update(repr((m.kind, m.group, tuple(m.ids), m.interval)).encode())
    return h.hexdigest()


RECORD_STEPS = 251  # System::run length of the recording fixture (records at steps 0, 50, ..., 250)


def record_spec():
    """The network of the recording fixture: the 96 E + 24 I random network with all three
    plasticity rules, a recording interval of 50 steps and its stimulus pulse moved inside the
    recorded steps; spike recorders on both groups, a voltage recorder on 8 E neurons."""
    import bsnn
    from bsnn import generation
    r = bsnn.random_network(96, 24, steps=RECORD_STEPS + 1, seed=5, plasticity=("triplet", "istdp", "stdp"),
                            stim_events=8)
    r.recording_interval_steps = 50
    ids = sorted(set(int(i) for i in r.stimulus[1]))
    r.stimulus = generation.partial_group_multiple_square_waves(r.total_steps, ids, [0] * len(ids), [60], [140],
                                                                [0.6e-9])
    return r
