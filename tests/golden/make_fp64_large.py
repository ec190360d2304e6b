"""Records the FP64 reference run of the large network for the precision tests (CPU only).

    python tests/golden/make_fp64_large.py [--steps T] [--out FILE]

The precision forms (BF16 and per-row-scaled FP8 weight copies) are measured against an FP64 run
of the same network, seed and Poisson draws: the oracle (oracle/liboracle.so) in double precision
on large_plastic_10125 (8,100 E + 2,025 I, uniform[0, max_weight] weights, seed 751, triplet STDP
+ iSTDP, the stimulus pulse at steps 20,000-22,000), T clock steps (default 30,001: 3 simulated
seconds, the pulse included).  At about 0.1 s per step on the host this takes about an hour, so
the run is stored once, as tests/golden/fp64_large_plastic_10125.npz:

  steps              T
  spikes_per_bin     int64 [T / 1000 + 1, 2]  spikes of each population per 1,000-step bin
  v_steps, v         the membrane potentials (float64) of all neurons after steps 20, 100, 1000
  w_index_<c>        int64 [200000] flat indices of a fixed random sample of the weights of the
                     plastic connections c (E->E and I->E)
  w_sample_<c>       float64 [200000] those weights after the last step
  w_abs_mean_<c>     mean |w| over the whole matrix after the last step
  digest             the network's input digest (tests/golden/specs.spec_digest)
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "example-cuda-spiking-nn_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE))

from specs import spec_digest  # noqa: E402

SAMPLE = 200_000
V_STEPS = (20, 100, 1000)


def large_spec(steps):
    import bsnn
    return bsnn.synthetic_network("large_plastic_10125", steps=steps + 1, weight_values="uniform",
                                  recording_interval_steps=1000, seed=751)


def sample_indices(spec, c, n=SAMPLE, seed=12345):
    size = spec.conns[c].weights.size
    return np.sort(np.random.default_rng(seed + c).choice(size, size=min(n, size), replace=False))


def main():
    import oracle
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=30001)
    ap.add_argument("--out", default=str(HERE / "fp64_large_plastic_10125.npz"))
    a = ap.parse_args()
    T = a.steps
    spec = large_spec(T)
    o = oracle.OracleSimulation(spec.num_excitatory, spec.num_inhibitory, precision=oracle.PREC_F64,
                                **spec.sim_kwargs())
    spec.build(o)
    bins = []
    v = []
    done = 0
    t0 = time.time()
    while done < T:
        n = min(1000 - done % 1000, T - done)
        for vs in V_STEPS:  # stop at the voltage steps inside this stretch
            if done < vs <= done + n:
                o.run(done, vs - done)
                v.append(o.read_f64("membrane_potentials"))
                n -= vs - done
                done = vs
        if n > 0:
            o.run(done, n)
            done += n
        if done % 1000 == 0 or done == T:
            # the rings hold the last 1,000 steps: the bin just completed
            filled = (done - 1) % 1000 + 1
            bins.append([int(o.read_spike_history(m)[:, :filled].sum()) for m in (0, 1)])
            print(f"{done} steps, {time.time() - t0:.0f} s, bin spikes {bins[-1]}", flush=True)
    out = {"steps": np.array(T), "spikes_per_bin": np.array(bins, np.int64), "v_steps": np.array(V_STEPS),
           "v": np.array(v), "digest": np.array(spec_digest(spec))}
    for p in spec.plasts:
        c = p.conn
        w = o.read_weights_f64(c)
        idx = sample_indices(spec, c)
        out[f"w_index_{c}"] = idx
        out[f"w_sample_{c}"] = w.ravel()[idx]
        out[f"w_abs_mean_{c}"] = np.array(float(np.mean(np.abs(w))))
    o.close()
    np.savez_compressed(a.out, **out)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
