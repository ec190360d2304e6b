"""Per-phase clock tallies of the step kernel, from the instrumented library build.

    make -C example-cuda-spiking-nn_b200 libbsnn_phase.so
    cd example-cuda-spiking-nn_b200 && python -m bsnn.phase_timing [--workload NAME] [--weight-format F]
                                                                   [--steps N] [--sm-mhz MHZ]

The instrumented kernel (compiled with -DBSNN_PHASE_TIMING) has thread 0 of every CTA add the SM
clock cycles of each phase of every step to a tally (bsnn_debug_phase_ns).  This runs a workload,
takes the difference of the tallies over `--steps` clock steps after as many warm-up steps, and
prints, per phase, the mean over the CTAs and the slowest CTA in microseconds per clock step at
`--sm-mhz` (the SM clock the run held; 1965 MHz is the B200's maximum).  The grid barrier's time
is the wait for the slowest CTA plus the release; the sum of the phases is the step.
"""
from __future__ import annotations

import argparse
import ctypes

import numpy as np

from . import _ffi
from .core import Simulation
from .network import synthetic_network

PHASES = ((3, "partial-sum loads"), (0, "other step inputs"), (1, "neuron phase beside update and normalisation"),
          (2, "spike bits and row x"), (4, "weight pass"), (5, "grid barrier"))


def load_phase_library() -> ctypes.CDLL:
    lib = _ffi.load_library(_ffi.PACKAGE_DIR / "libbsnn_phase.so")
    lib.bsnn_debug_phase_ns.restype = ctypes.c_int32
    lib.bsnn_debug_phase_ns.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong)]
    return lib


def phase_tallies(workload: str = "example_plastic_3125", weight_format: str = "f32", steps: int = 2000,
                  sm_mhz: float = 1965.0, device: int = 0) -> dict:
    """{phase name: (mean over CTAs, slowest CTA)} in microseconds per clock step."""
    lib = load_phase_library()
    spec = synthetic_network(workload, steps=2 * steps + 1, weight_values="uniform", recording_interval_steps=10000)
    sim = Simulation(spec.num_excitatory, spec.num_inhibitory, device=device, library=lib, **spec.sim_kwargs())
    try:
        spec.build(sim)
        if weight_format != "f32":
            sim.set_weight_format(weight_format)
        sim.run(0, steps)
        sim.synchronize()
        grid = sim.info().grid_ctas
        buf = (ctypes.c_ulonglong * (8 * grid))()

        def read():
            sim._check(lib.bsnn_debug_phase_ns(sim.handle, buf))
            return np.array(buf[:], dtype=np.float64).reshape(grid, 8)

        t0 = read()
        sim.run(steps, steps)
        sim.synchronize()
        us = (read() - t0) / steps / sm_mhz
    finally:
        sim.close()
    return {name: (float(us[:, p].mean()), float(us[:, p].max())) for p, name in PHASES}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", default="example_plastic_3125")
    ap.add_argument("--weight-format", default="f32", choices=["f32", "f32_rowscaled", "bf16", "fp8_e4m3"])
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--sm-mhz", type=float, default=1965.0)
    a = ap.parse_args()
    t = phase_tallies(a.workload, a.weight_format, a.steps, a.sm_mhz)
    print(f"{a.workload} ({a.weight_format}), us per clock step at {a.sm_mhz:.0f} MHz")
    print(f"{'phase':<46} {'mean':>8} {'slowest':>8}")
    for name, (mean, mx) in t.items():
        print(f"{name:<46} {mean:8.2f} {mx:8.2f}")
    print(f"{'step (sum of the means)':<46} {sum(m for m, _ in t.values()):8.2f}")


if __name__ == "__main__":
    main()
