"""Run a few device-resident steps of a named workload (for profilers and quick checks).

    python -m wavesim_b200.run_workload --workload swe2048 --steps 6
    python -m wavesim_b200.run_workload --workload config3 --steps 3

Workloads: the benchmark configurations of `workloads` (config1, config2, config3, config5), the
4096 x 4096 shallow-water stencil (swe4096) and a 2048 x 2048 one (swe2048, a case small enough
for a full profiler capture). The run starts from the workload's wave-train state (config1: still
water), steps on the device with the solver's adaptive time step and prints the time reached and
the dispersive solve's statistics.
"""
from __future__ import annotations

import argparse

from . import workloads as W
from .model import State
from .solver import Solver

NAMED = {
    "config1": W.config1, "config2": W.config2, "config3": W.config3, "config5": W.config5,
    "swe4096": W.swe_large, "swe2048": lambda: W.swe_beach(2048, 2048, 2.0, seed=7, name="swe_beach_2048x2048_dx2"),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="config3", choices=sorted(NAMED))
    ap.add_argument("--steps", type=int, default=3)
    a = ap.parse_args()
    w = NAMED[a.workload]()
    sol = w.solver(Solver)
    s0 = W.wave_train_state(w) if a.workload != "config1" else State.lake_at_rest(w.grid, w.bed, 0.0)
    sol.upload(s0)
    sol.step_n(a.steps)
    sol.synchronize()
    print(f"{w.name}: t = {sol.time_device():.3f} s after {a.steps} steps; solves {sol.dispersion_stats()}")


if __name__ == "__main__":
    main()
