"""Training of the learned preconditioner on the GPU, on SGN systems the solver itself generates.

Runs of the seeded beach workload draw a swell height H ~ U(0.5, 4) m, a period T ~ U(8, 18) s
and an angle ~ U(-20, 20) degrees (and their own random bed); each run starts from its linear
wave train and, every few steps, hands the system of its last dispersive solve (c, h, bed) to
the network (`LearnedPreconditioner.harvest`). Training then takes Adam steps on batches of
random patches of those systems with random error fields (`LearnedPreconditioner.train`): every
kernel involved is the library's own.

    python -m wavesim_b200.train_lpc --out lpc_dx2.npy [--steps 20000]
"""
from __future__ import annotations

import argparse
import math
import time

import numpy as np

from . import workloads as W
from .lpc import UNetSpec
from .solver import LearnedPreconditioner, Solver


def harvest_runs(net: LearnedPreconditioner, runs: int = 8, nx: int = 512, ny: int = 256, dx: float = 2.0,
                 steps: int = 120, every: int = 20, seed: int = 0) -> dict:
    """`runs` solver runs of `steps` steps each, harvested every `every` steps."""
    rng = np.random.default_rng(seed)
    draws = []
    t0 = time.perf_counter()
    for r in range(runs):
        height = float(rng.uniform(0.5, 4.0))
        period = float(rng.uniform(8.0, 18.0))
        angle = float(rng.uniform(-20.0, 20.0))
        w = W.sgn_beach(nx, ny, dx, seed=int(rng.integers(1 << 30)), height=height, period=period, angle_deg=angle,
                        name=f"harvest_{r}")
        sol = w.solver(Solver)
        sol.upload(W.wave_train_state(w))
        for _ in range(steps // every):
            sol.step_n(every)
            sol.synchronize()
            net.harvest(sol)
        draws.append({"H_m": round(height, 3), "T_s": round(period, 3), "angle_deg": round(w.meta["angle_deg"], 3)})
    return {"runs": runs, "grid": f"{nx}x{ny} at {dx:g} m", "systems": net.n_systems, "draws": draws,
            "seconds": time.perf_counter() - t0}


def train(net: LearnedPreconditioner, steps: int = 20000, batch: int = 16, patch: int = 0, lr: float = 2e-3,
          seed: int = 0) -> dict:
    """Adam with the learning rate dropped by 4 for the last quarter; returns the loss record."""
    t0 = time.perf_counter()
    patch = patch or 64 * net.spec.stride  # the network sees 64 x 64 patches of its own grid
    main = int(math.ceil(0.75 * steps))
    l1 = net.train(main, batch=batch, patch=patch, lr=lr, seed=seed)
    l2 = net.train(steps - main, batch=batch, patch=patch, lr=lr / 4.0, seed=seed + 1)
    losses = np.concatenate([l1, l2])
    k = max(1, min(50, losses.size // 10))
    return {"steps": int(steps), "batch": batch, "patch": patch, "samples": int(steps) * batch,
            "loss_first": float(losses[:k].mean()), "loss_last": float(losses[-k:].mean()),
            "seconds": time.perf_counter() - t0}


def trained_network(dx: float = 2.0, steps: int = 20000, seed: int = 0, spec: UNetSpec | None = None):
    """A network harvested and trained from scratch on this GPU; returns (network, record)."""
    net = LearnedPreconditioner(spec or UNetSpec(), seed=seed)
    h = harvest_runs(net, dx=dx, seed=seed)
    t = train(net, steps=steps, seed=seed)
    return net, {"harvest": h, "training": t, "params": net.n_params}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--dx", type=float, default=2.0)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    net, rec = trained_network(a.dx, a.steps, a.seed)
    net.save(a.out)
    print(rec)


if __name__ == "__main__":
    main()
