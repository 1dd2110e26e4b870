"""Training of the learned preconditioner on the GPU, on SGN systems the solver itself generates.

Runs of a seeded workload family (the beach of the 2 m configurations, or config 5's reef) draw a
swell height H ~ U(0.5, 4) m, a period T ~ U(8, 18) s
and an angle ~ U(-20, 20) degrees (and their own random bed); the harvest runs have walls at
their y ends, so the maker takes the drawn angle exactly (a periodic width would snap it to the
nearest angle that fits, which on a 512 m harvest grid leaves most draws at 0 degrees or outside
the range); each run starts from its linear
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


# Harvest grids per workload family: the beach of the 2 m configurations, and config 5's reef
# (wide enough at 1 m for its 20 m shelf, the shoal and the beach: 1024 m x 256 m).
HARVEST_GRIDS = {"beach": (512, 256), "reef": (1024, 256)}


def harvest_runs(net: LearnedPreconditioner, runs: int = 8, nx: int = 0, ny: int = 0, dx: float = 2.0,
                 steps: int = 120, every: int = 20, seed: int = 0, validation: list | None = None,
                 family: str = "beach") -> dict:
    """`runs` solver runs of `steps` steps each, harvested every `every` steps, on seeded beds of
    `family` ("beach": `workloads.sgn_beach`; "reef": `workloads.sgn_reef`, config 5's bed) at the
    family's harvest grid unless nx, ny are given. With `validation` (a list), each run's last
    system is also appended to it whole, with its right-hand side and converged solution:
    (c, heff, bed, bx, by, wx, wy) as (ny, nx) FP32 arrays."""
    if family not in HARVEST_GRIDS:
        raise ValueError(f"unknown harvest family {family!r}")
    nx, ny = (nx, ny) if nx and ny else HARVEST_GRIDS[family]
    rng = np.random.default_rng(seed)
    draws = []
    t0 = time.perf_counter()
    for r in range(runs):
        height = float(rng.uniform(0.5, 4.0))
        period = float(rng.uniform(8.0, 18.0))
        angle = float(rng.uniform(-20.0, 20.0))
        if family == "reef":
            w = W.sgn_reef(nx, ny, dx, seed=int(rng.integers(1 << 30)), height=height, period=period,
                           angle_deg=angle, name=f"harvest_{r}")
        else:
            w = W.sgn_beach(nx, ny, dx, seed=int(rng.integers(1 << 30)), height=height, period=period,
                            angle_deg=angle, name=f"harvest_{r}", periodic=False)
        sol = w.solver(Solver)
        sol.upload(W.wave_train_state(w))
        for _ in range(steps // every):
            sol.step_n(every)
            sol.synchronize()
            net.harvest(sol)
        if validation is not None:
            sysd = sol.dispersion_system()
            sysd["bed"] = w.grid.inner(w.bed.b).copy()
            validation.append({k: np.asarray(v, dtype=np.float32) for k, v in sysd.items()})
        draws.append({"H_m": round(height, 3), "T_s": round(period, 3), "angle_deg": round(w.meta["angle_deg"], 3)})
    return {"runs": runs, "family": family, "grid": f"{nx}x{ny} at {dx:g} m", "systems": net.n_systems, "draws": draws,
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


def validation_loss(net: LearnedPreconditioner, systems: list, dx: float, patch: int = 64, per_system: int = 8,
                    seed: int = 1) -> float:
    """The training objective on SGN systems harvested whole from solver runs (depth, bed, right-hand
    side, converged solution), with the converged solution itself as the error field: on random
    patches (zero outside, as in training), the mean of <d, A d> / <e, A e> with d = e - M A e is
    the share of a real solution's energy that one application of the preconditioner leaves."""
    rng = np.random.default_rng(seed)
    cs, hs, bs, es = [], [], [], []
    for sy in systems:
        ny, nx = sy["c"].shape
        for _ in range(per_system):
            y0 = int(rng.integers(0, ny - patch + 1))
            x0 = int(rng.integers(0, nx - patch + 1))
            sl = (slice(y0, y0 + patch), slice(x0, x0 + patch))
            wet = sy["heff"][sl] >= np.float32(0.05)
            cs.append(sy["c"][sl])
            hs.append(sy["heff"][sl])
            bs.append(sy["bed"][sl])
            es.append(np.stack([sy["wx"][sl] * wet, sy["wy"][sl] * wet]))
    loss, _ = net.loss_grad(np.stack(cs), np.stack(hs), np.stack(bs), np.stack(es), dx, dx)
    return float(loss)


def trained_network(dx: float = 2.0, steps: int = 20000, seed: int = 0, spec: UNetSpec | None = None,
                    family: str = "beach"):
    """A network harvested (from runs of `family`) and trained from scratch on this GPU; returns
    (network, record). The
    record holds the validation loss on the harvest runs' whole systems (their right-hand sides and
    converged solutions) for the trained network and for the same cycle without a network (an
    untrained network's output layer is zero: the two Jacobi sweeps alone)."""
    spec = spec or UNetSpec()
    net = LearnedPreconditioner(spec, seed=seed)
    val = []
    h = harvest_runs(net, dx=dx, seed=seed, validation=val, family=family)
    t = train(net, steps=steps, seed=seed)
    v = {"systems": len(val), "patches": 8 * len(val), "error_field": "the converged solution of the system",
         "loss_trained": validation_loss(net, val, dx),
         "loss_without_network": validation_loss(LearnedPreconditioner(spec, seed=seed), val, dx)}
    return net, {"harvest": h, "training": t, "validation": v, "params": net.n_params}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--dx", type=float, default=2.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--family", default="beach", choices=sorted(HARVEST_GRIDS))
    a = ap.parse_args()
    net, rec = trained_network(a.dx, a.steps, a.seed, family=a.family)
    net.save(a.out)
    print(rec)


if __name__ == "__main__":
    main()
