"""Shared helpers of the element-wise parity tests: the device build and the FP64 oracle run from
the same state with the same dt sequence (the oracle's stable_dt), so differences are the device's
FP32 arithmetic alone. Metrics: the free surface eta over cells wet in both, the wet/dry mask
(h > 1e-3), the breaking mask (indicator >= 0.8, the driver's threshold,
crates/wavesim/src/lib.rs:1222) and the volume."""
import json
import math
import os

import numpy as np

from oracle.oracle import OracleSolver, set_threads
from wavesim_b200 import Solver

OUT = os.environ.get("WC_PARITY_OUT")


def record(name, metrics):
    print(name, json.dumps(metrics))
    if OUT:
        path = os.path.join(OUT, "parity_metrics.jsonl")
        with open(path, "a") as f:
            f.write(json.dumps({"case": name, **metrics}) + "\n")


def surface_metrics(w, sg, so, gpu=None, orc=None):
    g = w.grid
    hg, ho = g.inner(sg.h), g.inner(so.h)
    eg, eo = hg + g.inner(w.bed.b), ho + g.inner(w.bed.b)
    wet_both = (hg > 1e-3) & (ho > 1e-3)
    d = np.abs(eg - eo)[wet_both]
    m = {
        "time_s": so.time,
        "eta_max_abs_diff_m": float(d.max()),
        "eta_rms_diff_m": float(np.sqrt(np.mean(d * d))),
        "eta_range_m": float(eo[ho > 1e-3].max() - eo[ho > 1e-3].min()),
        "wet_mask_agreement": float(np.mean((hg > 1e-3) == (ho > 1e-3))),
        "volume_rel_diff": abs(sg.volume(g) - so.volume(g)) / so.volume(g),
    }
    if gpu is not None and orc is not None:
        bg = gpu.breaking_indicator(sg) >= 0.8
        bo = orc.breaking_indicator(so) >= 0.8
        m["breaking_mask_agreement"] = float(np.mean(bg == bo))
        m["breaking_cells_oracle"] = int(bo.sum())
    return m


def compare(w, state, steps, gpu=None):
    """`steps` steps of the device build (`gpu`, or a fresh solver of `w`) and the oracle from
    `state`; returns (metrics, device state, oracle state, device solver)."""
    set_threads(0)
    gpu = gpu or w.solver(Solver)
    orc = w.solver(OracleSolver)
    sg, so = state.clone(), state.clone()
    for _ in range(steps):
        dt = orc.stable_dt(so)
        assert math.isfinite(dt) and dt > 0
        orc.step(so, dt)
        gpu.step(sg, dt)
    m = {"steps": steps, **surface_metrics(w, sg, so, gpu, orc)}
    if w.dispersion is not None:
        m["oracle_iterations_per_solve"] = orc.dispersion_stats().iterations / max(1, orc.dispersion_stats().solves)
        m["device_iterations_per_solve"] = gpu.dispersion_stats().iterations / max(1, gpu.dispersion_stats().solves)
    return m, sg, so, gpu
