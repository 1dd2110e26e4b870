"""Element-wise parity of the device build with the FP64 oracle on the same inputs.

Both engines start from the same state and take the same dt sequence (the oracle's
stable_dt), so differences are the device's FP32 arithmetic alone. Tolerances (FP32 against
FP64, stated per test): the free surface eta over cells wet in both, the wet/dry mask (h > 1e-3),
and the breaking mask (indicator >= 0.8, the driver's threshold, crates/wavesim/src/lib.rs:1222).
"""
import json
import math
import os

import numpy as np
import pytest

from oracle.oracle import OracleSolver
from wavesim_b200 import Bathymetry, Dispersion, Grid, Order, Solver, State
from wavesim_b200 import workloads as W

pytestmark = pytest.mark.gpu

OUT = os.environ.get("WC_PARITY_OUT")


def record(name, metrics):
    print(name, json.dumps(metrics))
    if OUT:
        path = os.path.join(OUT, "parity_metrics.jsonl")
        with open(path, "a") as f:
            f.write(json.dumps({"case": name, **metrics}) + "\n")


def compare(w, state, steps, every=None):
    gpu = w.solver(Solver)
    orc = w.solver(OracleSolver)
    sg, so = state.clone(), state.clone()
    g = w.grid
    for _ in range(steps):
        dt = orc.stable_dt(so)
        assert math.isfinite(dt) and dt > 0
        orc.step(so, dt)
        gpu.step(sg, dt)
    hg, ho = g.inner(sg.h), g.inner(so.h)
    eg, eo = hg + g.inner(w.bed.b), ho + g.inner(w.bed.b)
    wet_both = (hg > 1e-3) & (ho > 1e-3)
    d = np.abs(eg - eo)[wet_both]
    wet_agree = float(np.mean((hg > 1e-3) == (ho > 1e-3)))
    bg = gpu.breaking_indicator(sg) >= 0.8
    bo = orc.breaking_indicator(so) >= 0.8
    m = {
        "steps": steps,
        "time_s": so.time,
        "eta_max_abs_diff_m": float(d.max()),
        "eta_rms_diff_m": float(np.sqrt(np.mean(d * d))),
        "eta_range_m": float(eo[ho > 1e-3].max() - eo[ho > 1e-3].min()),
        "wet_mask_agreement": wet_agree,
        "breaking_mask_agreement": float(np.mean(bg == bo)),
        "breaking_cells_oracle": int(bo.sum()),
        "volume_rel_diff": abs(sg.volume(g) - so.volume(g)) / so.volume(g),
    }
    if w.dispersion is not None:
        m["oracle_iterations_per_solve"] = orc.dispersion_stats().iterations / max(1, orc.dispersion_stats().solves)
        m["device_iterations_per_solve"] = gpu.dispersion_stats().iterations / max(1, gpu.dispersion_stats().solves)
    return m, sg, so


def test_swe_plane_beach_config1_matches_the_oracle():
    """256x64 plane beach, second order, maker + sponges + Manning, 1000 steps (48 s)."""
    w = W.config1()
    s0 = State.lake_at_rest(w.grid, w.bed, 0.0)
    m, _, _ = compare(w, s0, 1000)
    record("swe_plane_beach_256x64_1000steps", m)
    # FP32 against FP64 after 1000 steps of a 1 m wave: measured 2.6e-6 m max, 6.5e-7 m rms.
    assert m["eta_max_abs_diff_m"] < 2e-5
    assert m["eta_rms_diff_m"] < 3e-6
    assert m["wet_mask_agreement"] > 0.999
    assert m["breaking_mask_agreement"] > 0.999
    assert m["volume_rel_diff"] < 1e-6


def test_fifth_order_sgn_periodic_beach_matches_the_oracle():
    """Fifth order + SGN (Jacobi PCG to 1e-8), periodic y, oblique maker: 192x96 at 2 m."""
    w = W.sgn_beach(192, 96, 2.0, seed=11, name="sgn_small")
    s0 = W.wave_train_state(w)
    m, sg, _ = compare(w, s0, 150)
    record("sgn_beach_192x96_150steps", m)
    # Measured 4.1e-6 m max, 4.5e-7 m rms on a 3.4 m surface range.
    assert m["eta_max_abs_diff_m"] < 3e-5
    assert m["eta_rms_diff_m"] < 3e-6
    assert m["wet_mask_agreement"] > 0.995
    assert m["breaking_mask_agreement"] > 0.995
    assert m["volume_rel_diff"] < 1e-5


def test_dam_break_wet_dry_front_matches_the_oracle():
    """Second order dam break onto a dry bed (a moving wet/dry front)."""
    grid = Grid(200, 8, 0.5, 0.5)
    bed = Bathymetry.flat(grid, 0.0)
    s = State.zeros(grid)
    X, _ = grid.centres()
    grid.inner(s.h)[:] = np.where(X < 50.0, 2.0, 0.0)
    gpu = Solver(grid, bed).with_order(Order.Second)
    orc = OracleSolver(grid, bed).with_order(Order.Second)
    sg, so = s.clone(), s.clone()
    for _ in range(200):
        dt = orc.stable_dt(so)
        orc.step(so, dt)
        gpu.step(sg, dt)
    d = np.abs(grid.inner(sg.h) - grid.inner(so.h))
    record("dam_break_dry_200steps", {"h_max_abs_diff_m": float(d.max())})
    assert d.max() < 1e-5  # measured 3.0e-7 m on a 2 m column
    assert abs(sg.volume(grid) - so.volume(grid)) < 1e-12 * so.volume(grid)


def test_device_resident_steps_match_host_steps():
    """wc_step_device (state in HBM) and wc_step (host arrays each step) give the same state."""
    w = W.sgn_beach(128, 64, 2.0, seed=3, name="resident")
    s0 = W.wave_train_state(w)
    a = w.solver(Solver)
    b = w.solver(Solver)
    sa = s0.clone()
    b.upload(s0)
    for _ in range(20):
        a.step(sa, 0.03)
        b.step_device(0.03)
    b.synchronize()
    sb = s0.clone()
    b.download(sb)
    g = w.grid
    assert np.max(np.abs(g.inner(sa.h) - g.inner(sb.h))) < 1e-12
    assert np.max(np.abs(g.inner(sa.hu) - g.inner(sb.hu))) < 1e-9
    assert abs(sa.time - sb.time) < 1e-12


def test_runs_are_reproducible_bit_for_bit():
    """Fixed reduction trees and a fixed CTA-to-tile map: the same run gives the same bits."""
    w = W.sgn_beach(128, 64, 2.0, seed=5, name="repro")
    s0 = W.wave_train_state(w)
    outs = []
    for _ in range(2):
        sol = w.solver(Solver)
        sol.upload(s0)
        sol.step_n(30)
        sol.synchronize()
        s = s0.clone()
        sol.download(s)
        outs.append((s.h.copy(), s.hu.copy(), s.time, sol.dispersion_stats()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2] and outs[0][3] == outs[1][3]


def test_adaptive_device_stepping_stops_at_t_end():
    """wc_step_n takes min(stable_dt, t_end - t) per step and stops once t_end is reached."""
    grid = Grid(64, 16, 1.0, 1.0)
    bed = Bathymetry.flat(grid, 2.0)
    s = State.lake_at_rest(grid, bed, 0.0)
    X, _ = grid.centres()
    grid.inner(s.h)[:] += 0.2 * np.exp(-((X - 32.0) / 4.0) ** 2)
    sol = Solver(grid, bed).with_order(Order.Fifth)
    sol.upload(s)
    sol.step_n(10_000, t_end=3.0)
    sol.synchronize()
    assert abs(sol.time_device() - 3.0) < 1e-12
    vol, mom, mn = sol.diagnostics_device()
    assert abs(vol - s.volume(grid)) < 1e-12 * vol
    assert mn >= 0.0
    dt = sol.stable_dt_device()
    assert math.isfinite(dt) and dt > 0
