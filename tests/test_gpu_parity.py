"""Element-wise parity of the device build with the FP64 oracle on the same inputs.

Both engines start from the same state and take the same dt sequence (the oracle's
stable_dt), so differences are the device's FP32 arithmetic alone. Tolerances (FP32 against
FP64, stated per test): the free surface eta over cells wet in both, the wet/dry mask (h > 1e-3),
and the breaking mask (indicator >= 0.8, the driver's threshold, crates/wavesim/src/lib.rs:1222).
"""
import math

import numpy as np
import pytest

from oracle.oracle import OracleSolver
from wavesim_b200 import Bathymetry, Dispersion, Grid, Order, Solver, State
from wavesim_b200 import workloads as W

pytestmark = pytest.mark.gpu

from parity import compare, record


def test_swe_plane_beach_config1_matches_the_oracle():
    """256x64 plane beach, second order, maker + sponges + Manning, 1000 steps (48 s)."""
    w = W.config1()
    s0 = State.lake_at_rest(w.grid, w.bed, 0.0)
    m, _, _, _ = compare(w, s0, 1000)
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
    m, sg, _, _ = compare(w, s0, 150)
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


def test_device_diagnostics_match_the_oracle():
    """wc_diagnostics_device (FP64 reductions over the resident state) against the reference's
    State::volume / max_abs_momentum / min_depth (state.rs:78-102) restated in the oracle: on the
    device state itself (downloaded: the same values), max momentum and min depth are exact and
    the volume agrees to FP64 rounding (the sums run in another order); against the oracle's own
    run from the same start, to FP32 level."""
    from oracle.oracle import diagnostics

    w = W.sgn_beach(192, 96, 2.0, seed=11, name="sgn_small")
    s0 = W.wave_train_state(w)
    m, sg, so, gpu = compare(w, s0, 40)
    gpu.upload(sg)
    vol, mom, mn = gpu.diagnostics_device()
    s_dev = sg.clone()
    gpu.download(s_dev)
    ovol, omom, omn = diagnostics(w.grid, s_dev)
    record("diagnostics_192x96_40steps", {"volume": vol, "max_abs_momentum": mom, "min_depth": mn,
                                          "oracle_run": list(diagnostics(w.grid, so))})
    assert mom == omom and mn == omn
    assert abs(vol - ovol) <= 1e-13 * ovol
    rvol, rmom, rmn = diagnostics(w.grid, so)
    assert abs(vol - rvol) <= 1e-6 * rvol
    assert abs(mom - rmom) <= 1e-4 * rmom
    assert abs(mn - rmn) <= 1e-5


@pytest.mark.parametrize("case", ["config1_walls", "beach_periodic_ragged", "first_order_dam_break"])
def test_streaming_and_tiled_shallow_water_stages_give_the_same_bits(case, monkeypatch):
    """First- and second-order shallow-water stages run in the register-streaming kernel by
    default; the shared-memory tiled kernel (WAVECORE_B200_STAGE=tiled) computes the same
    operations. On walls with maker, sponges and Manning, on a periodic beach whose sides are not
    whole strips (300 x 77), and on a first-order dam break, both give the same bits."""
    if case == "config1_walls":
        w = W.config1()
        s0 = State.lake_at_rest(w.grid, w.bed, 0.0)
        make = lambda: w.solver(Solver)
    elif case == "beach_periodic_ragged":
        w = W.swe_beach(300, 77, 2.0, seed=3)
        s0 = W.wave_train_state(w)
        make = lambda: w.solver(Solver)
    else:
        grid = Grid(150, 40, 0.5, 0.5)
        bed = Bathymetry.flat(grid, 0.0)
        s0 = State.zeros(grid)
        X, _ = grid.centres()
        grid.inner(s0.h)[:] = np.where(X < 30.0, 2.0, 0.0)
        make = lambda: Solver(grid, bed).with_order(Order.First)
    monkeypatch.setenv("WAVECORE_B200_STAGE", "tiled")
    tiled = make()
    monkeypatch.delenv("WAVECORE_B200_STAGE")
    stream = make()
    outs = []
    for sol in (tiled, stream):
        sol.upload(s0)
        sol.step_n(60)
        sol.synchronize()
        s = s0.clone()
        sol.download(s)
        outs.append(s)
    a, b = outs
    assert a.time == b.time
    assert np.array_equal(a.h, b.h) and np.array_equal(a.hu, b.hu) and np.array_equal(a.hv, b.hv)


@pytest.mark.parametrize("case", ["sgn_periodic_ragged", "sgn_walls_ragged", "fifth_order_walls"])
def test_tma_staged_and_gathered_stage_boxes_give_the_same_bits(case, monkeypatch):
    """Fifth-order and dispersive stages stage every interior tile's box (the tile and its 4-cell
    halo of state and bed) by TMA box loads; tiles at the grid's edges, whose boxes hold ghost
    cells, gather with the boundary rule as before. WAVECORE_B200_STAGE_TMA=0 gathers every box.
    On a periodic and a walled dispersive beach whose sides are not whole tiles (300 x 90, 20 steps
    with the PCG solve) and on a walled fifth-order shallow-water beach (60 steps), both give the
    same bits."""
    import dataclasses
    if case == "sgn_periodic_ragged":
        w = W.sgn_beach(300, 90, 2.0, seed=5, name="periodic")
        steps = 20
    elif case == "sgn_walls_ragged":
        w = W.sgn_beach(300, 90, 2.0, seed=6, name="walls", periodic=False)
        steps = 20
    else:
        w = dataclasses.replace(W.swe_beach(300, 77, 2.0, seed=3), order=Order.Fifth)
        steps = 60
    s0 = W.wave_train_state(w)
    monkeypatch.setenv("WAVECORE_B200_STAGE_TMA", "0")
    gathered = w.solver(Solver)
    monkeypatch.delenv("WAVECORE_B200_STAGE_TMA")
    boxed = w.solver(Solver)
    outs = []
    for sol in (gathered, boxed):
        sol.upload(s0)
        sol.step_n(steps)
        sol.synchronize()
        s = s0.clone()
        sol.download(s)
        outs.append(s)
    a, b = outs
    assert a.time == b.time
    assert np.array_equal(a.h, b.h) and np.array_equal(a.hu, b.hu) and np.array_equal(a.hv, b.hv)


@pytest.mark.parametrize("iters", [3, 4])
def test_streaming_solve_adds_the_pending_step_of_w(iters, monkeypatch):
    """The streaming Jacobi solve adds the iterations' steps to w in pairs (every second sweep adds
    its own and the previous sweep's), and after an odd number of iterations the stage epilogue
    adds the one still pending. With every solve stopped after 3 or 4 iterations, the streaming and
    the tiled solve (which adds each step at once) agree to rounding: a step left out would leave
    w short by a whole CG step."""
    import dataclasses
    base = W.sgn_beach(200, 90, 2.0, seed=5, name="periodic")
    w = dataclasses.replace(base, dispersion=Dispersion(tolerance=1e-14, max_iterations=iters))
    s0 = W.wave_train_state(w)
    monkeypatch.setenv("WAVECORE_B200_SOLVE", "tiled")
    tiled = w.solver(Solver)
    monkeypatch.delenv("WAVECORE_B200_SOLVE")
    stream = w.solver(Solver)
    outs = []
    for sol in (tiled, stream):
        sol.upload(s0)
        sol.step_n(4)
        sol.synchronize()
        s = s0.clone()
        sol.download(s)
        outs.append((s, sol.dispersion_stats()))
    (a, sa), (b, sb) = outs
    g = w.grid
    assert sa.solves == sb.solves == 8
    assert sa.unconverged == sb.unconverged == 8 and sa.iterations == sb.iterations == 8 * iters
    assert np.max(np.abs(g.inner(a.h) - g.inner(b.h))) < 1e-6
    assert np.max(np.abs(g.inner(a.hu) - g.inner(b.hu))) < 1e-5
    assert np.max(np.abs(g.inner(a.hv) - g.inner(b.hv))) < 1e-5


def test_streaming_and_tiled_jacobi_solves_agree(monkeypatch):
    """The Jacobi solve runs with register-streaming sweeps by default; the tiled sweeps
    (WAVECORE_B200_SOLVE=tiled) do the same arithmetic per cell but add the dot products' partial
    sums over other sets of cells, so the FP64 dots round differently: the two agree to the solve's
    tolerance, and their iteration counts within one per solve. Walls and periodic, sides that are
    not whole strips."""
    for w in (W.sgn_beach(200, 90, 2.0, seed=5, name="periodic"),
              W.sgn_beach(150, 70, 2.0, seed=6, name="walls", periodic=False)):
        s0 = W.wave_train_state(w)
        monkeypatch.setenv("WAVECORE_B200_SOLVE", "tiled")
        tiled = w.solver(Solver)
        monkeypatch.delenv("WAVECORE_B200_SOLVE")
        stream = w.solver(Solver)
        outs = []
        for sol in (tiled, stream):
            sol.upload(s0)
            sol.step_n(30)
            sol.synchronize()
            s = s0.clone()
            sol.download(s)
            outs.append((s, sol.dispersion_stats()))
        (a, sa), (b, sb) = outs
        g = w.grid
        assert abs(a.time - b.time) < 1e-9 * a.time
        assert np.max(np.abs(g.inner(a.h) - g.inner(b.h))) < 2e-6, w.name
        assert np.max(np.abs(g.inner(a.hu) - g.inner(b.hu))) < 2e-5, w.name
        assert sa.solves == sb.solves and sb.unconverged == 0
        assert abs(sa.iterations - sb.iterations) <= sa.solves, (sa, sb)
