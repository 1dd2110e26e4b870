"""The reference's known-answer tests, written once over a solver class.

Each function takes `Solver` (the FP64 oracle's `OracleSolver` or the device build's
`wavesim_b200.Solver`, both with wavecore's builder API) and asserts the bound the reference's
test asserts, or a stated FP32 bound where the device build computes in single precision.
Sources are mlaegn/wavesim `crates/wavecore/tests/*.rs`.
"""
from __future__ import annotations

import math

import numpy as np

from wavesim_b200.model import (
    G,
    GHOST,
    Bathymetry,
    Dispersion,
    Grid,
    Order,
    Sponge,
    State,
    WaveMaker,
    linear_wave,
)

ORDERS3 = [Order.First, Order.Second, Order.Fifth]


def _run(solver, s, steps):
    """well_balanced.rs:7-13."""
    for _ in range(steps):
        dt = solver.stable_dt(s)
        assert math.isfinite(dt) and dt > 0.0, "no valid time step"
        solver.step(s, dt)


def run_to(solver, s, t_end):
    """dispersion.rs:21-27."""
    while s.time < t_end:
        dt = solver.stable_dt(s)
        assert math.isfinite(dt), "no water in the domain"
        solver.step(s, min(dt, t_end - s.time))


# ---- well_balanced.rs -------------------------------------------------------------------------


def lake_at_rest_over_rough_wet_bed(Solver, momentum_bound=1e-11, orders=ORDERS3, steps=500):
    """well_balanced.rs:15-35."""
    for order in orders:
        grid = Grid(64, 48, 3.0, 3.0)
        bed = Bathymetry.rough(grid, 8.0, 3.0)
        s = State.lake_at_rest(grid, bed, 0.0)
        solver = Solver(grid, bed).with_order(order)
        v0 = s.volume(grid)
        _run(solver, s, steps)
        assert s.max_abs_momentum(grid) < momentum_bound, (order, s.max_abs_momentum(grid))
        assert abs(s.volume(grid) - v0) < 1e-9 * v0, order
        assert s.min_depth(grid) >= 0.0, order


def lake_at_rest_with_dry_bumps(Solver, momentum_bound=1e-11, orders=ORDERS3, steps=500):
    """well_balanced.rs:37-62."""
    for order in orders:
        grid = Grid(64, 48, 3.0, 3.0)
        bed = Bathymetry.rough(grid, 0.5, 2.5)
        s = State.lake_at_rest(grid, bed, 0.0)
        solver = Solver(grid, bed).with_order(order)
        v0 = s.volume(grid)
        dry = int(np.count_nonzero(grid.inner(s.h) == 0.0))
        assert dry > 0, "test bed has no dry cells"
        _run(solver, s, steps)
        assert s.max_abs_momentum(grid) < momentum_bound, (order, s.max_abs_momentum(grid))
        assert abs(s.volume(grid) - v0) < 1e-9 * v0, order
        assert s.min_depth(grid) >= 0.0, order


def dam_break_conserves_volume_and_stays_positive(Solver, orders=ORDERS3):
    """well_balanced.rs:64-84."""
    for order in orders:
        grid = Grid(100, 4, 1.0, 1.0)
        bed = Bathymetry.flat(grid, 0.0)
        s = State.zeros(grid)
        inner = grid.inner(s.h)
        inner[:, :50] = 2.0
        solver = Solver(grid, bed).with_order(order)
        v0 = s.volume(grid)
        _run(solver, s, 300)
        assert abs(s.volume(grid) - v0) < 1e-9 * v0, order
        assert s.min_depth(grid) >= 0.0, order
        assert s.h[grid.idx(GHOST + 70, GHOST + 2)] > 0.0, order


def walls_and_periodic_seam_keep_the_water(Solver, bound=1e-12):
    """well_balanced.rs:86-121: closed basin / periodic seam volume to 1e-12."""
    grid = Grid(40, 30, 1.0, 1.0)
    bed = Bathymetry.flat(grid, 2.0)
    changes = {}
    for periodic in (False, True):
        for dispersive in (False, True):
            solver = Solver(grid, bed.clone()).with_order(Order.Fifth)
            if dispersive:
                solver = solver.with_dispersion(Dispersion())
            if periodic:
                solver = solver.with_periodic_y()
            s = State.lake_at_rest(grid, bed, 0.0)
            cy = 0.5 if periodic else 2.5
            X, Y = grid.centres()
            r2 = (X - 20.0) ** 2 + (Y - cy) ** 2
            grid.inner(s.h)[:] += 1.3 * np.exp(-r2 / 32.0)
            v0 = s.volume(grid)
            _run(solver, s, 300)
            change = (s.volume(grid) - v0) / v0
            changes[(periodic, dispersive)] = change
            assert abs(change) < bound, (periodic, dispersive, change)
    return changes


# ---- stoker.rs ----------------------------------------------------------------------------------

LENGTH, DAM = 100.0, 50.0


class Exact:
    """stoker.rs:10-70: exact 1D dam break."""

    def __init__(self, h_l, h_r):
        self.h_l, self.h_r = h_l, h_r
        c_l = math.sqrt(G * h_l)
        if h_r <= 0.0:
            self.h_m, self.u_m, self.shock = 0.0, 0.0, 2.0 * c_l
            return

        def f(h_m):
            return 2.0 * (c_l - math.sqrt(G * h_m)) - (h_m - h_r) * math.sqrt(0.5 * G * (h_m + h_r) / (h_m * h_r))

        lo, hi = h_r, h_l
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if f(mid) > 0.0:
                lo = mid
            else:
                hi = mid
        self.h_m = 0.5 * (lo + hi)
        self.u_m = 2.0 * (c_l - math.sqrt(G * self.h_m))
        self.shock = self.h_m * self.u_m / (self.h_m - h_r)

    def depth(self, xi):
        c_l = math.sqrt(G * self.h_l)
        if xi < -c_l:
            return self.h_l
        if self.h_r <= 0.0:
            return (2.0 * c_l - xi) ** 2 / (9.0 * G) if xi < 2.0 * c_l else 0.0
        if xi <= self.u_m - math.sqrt(G * self.h_m):
            return (2.0 * c_l - xi) ** 2 / (9.0 * G)
        if xi < self.shock:
            return self.h_m
        return self.h_r


def dam_break_error(Solver, nx, order, h_l, h_r, t_end):
    """stoker.rs:72-99: L1 depth error against the exact solution."""
    dx = LENGTH / nx
    grid = Grid(nx, 4, dx, dx)
    bed = Bathymetry.flat(grid, 0.0)
    s = State.zeros(grid)
    X, _ = grid.centres()
    grid.inner(s.h)[:] = np.where(X < DAM, h_l, h_r)
    solver = Solver(grid, bed).with_order(order)
    t = 0.0
    while t < t_end:
        dt = min(solver.stable_dt(s), t_end - t)
        solver.step(s, dt)
        t += dt
    exact = Exact(h_l, h_r)
    j = GHOST + 2
    err = 0.0
    for i in range(GHOST, GHOST + nx):
        x, _ = grid.centre(i, j)
        err += abs(s.h[grid.idx(i, j)] - exact.depth((x - DAM) / t_end)) * dx
    return err


def check_dam_break(Solver, h_l, h_r):
    """stoker.rs:100-140; returns the observed rates per order."""
    t = 4.0
    first = dam_break_error(Solver, 400, Order.First, h_l, h_r, t)
    rates = {}
    for order in (Order.Second, Order.Fifth):
        coarse = dam_break_error(Solver, 200, order, h_l, h_r, t)
        fine = dam_break_error(Solver, 400, order, h_l, h_r, t)
        rate = math.log2(coarse / fine)
        assert fine < 0.25 * first, (order, fine, first)
        assert rate > 0.9, (order, rate)
        rates[order] = rate
    return rates


# ---- time_step.rs -------------------------------------------------------------------------------


def _lake(Solver):
    grid = Grid(20, 10, 2.0, 2.0)
    bed = Bathymetry.flat(grid, 2.0)
    return Solver(grid, bed), State.lake_at_rest(grid, bed, 0.0)


def nan_cell_is_seen_not_skipped(Solver):
    """time_step.rs:12-29."""
    solver, s = _lake(Solver)
    g = solver.grid
    still = solver.stable_dt(s)
    s.hu[g.idx(GHOST + 7, GHOST + 3)] = float("nan")
    assert math.isnan(solver.stable_dt(s))
    c = solver.limiting_cell(s)
    assert (c.i, c.j) == (7, 3)
    assert math.isnan(c.speed) and c.depth == 2.0
    _, s = _lake(Solver)
    s.h[:] = float("nan")
    assert math.isnan(solver.stable_dt(s))
    assert math.isfinite(still) and still > 0.0


def limiting_cell_is_the_fastest_water(Solver):
    """time_step.rs:31-48."""
    solver, s = _lake(Solver)
    g = solver.grid
    k = g.idx(GHOST + 12, GHOST + 4)
    s.h[k] = 1e-3
    s.hu[k] = 0.5
    c = solver.limiting_cell(s)
    assert (c.i, c.j) == (12, 4)
    assert abs(c.speed - 500.0) < 1e-9 and c.depth == 1e-3
    film = (500.0 + math.sqrt(9.81e-3)) / 2.0 + math.sqrt(9.81e-3) / 2.0
    assert abs(solver.stable_dt(s) - solver.cfl / film) < 1e-9 * solver.cfl / film
    s.hu[k] = float("inf")
    assert solver.stable_dt(s) == 0.0


def still_water_limited_by_depth_dry_land_by_nothing(Solver):
    """time_step.rs:50-62."""
    solver, s = _lake(Solver)
    c = solver.limiting_cell(s)
    assert (c.depth, c.speed) == (2.0, 0.0)
    grid = Grid(6, 4, 2.0, 2.0)
    bed = Bathymetry.flat(grid, -1.0)
    dry = State.lake_at_rest(grid, bed, 0.0)
    solver = Solver(grid, bed)
    assert solver.limiting_cell(dry) is None
    assert solver.stable_dt(dry) == float("inf")


# ---- dispersion.rs (tests) ----------------------------------------------------------------------


def sgn_omega(h, k):
    return math.sqrt(G * h * k * k / (1.0 + (k * h) ** 2 / 3.0))


def model(Solver, grid, bed, dispersive, order):
    s = Solver(grid, bed).with_order(order)
    return s.with_dispersion(Dispersion()) if dispersive else s


def standing_wave_omega(Solver, dispersive, order):
    """dispersion.rs:53-89."""
    depth, length, mode, amplitude = 5.0, 100.0, 8.0, 0.01
    dx = 0.5
    grid = Grid(200, 4, dx, dx)
    solver = model(Solver, grid, Bathymetry.flat(grid, depth), dispersive, order)
    k = mode * math.pi / length
    s = State.zeros(grid)
    X, _ = grid.centres()
    grid.inner(s.h)[:] = depth + amplitude * np.cos(k * X)
    probe = grid.idx(GHOST, GHOST + 2)
    crossings = []
    previous = (0.0, amplitude * math.cos(k * 0.25))
    while s.time < 14.0:
        dt = solver.stable_dt(s)
        solver.step(s, dt)
        eta = s.h[probe] - depth
        if previous[1] * eta < 0.0:
            f = previous[1] / (previous[1] - eta)
            crossings.append(previous[0] + f * (s.time - previous[0]))
        previous = (s.time, eta)
    assert len(crossings) >= 5
    return (len(crossings) - 1) * math.pi / (crossings[-1] - crossings[0])


def standing_wave_at_sgn_frequency(Solver):
    """dispersion.rs:91-117; returns the measured frequencies."""
    depth, k = 5.0, 8.0 * math.pi / 100.0
    sgn = sgn_omega(depth, k)
    shallow = math.sqrt(G * depth) * k
    exact = math.sqrt(G * k * math.tanh(k * depth))
    measured_shallow = standing_wave_omega(Solver, False, Order.Second)
    assert abs(measured_shallow / shallow - 1.0) < 0.01
    out = {"shallow": measured_shallow}
    for order in (Order.Second, Order.Fifth):
        m = standing_wave_omega(Solver, True, order)
        assert abs(m / sgn - 1.0) < 0.01, (order, m, sgn)
        assert abs(m / exact - 1.0) < 0.03
        out[order] = m
    assert abs(shallow / exact - 1.0) > 0.15
    return out


def still_water_stays_still_with_dispersion(Solver, momentum_bound=1e-9):
    """dispersion.rs:629-652."""
    for (mean_depth, amplitude) in ((8.0, 3.0), (0.5, 2.5)):
        for order in (Order.Second, Order.Fifth):
            grid = Grid(64, 48, 3.0, 3.0)
            bed = Bathymetry.rough(grid, mean_depth, amplitude)
            s = State.lake_at_rest(grid, bed, 0.0)
            solver = Solver(grid, bed).with_order(order).with_dispersion(Dispersion())
            v0 = s.volume(grid)
            run_to(solver, s, 30.0)
            assert s.max_abs_momentum(grid) < momentum_bound, (mean_depth, order, s.max_abs_momentum(grid))
            assert abs(s.volume(grid) - v0) < 1e-9 * v0
            assert s.min_depth(grid) >= 0.0


def run_and_analyse(solver, s, t_end, omega, window, probes):
    """tests/common/mod.rs:5-68: first-harmonic amplitude and phase at probes."""
    g = solver.grid
    sums = [[0.0, 0.0] for _ in probes]
    bed = solver.bed.b
    while s.time < t_end:
        dt = solver.stable_dt(s)
        assert math.isfinite(dt)
        dt = min(dt, t_end - s.time)
        solver.step(s, dt)
        t = s.time
        if t <= window[0] or t > window[1]:
            continue
        c, sn = math.cos(omega * t), math.sin(omega * t)
        for acc, (i, j) in zip(sums, probes):
            e = s.h[g.idx(i, j)] + bed[g.idx(i, j)]
            acc[0] += e * c * dt
            acc[1] -= e * sn * dt
    scale = 2.0 / (window[1] - window[0])
    return [(scale * math.hypot(re, im), math.atan2(im, re)) for re, im in sums]


def col(grid, x):
    return GHOST + int(x / grid.dx)


def swell_crosses_coarse_shelf(Solver):
    """dispersion.rs:456-492; returns the fraction of the height kept over 1 km."""
    dx, depth, period, amplitude = 6.0, 12.0, 14.0, 0.1
    grid = Grid(310, 4, dx, dx)
    bed = Bathymetry.flat(grid, depth)
    maker = WaveMaker(x=260.0, amplitude=amplitude, period=period, angle=0.0, sigma=2.0 * dx, ramp_periods=2.0)
    solver = (
        Solver(grid, bed)
        .with_order(Order.Fifth)
        .with_dispersion(Dispersion())
        .with_wavemaker(maker)
        .with_sponge(Sponge(37, 1.5).edges(True, True, False, False))
    )
    s = State.lake_at_rest(grid, solver.bed, 0.0)
    j = GHOST + 2
    probes = [(col(grid, 460.0), j), (col(grid, 1460.0), j)]
    omega = 2.0 * math.pi / period
    window = (160.0, 160.0 + 4.0 * period)
    out = run_and_analyse(solver, s, window[1], omega, window, probes)
    kept = out[1][0] / out[0][0]
    assert kept > 0.97, kept
    return kept


# ---- waves.rs -----------------------------------------------------------------------------------


def sponge_over_land_never_speeds_water_up(Solver):
    """waves.rs:299-337."""
    grid = Grid(20, 20, 2.0, 2.0)
    bed = Bathymetry.flat(grid, -0.5)
    s = State.zeros(grid)
    grid.inner(s.h)[:] = 1.0
    grid.inner(s.hu)[:] = 1.0
    grid.inner(s.hv)[:] = 0.5
    solver = Solver(grid, bed).with_sponge(Sponge(1_000_000, 1.5).edges(True, False, False, False))
    for _ in range(3):
        solver.step(s, 0.05)
    for i in range(GHOST + 7, GHOST + 13):
        for j in range(GHOST + 7, GHOST + 13):
            k = grid.idx(i, j)
            assert s.h[k] < 1.0
            u, v = s.hu[k] / s.h[k], s.hv[k] / s.h[k]
            assert abs(u - 1.0) < 1e-6 and abs(v - 0.5) < 1e-6, (i, j, u, v)


def wave_maker_radiates_the_requested_amplitude(Solver):
    """waves.rs:11-49 (slow in the reference)."""
    dx = 0.5
    grid = Grid(800, 4, dx, dx)
    bed = Bathymetry.flat(grid, 2.0)
    period, amplitude = 20.0, 0.05
    maker = WaveMaker(x=200.0, amplitude=amplitude, period=period, angle=0.0, sigma=2.0, ramp_periods=2.0)
    solver = Solver(grid, bed).with_wavemaker(maker).with_sponge(Sponge(120, 1.0).edges(True, True, False, False))
    s = State.lake_at_rest(grid, solver.bed, 0.0)
    j = GHOST + 2
    probes = [(col(grid, 120.0), j), (col(grid, 290.0), j)]
    omega = 2.0 * math.pi / period
    out = run_and_analyse(solver, s, 180.0, omega, (100.0, 180.0), probes)
    errs = []
    for amp, _ in out:
        err = abs(amp - amplitude) / amplitude
        assert err < 0.02, err
        errs.append(err)
    return errs


# ---- shallow_cells.rs -----------------------------------------------------------------------------


def _hump():
    grid = Grid(120, 4, 1.0, 1.0)
    bed = Bathymetry.flat(grid, 2.0)
    s = State.lake_at_rest(grid, bed, 0.0)
    X, _ = grid.centres()
    grid.inner(s.h)[:] += 0.1 * np.exp(-(((X - 40.0) / 5.0) ** 2))
    return grid, bed, s


def _surface(solver, s, steps):
    for _ in range(steps):
        solver.step(s, 0.05)
    return grid_inner_copy(solver.grid, s.h)


def grid_inner_copy(grid, a):
    return grid.inner(a).copy().ravel()


def held_cells_run_exactly_as_shallow_water(Solver, bound=1e-9):
    """shallow_cells.rs:38-64."""
    grid, bed, s = _hump()

    def dispersive():
        return Solver(grid, bed.clone()).with_order(Order.Fifth).with_dispersion(Dispersion())

    shallow = Solver(grid, bed.clone()).with_order(Order.Second)
    allc = np.ones(grid.nx * grid.ny, dtype=bool)
    held = _surface(dispersive().with_shallow_cells(allc), s.clone(), 200)
    plain = _surface(shallow, s.clone(), 200)
    free = _surface(dispersive(), s.clone(), 200)
    gap = np.max(np.abs(held - plain))
    assert gap < bound, gap
    assert np.max(np.abs(free - plain)) > 1e-4
    return gap


def only_the_held_cells_change(Solver):
    """shallow_cells.rs:66-90."""
    grid, bed, s = _hump()

    def dispersive():
        return Solver(grid, bed.clone()).with_order(Order.Fifth).with_dispersion(Dispersion())

    far = np.array([[i >= 110 for i in range(grid.nx)] for _ in range(grid.ny)]).ravel()
    allc = np.ones(grid.nx * grid.ny, dtype=bool)
    held = _surface(dispersive().with_shallow_cells(far), s.clone(), 200)
    everywhere = _surface(dispersive().with_shallow_cells(allc), s.clone(), 200)
    free = _surface(dispersive(), s.clone(), 200)
    near, whole = np.max(np.abs(held - free)), np.max(np.abs(everywhere - free))
    assert near < 0.01 * whole, (near, whole)


def breaking_indicator_reads_surface_not_held_cells(Solver, atol=0.0):
    """shallow_cells.rs:92-107."""
    grid, bed, s = _hump()

    def make():
        return Solver(grid, bed.clone()).with_order(Order.Fifth).with_dispersion(Dispersion())

    held = make().with_shallow_cells(np.ones(grid.nx * grid.ny, dtype=bool))
    ind = held.breaking_indicator(s)
    ref = make().breaking_indicator(s)
    assert np.max(np.abs(ind - ref)) <= atol
    assert np.all(ind < 0.1)
