"""The oracle's followed breaking fronts (crates/wavecore/src/eddy.rs) against the reference's own
unit tests of that file (eddy.rs:304-443), ported with their bounds, plus the step-level facts the
solver relies on (solver.rs:479-532). CPU only."""
import math

import numpy as np

from oracle import oracle as orc
from oracle.oracle import OracleSolver
from wavesim_b200.model import GHOST, Bathymetry, Breaking, Dispersion, EddyViscosity, G, Grid, State


def span(e, h):
    return e.duration * math.sqrt(h / G)


# ---- eddy.rs:308-316 ----------------------------------------------------------------------------

def test_the_threshold_falls_from_onset_to_settled_over_the_duration():
    e = EddyViscosity()
    h = 1.0
    sp = 5.0 * math.sqrt(h / G)
    assert orc.eddy_threshold(e, 0.0, h) == 0.65
    assert abs(orc.eddy_threshold(e, 0.5 * sp, h) - 0.40) < 1e-12
    assert orc.eddy_threshold(e, 2.0 * sp, h) == 0.15


def channel(grid, breaking, momentum):
    """eddy.rs:318-330: still water 1 m deep, hu set by momentum(i) along x (padded i)."""
    s = State.zeros(grid)
    for i, j in grid.interior():
        k = grid.idx(i, j)
        s.h[k] = 1.0
        s.hu[k] = momentum(i)
    s.breaking[:] = breaking
    s.fill_walls(grid)
    return s


# ---- eddy.rs:332-366 ----------------------------------------------------------------------------

def test_diffusion_conserves_momentum_and_smooths_a_jump():
    grid = Grid(40, 3, 0.1, 0.1)
    none = np.zeros(grid.cells())
    s = channel(grid, none, lambda i: 0.5 if i < GHOST + 20 else 0.0)
    nu = np.zeros(grid.cells())
    for i, j in grid.interior():
        if GHOST + 8 <= i < GHOST + 32:
            nu[grid.idx(i, j)] = 0.05

    def total(s):
        return sum(s.hu[grid.idx(i, j)] for i, j in grid.interior())

    before = total(s)
    steps = orc.eddy_diffuse(grid, s, nu, 0.5)
    assert steps > 1, f"the sub-steps were not needed: {steps}"
    assert abs(total(s) - before) < 1e-9 * before
    j = GHOST + 1
    a, b = s.hu[grid.idx(GHOST + 19, j)], s.hu[grid.idx(GHOST + 20, j)]
    assert a < 0.5 and b > 0.0 and a > b, f"not smoothed: {a} {b}"
    assert all(-1e-12 <= s.hu[grid.idx(i, j)] <= 0.5 + 1e-12 for i, j in grid.interior()), "diffusion overshot"


# ---- eddy.rs:368-442 ----------------------------------------------------------------------------

def test_a_front_starts_where_the_switch_says_moves_on_with_its_age_and_lingers_behind():
    grid = Grid(20, 3, 0.1, 0.1)
    e = EddyViscosity()
    dt, c = 0.01, math.sqrt(G)

    def cell(i):
        return grid.idx(GHOST + i, GHOST + 1)

    def towards(at, rate):
        a = rate * c * 0.1
        return lambda i: a if i < GHOST + at else (0.0 if i == GHOST + at else -a)

    smooth = np.ones(grid.cells())
    none = np.zeros(grid.cells())
    # Rising fast but smooth by the switch: no front.
    s = channel(grid, none, towards(5, 0.8))
    orc.eddy_follow(grid, e, s, smooth, dt)
    assert np.all(s.breaking == 0.0), "a front without the switch"
    # The switch reads breaking at cells 3 to 7, but only 4 to 6 rise: fronts there.
    broken = smooth.copy()
    for i in range(3, 8):
        broken[cell(i)] = 0.0
    s = channel(grid, none, towards(5, 0.8))
    nu = orc.eddy_follow(grid, e, s, broken, dt)
    assert s.breaking[cell(5)] == dt
    assert s.breaking[cell(4)] == dt
    assert s.breaking[cell(3)] == 0.0, "a front where the surface does not rise"
    assert nu[cell(5)] > 0.0
    assert nu[cell(4)] == 0.0, "rising at 0.4 has a viscosity"
    # A front broken for longer than the transition goes on where the surface rises at
    # 0.35 sqrt(g h); a step on the rise has moved a cell and the front keeps its age; the cell
    # it has left behind starts to linger.
    old = 2.0 * span(e, 1.0)
    bore = none.copy()
    for i in range(4, 7):
        bore[cell(i)] = old
    s = channel(grid, bore, towards(6, 0.7))
    orc.eddy_follow(grid, e, s, smooth, dt)
    assert s.breaking[cell(6)] == old + dt
    assert s.breaking[cell(5)] == old + dt, "a bore rising at 0.35 stopped"
    linger = e.linger * math.sqrt(1.0 / G)
    assert s.breaking[cell(4)] == -linger
    # In still water the fronts stop and linger too, the lingering counts down, and nothing
    # has a viscosity.
    s = channel(grid, s.breaking.copy(), lambda i: 0.0)
    nu = orc.eddy_follow(grid, e, s, smooth, dt)
    assert s.breaking[cell(6)] == -linger
    assert abs(s.breaking[cell(4)] + linger - dt) < 1e-15
    assert np.all(nu == 0.0), "still water has a viscosity"


# ---- solver.rs:479-532: the step with followed fronts -------------------------------------------

def _eddy_dispersion(**kw):
    return Dispersion(breaking=Breaking(viscosity=EddyViscosity(**kw)), tolerance=1e-8)


def test_still_water_with_followed_fronts_stays_still():
    grid = Grid(24, 12, 1.0, 1.0)
    bed = Bathymetry.plane_beach(grid, 0.05, 2.0)
    sol = OracleSolver(grid, bed).with_dispersion(_eddy_dispersion())
    s = State.lake_at_rest(grid, bed, 0.0)
    h0 = s.h.copy()
    for _ in range(5):
        sol.step(s, 0.05)
    inner = grid.inner
    assert np.array_equal(inner(s.h), inner(h0))
    assert np.all(inner(s.hu) == 0.0) and np.all(inner(s.hv) == 0.0)
    assert np.all(inner(s.breaking) == 0.0)


def _bore(grid, up=2.0):
    """A dam break on a flat bed 1 m deep: `up` metres more water west of x = 5 m. The bore it
    sends east keeps breaking by Kennedy's criterion."""
    bed = Bathymetry.flat(grid, 1.0)
    s = State.lake_at_rest(grid, bed, 0.0)
    for i, j in grid.interior():
        if (i - GHOST + 0.5) * grid.dx < 5.0:
            s.h[grid.idx(i, j)] += up
    s.fill_walls(grid)
    return bed, s


def test_a_bore_is_followed_and_keeps_the_switch_off_where_it_breaks():
    grid = Grid(64, 8, 0.25, 0.25)
    bed, s0 = _bore(grid)
    dt = 0.008
    follow = OracleSolver(grid, bed).with_dispersion(_eddy_dispersion())
    s = s0.clone()
    ages = []
    for _ in range(60):
        follow.step(s, dt)
        ages.append(float(grid.inner(s.breaking).max()))
    mem = grid.inner(s.breaking)
    assert np.any(mem > 0.0), "no front followed"
    assert np.any(mem < 0.0), "nothing lingers behind the front"
    # the oldest front has broken since the first step: its age grows by dt every step
    assert abs(ages[-1] - 60 * dt) < 1e-9
    # the indicator reads 1 wherever the memory holds a front and the water carries a wave
    ind = follow.breaking_indicator(s).reshape(grid.ny, grid.nx)
    h = grid.inner(s.h)
    held = (mem != 0.0) & (h >= 0.05)
    assert held.any() and np.all(ind[held] == 1.0)


def test_without_viscosity_the_memory_is_carried_unchanged_and_the_step_is_the_plain_one():
    grid = Grid(64, 8, 0.25, 0.25)
    bed, s0 = _bore(grid)
    plain = OracleSolver(grid, bed).with_dispersion(Dispersion(tolerance=1e-8))
    a = s0.clone()
    a.breaking[:] = 0.25
    for _ in range(5):
        plain.step(a, 0.008)
    assert np.all(a.breaking == 0.25)
    assert plain.follow_breaking(a.clone(), 0.008) == 0


def test_the_viscosity_takes_sub_steps_and_mixing_zero_takes_none():
    grid = Grid(64, 8, 0.25, 0.25)
    bed, s0 = _bore(grid)
    sol = OracleSolver(grid, bed).with_dispersion(_eddy_dispersion())
    zero = OracleSolver(grid, bed).with_dispersion(_eddy_dispersion(mixing=0.0))
    a, b = s0.clone(), s0.clone()
    for _ in range(20):
        sol.step(a, 0.008)
        zero.step(b, 0.008)
    assert sol.follow_breaking(a.clone(), 0.008) >= 1
    assert zero.follow_breaking(b.clone(), 0.008) == 0
    # the same fronts are followed either way on the first step; the viscosity then changes the flow
    assert np.any(grid.inner(a.hu) != grid.inner(b.hu))
