"""The FP64 oracle against the reference's own known-answer tests (CPU only).

The reference (mlaegn/wavesim) stores no numeric solver vectors and its Rust toolchain is absent
here, so the oracle is pinned by the reference's unit and integration tests, ported with their
bounds, and by the measured values the reference reports for them (README.md:326-336), which the
oracle must reproduce.
"""
import math

import numpy as np
import pytest

import knowns
from oracle import oracle as orc
from oracle.oracle import OracleSolver
from wavesim_b200.model import GHOST, Bathymetry, Dispersion, Grid, Order, State, linear_wave, manning_factor


# ---- solver.rs:740-754 ----------------------------------------------------------------------------

def test_fifth_order_face_values_are_exact_for_quartics():
    p = lambda x: 1.0 + 2.0 * x - x * x + 0.5 * x**3 - 0.25 * x**4
    integral = lambda x: x + x * x - x**3 / 3.0 + 0.125 * x**4 - 0.05 * x**5
    v = [integral(m - 1.5) - integral(m - 2.5) for m in range(5)]
    lo, hi = orc.face_values(v, 1.0)
    assert abs(lo - p(-0.5)) < 1e-12
    assert abs(hi - p(0.5)) < 1e-12
    lo, hi = orc.face_values([0.0, 0.0, 1.0, 1.0, 1.0], 0.0)
    assert 0.0 <= lo <= 1.0 and 0.0 <= hi <= 1.0


# ---- dispersion.rs:637-835 ----------------------------------------------------------------------

class Lcg:
    """dispersion.rs:641-651: deterministic numbers in [-1, 1)."""

    def __init__(self, seed):
        self.s = seed

    def next(self):
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        return ((self.s >> 11) / float(1 << 53)) * 2.0 - 1.0


def _setup(rng_seed=7):
    grid = Grid(13, 9, 2.0, 3.0)
    n = grid.cells()
    rng = Lcg(rng_seed)
    heff = np.zeros(n)
    mask = np.ones(n)
    c = np.zeros(n)
    for k in range(n):
        heff[k] = 0.5 + 4.0 * (rng.next() + 1.0)
        c[k] = 3.0 * (rng.next() + 1.0)
    return grid, heff, mask, c, rng


def _random_field(grid, rng):
    x = np.zeros(grid.cells())
    y = np.zeros(grid.cells())
    for i, j in grid.interior():
        x[grid.idx(i, j)] = rng.next()
        y[grid.idx(i, j)] = rng.next()
    return x, y


def test_operator_is_symmetric_and_positive_definite():
    for periodic in (False, True):
        grid, heff, mask, c, rng = _setup()
        if periodic:
            orc.wrap_ghosts_y(grid, c)
            orc.wrap_ghosts_y(grid, heff)
        orc.mirror_ghosts(grid, c)
        if periodic:
            orc.wrap_ghosts_y(grid, c)
        for _ in range(5):
            x1, y1 = _random_field(grid, rng)
            x2, y2 = _random_field(grid, rng)
            ax1, ay1 = orc.matvec(grid, periodic, heff, mask, c, x1, y1)
            ax2, ay2 = orc.matvec(grid, periodic, heff, mask, c, x2, y2)
            left = orc.dot(grid, x2, y2, ax1, ay1)
            right = orc.dot(grid, x1, y1, ax2, ay2)
            assert abs(left - right) < 1e-10 * max(abs(left), 1.0)
            assert orc.dot(grid, x1, y1, ax1, ay1) > 0.0


def test_masked_operator_is_still_spd_and_masked_cells_stay_zero():
    grid, heff, mask, c, rng = _setup()
    orc.mirror_ghosts(grid, c)
    for k in range(grid.cells()):
        mask[k] = 1.0 if rng.next() > -0.3 else 0.0
    orc.mirror_ghosts(grid, mask)
    assert any(mask[grid.idx(i, j)] == 0.0 for i, j in grid.interior())

    def masked(v):
        x, y = v
        for i, j in grid.interior():
            k = grid.idx(i, j)
            x[k] *= mask[k]
            y[k] *= mask[k]
        return x, y

    for _ in range(5):
        x1, y1 = masked(_random_field(grid, rng))
        x2, y2 = masked(_random_field(grid, rng))
        ax1, ay1 = orc.matvec(grid, False, heff, mask, c, x1, y1)
        ax2, ay2 = orc.matvec(grid, False, heff, mask, c, x2, y2)
        left = orc.dot(grid, x2, y2, ax1, ay1)
        right = orc.dot(grid, x1, y1, ax2, ay2)
        assert abs(left - right) < 1e-10 * max(abs(left), 1.0)
        assert orc.dot(grid, x1, y1, ax1, ay1) > 0.0
        for i, j in grid.interior():
            k = grid.idx(i, j)
            if mask[k] == 0.0:
                assert (ax1[k], ay1[k]) == (0.0, 0.0)


def test_a_thin_film_neither_feels_nor_feeds_the_dispersive_system():
    grid = Grid(12, 8, 2.0, 2.0)
    film = grid.idx(GHOST + 6, GHOST + 4)

    def run(film_speed):
        s = State.zeros(grid)
        for i, j in grid.interior():
            k = grid.idx(i, j)
            s.h[k] = 2.0
            s.hu[k] = 2.0 * 0.3 * math.sin(0.7 * i)
            s.hv[k] = 2.0 * 0.2 * math.cos(0.5 * j)
        s.h[film] = 0.001
        s.hu[film] = 0.001 * film_speed
        s.hv[film] = 0.0
        s.fill_boundaries(grid, False)
        phi = np.ones(grid.cells())
        phi[film] = 0.0
        n = grid.cells()
        lh = np.array([0.01 * (k % 7) for k in range(n)])
        lhu = np.array([0.05 * (k % 5) for k in range(n)])
        lhv = np.array([0.03 * (k % 3) for k in range(n)])
        before = (lhu[film], lhv[film])
        lhu, lhv = orc.dispersion_apply(grid, False, Dispersion(), s, lh, lhu, lhv, phi)
        return lhu, lhv, before

    a_u, a_v, before = run(1.0)
    b_u, b_v, _ = run(1000.0)
    for i, j in grid.interior():
        k = grid.idx(i, j)
        if k == film:
            assert (a_u[k], a_v[k]) == before
            assert (b_u[k], b_v[k]) == before
        else:
            assert a_u[k] == b_u[k] and a_v[k] == b_v[k], (i, j)


def test_smoothstep_is_a_clamped_cubic():
    assert orc.smoothstep(1.0, 3.0, 0.0) == 0.0
    assert orc.smoothstep(1.0, 3.0, 4.0) == 1.0
    assert abs(orc.smoothstep(1.0, 3.0, 2.0) - 0.5) < 1e-15


# ---- forcing / waves.rs -----------------------------------------------------------------------

def test_linear_wave_relation_inverts_the_dispersion_relation():
    """tests/dispersion.rs:119-152, on the oracle and on the host mirror."""
    for h, period in [(2.0, 10.0), (5.0, 8.0), (8.0, 14.0), (0.5, 4.0)]:
        omega = 2.0 * math.pi / period
        k, c, cg = orc.linear_wave(omega, h, True)
        lw = linear_wave(omega, h, True)
        assert (lw.k, lw.phase_speed, lw.group_speed) == (k, c, cg)
        assert abs(knowns.sgn_omega(h, k) / omega - 1.0) < 1e-12
        assert abs(c - omega / k) < 1e-12
        eps = 1e-6 * k
        numerical = (knowns.sgn_omega(h, k + eps) - knowns.sgn_omega(h, k - eps)) / (2.0 * eps)
        assert abs(cg / numerical - 1.0) < 1e-7
        assert cg < c
        ks, cs, cgs = orc.linear_wave(omega, h, False)
        c0 = math.sqrt(9.81 * h)
        assert abs(cs - c0) < 1e-12 and abs(cgs - c0) < 1e-12 and abs(ks * c0 - omega) < 1e-12
        assert c <= c0


def test_linear_wave_refuses_a_wave_too_short():
    with pytest.raises(orc.OracleError):
        orc.linear_wave(10.0, 10.0, True)


def test_manning_factor_is_the_exact_quadratic_drag_step():
    """tests/waves.rs:224-236."""
    h, u0, dt, n = 1.5, 0.8, 0.2, 0.03
    k = 9.81 * n * n / h ** (4.0 / 3.0)
    exact = u0 / (1.0 + k * u0 * dt)
    assert abs(orc.manning_factor(h, u0, dt, n) * u0 - exact) < 1e-15
    assert orc.manning_factor(h, u0, dt, 0.0) == 1.0
    assert orc.manning_factor(h, 100.0, 100.0, 0.1) > 0.0
    assert manning_factor(h, u0, dt, n) == orc.manning_factor(h, u0, dt, n)


# ---- integration tests (crates/wavecore/tests) ---------------------------------------------------

def test_lake_at_rest_over_rough_wet_bed():
    knowns.lake_at_rest_over_rough_wet_bed(OracleSolver)


def test_lake_at_rest_with_dry_bumps():
    knowns.lake_at_rest_with_dry_bumps(OracleSolver)


def test_dam_break_conserves_volume_and_stays_positive():
    knowns.dam_break_conserves_volume_and_stays_positive(OracleSolver)


def test_walls_and_periodic_seam_keep_the_water():
    knowns.walls_and_periodic_seam_keep_the_water(OracleSolver)


def test_wet_bed_dam_break_matches_stoker_at_the_reported_rate():
    rates = knowns.check_dam_break(OracleSolver, 2.0, 0.5)
    # README.md:326 reports the measured rate 1.07 for this test.
    assert abs(rates[Order.Second] - 1.07) < 0.01, rates


def test_dry_bed_dam_break_matches_ritter_at_the_reported_rate():
    rates = knowns.check_dam_break(OracleSolver, 2.0, 0.0)
    # README.md:327 reports the measured rate 1.03.
    assert abs(rates[Order.Second] - 1.03) < 0.01, rates


def test_nan_cell_is_seen_not_skipped():
    knowns.nan_cell_is_seen_not_skipped(OracleSolver)


def test_limiting_cell_is_the_fastest_water():
    knowns.limiting_cell_is_the_fastest_water(OracleSolver)


def test_still_water_limited_by_depth_dry_land_by_nothing():
    knowns.still_water_limited_by_depth_dry_land_by_nothing(OracleSolver)


def test_standing_wave_oscillates_at_the_sgn_frequency_reported():
    out = knowns.standing_wave_at_sgn_frequency(OracleSolver)
    # README.md:336: 1.4261 rad/s with the fifth-order scheme.
    assert abs(out[Order.Fifth] - 1.4261) < 5e-5, out


def test_still_water_stays_still_with_dispersion():
    knowns.still_water_stays_still_with_dispersion(OracleSolver)


def test_swell_crosses_a_coarse_shelf_and_keeps_the_reported_height():
    kept = knowns.swell_crosses_coarse_shelf(OracleSolver)
    # README.md:345 (verification table): measured 100.7%.
    assert abs(kept - 1.007) < 0.0005, kept


def test_sponge_over_land_never_speeds_water_up():
    knowns.sponge_over_land_never_speeds_water_up(OracleSolver)


def test_held_cells_run_exactly_as_shallow_water():
    knowns.held_cells_run_exactly_as_shallow_water(OracleSolver)


def test_only_the_held_cells_change():
    knowns.only_the_held_cells_change(OracleSolver)


def test_breaking_indicator_reads_surface_not_held_cells():
    knowns.breaking_indicator_reads_surface_not_held_cells(OracleSolver)


def test_periodic_domain_refuses_a_maker_that_does_not_fit():
    """solver.rs:421-429: 15 deg at T=14 s in 20 m over Ly=1024 m is 1.455 turns."""
    from wavesim_b200.model import WaveMaker
    grid = Grid(64, 512, 2.0, 2.0)
    bed = Bathymetry.flat(grid, 20.0)
    maker = WaveMaker(x=60.0, amplitude=1.0, period=14.0, angle=math.radians(15.0), sigma=4.0, ramp_periods=4.0)
    with pytest.raises(orc.OracleError) as e:
        OracleSolver(grid, bed).with_dispersion(Dispersion()).with_wavemaker(maker).with_periodic_y().check()
    assert e.value.status == 2


def test_threaded_oracle_is_bit_identical_to_serial():
    """par.rs:1-6: row threading never changes a result."""
    grid = Grid(256, 200, 2.0, 2.0)
    bed = Bathymetry.rough(grid, 6.0, 2.0)
    outs = []
    for threads in (1, 4):
        orc.set_threads(threads)
        s = State.lake_at_rest(grid, bed, 0.0)
        X, Y = grid.centres()
        grid.inner(s.h)[:] += 0.3 * np.exp(-((X - 200) ** 2 + (Y - 150) ** 2) / 800.0)
        solver = OracleSolver(grid, bed).with_order(Order.Fifth).with_dispersion(Dispersion(tolerance=1e-6))
        for _ in range(5):
            solver.step(s, solver.stable_dt(s))
        outs.append((s.h.copy(), s.hu.copy(), s.hv.copy(), solver.dispersion_stats()))
    orc.set_threads(1)
    for a, b in zip(outs[0][:3], outs[1][:3]):
        assert np.array_equal(a, b)
    assert outs[0][3] == outs[1][3]


@pytest.mark.slow
def test_wave_maker_radiates_the_requested_amplitude():
    knowns.wave_maker_radiates_the_requested_amplitude(OracleSolver)
