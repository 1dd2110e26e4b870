"""The reference's known-answer tests on the device build (B200, through the C ABI).

Bounds are the reference's own (crates/wavecore/tests/*.rs) except where FP32 arithmetic makes a
different, stated bound the right one; those are named in each test.
"""
import math

import numpy as np
import pytest

import knowns
from wavesim_b200 import Order, Solver

pytestmark = pytest.mark.gpu


def test_lake_at_rest_over_rough_wet_bed_is_exactly_still():
    # The device build keeps still water bitwise still (momentum exactly 0); the reference's
    # bound is 1e-11.
    knowns.lake_at_rest_over_rough_wet_bed(Solver, momentum_bound=1e-11)


def test_lake_at_rest_with_dry_bumps():
    knowns.lake_at_rest_with_dry_bumps(Solver, momentum_bound=1e-11)


def test_dam_break_conserves_volume_and_stays_positive():
    knowns.dam_break_conserves_volume_and_stays_positive(Solver)


def test_walls_and_periodic_seam_keep_the_water_to_1e12():
    knowns.walls_and_periodic_seam_keep_the_water(Solver, bound=1e-12)


def test_wet_bed_dam_break_matches_stoker():
    rates = knowns.check_dam_break(Solver, 2.0, 0.5)
    assert abs(rates[Order.Second] - 1.07) < 0.02, rates


def test_dry_bed_dam_break_matches_ritter():
    rates = knowns.check_dam_break(Solver, 2.0, 0.0)
    assert abs(rates[Order.Second] - 1.03) < 0.02, rates


def test_nan_cell_is_seen_not_skipped():
    knowns.nan_cell_is_seen_not_skipped(Solver)


def test_limiting_cell_is_the_fastest_water():
    knowns.limiting_cell_is_the_fastest_water(Solver)


def test_still_water_limited_by_depth_dry_land_by_nothing():
    knowns.still_water_limited_by_depth_dry_land_by_nothing(Solver)


def test_standing_wave_oscillates_at_the_sgn_frequency():
    out = knowns.standing_wave_at_sgn_frequency(Solver)
    # README.md:336 reports 1.4261 rad/s (fifth order); FP32 keeps it to 1e-3.
    assert abs(out[Order.Fifth] - 1.4261) < 1e-3, out


def test_still_water_stays_still_with_dispersion():
    knowns.still_water_stays_still_with_dispersion(Solver, momentum_bound=1e-9)


def test_swell_crosses_a_coarse_shelf_and_keeps_its_height():
    kept = knowns.swell_crosses_coarse_shelf(Solver)
    assert abs(kept - 1.007) < 0.003, kept


def test_sponge_over_land_never_speeds_water_up():
    knowns.sponge_over_land_never_speeds_water_up(Solver)


def test_held_cells_run_as_shallow_water():
    # The reference holds them to 1e-9 m in FP64; in FP32 the dispersive path and plain shallow
    # water round differently (pred + dt h w against hu + dt lhu), so the bound is 1e-6 m.
    knowns.held_cells_run_exactly_as_shallow_water(Solver, bound=1e-6)


def test_only_the_held_cells_change():
    knowns.only_the_held_cells_change(Solver)


def test_breaking_indicator_reads_surface_not_held_cells():
    knowns.breaking_indicator_reads_surface_not_held_cells(Solver)


def test_periodic_domain_refuses_a_maker_that_does_not_fit():
    from wavesim_b200 import Bathymetry, Dispersion, Grid, WaveMaker, WavecoreError
    grid = Grid(64, 512, 2.0, 2.0)
    bed = Bathymetry.flat(grid, 20.0)
    maker = WaveMaker(x=60.0, amplitude=1.0, period=14.0, angle=math.radians(15.0), sigma=4.0, ramp_periods=4.0)
    with pytest.raises(WavecoreError) as e:
        Solver(grid, bed).with_dispersion(Dispersion()).with_wavemaker(maker).with_periodic_y().check()
    assert e.value.status == 2
