"""The seeded workloads the benchmark and the training harvest draw from (host only)."""
import numpy as np
import pytest

from wavesim_b200 import Grid
from wavesim_b200 import workloads as W


def test_reef_family_runs_have_the_shelf_the_shoal_and_dry_land():
    # The training harvest for config 5 runs this family at 1024 x 256 cells of 1 m: wide enough
    # for the 20 m shelf, the shoal whose crest is 1 m deep at mid-width, and the beach.
    w = W.sgn_reef(1024, 256, 1.0, seed=3)
    b = w.grid.inner(w.bed.b)
    assert not w.periodic_y and w.dispersion is not None
    assert b[:, :100].mean() == pytest.approx(-20.0, abs=0.3)  # the shelf (ridged field: sigma 1 m)
    assert b.max() > 0.0  # dry land behind the shoreline at 0.85 Lx
    crest = b[128 - 3:128 + 3, 512 - 3:512 + 3].mean()
    assert -3.0 < crest < 1.0  # the shoal's crest at 1 m depth, give or take the ridged field
    assert w.maker.angle == pytest.approx(np.radians(10.0))  # walls: the drawn angle as is


def test_config5_bed_is_the_reef_bed_at_its_size():
    grid = Grid(256, 256, 1.0, 1.0)
    a = W.reef_bed(grid, 7, 0.85 * 256, 128.0, 128.0)
    b = W.reef_bed(grid, 7, 0.85 * 256, 128.0, 128.0)
    assert np.array_equal(a, b)  # seeded
    assert not np.array_equal(a, W.reef_bed(grid, 8, 0.85 * 256, 128.0, 128.0))


def test_harvest_refuses_an_unknown_family():
    from wavesim_b200.train_lpc import harvest_runs

    with pytest.raises(ValueError):
        harvest_runs(None, family="lagoon")
