"""wc_stable_dt_noalloc, the entry point for callers that cannot have the library allocate.

Some host applications give all of the GPU's memory to their own pool allocator at start-up, and
some simulation loops must not allocate or free per step (cudaFree synchronises the device); such
callers keep the state in their own device arrays and need the time step without the library
allocating anything. This checks that the no-allocation variant returns the same bits as
wc_stable_dt on the same state, on two calls in a row (the second call reuses the scratch the
first one left behind), on a small grid and on one large enough that the partial pass's capped
grid runs several cells per thread, and that it refuses a grid larger than its fixed scratch
serves. The file is named to be collected last.
"""
import math

import numpy as np
import pytest

from wavesim_b200 import Bathymetry, Grid, Solver, State, WavecoreError
from wavesim_b200.solver import stable_dt_noalloc

pytestmark = pytest.mark.gpu


def _wavy_state(grid, bed, seed):
    rng = np.random.default_rng(seed)
    s = State.lake_at_rest(grid, bed, 0.0)
    X, Y = grid.centres()
    grid.inner(s.h)[:] += 0.4 * np.exp(-((X - 60.0) ** 2 + (Y - 30.0) ** 2) / 200.0)
    grid.inner(s.hu)[:] = rng.uniform(-1.0, 1.0, X.shape) * grid.inner(s.h)
    grid.inner(s.hv)[:] = rng.uniform(-0.5, 0.5, X.shape) * grid.inner(s.h)
    s.fill_boundaries(grid, False)
    return s


@pytest.mark.parametrize("nx,ny", [(150, 70), (2048, 1024)])
def test_noalloc_stable_dt_matches_wc_stable_dt_on_two_calls_in_a_row(nx, ny):
    import torch

    grid = Grid(nx, ny, 2.0, 1.5)
    bed = Bathymetry.rough(grid, 3.0, 1.0)
    solver = Solver(grid, bed)
    for seed in (1, 2):
        s = _wavy_state(grid, bed, seed)
        expected = solver.stable_dt(s)
        assert math.isfinite(expected) and expected > 0.0
        d = [torch.from_numpy(a.copy()).cuda() for a in (s.h, s.hu, s.hv)]
        torch.cuda.synchronize()
        for _ in range(2):
            got = stable_dt_noalloc(grid, solver.cfl, *(t.data_ptr() for t in d))
            # The same FP64 operations cell by cell and a max, which does not depend on order:
            # the same bits.
            assert got == expected, (got, expected)
        del d


def test_noalloc_stable_dt_reports_nan_like_wc_stable_dt():
    import torch

    grid = Grid(40, 20, 1.0, 1.0)
    bed = Bathymetry.flat(grid, 2.0)
    s = State.lake_at_rest(grid, bed, 0.0)
    s.hu[grid.idx(10, 8)] = float("nan")
    solver = Solver(grid, bed)
    assert math.isnan(solver.stable_dt(s))
    d = [torch.from_numpy(a.copy()).cuda() for a in (s.h, s.hu, s.hv)]
    torch.cuda.synchronize()
    assert math.isnan(stable_dt_noalloc(grid, solver.cfl, *(t.data_ptr() for t in d)))


def test_noalloc_stable_dt_refuses_a_grid_beyond_its_scratch():
    import torch

    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    big = Grid(4097, 4096, 1.0, 1.0)  # refused before any device access
    with pytest.raises(WavecoreError) as e:
        stable_dt_noalloc(big, 0.4, small.data_ptr(), small.data_ptr(), small.data_ptr())
    assert e.value.status == 1 and "16777216" in str(e.value)
