"""Followed breaking fronts and their eddy viscosity (crates/wavecore/src/eddy.rs) on the device
against the FP64 oracle, through the C ABI.

The fronts and their memory are FP64 arithmetic on both sides: on a state whose values are FP32
numbers (so both engines start from the same bits), one application of `follow_breaking`
(solver.rs:509-532) must give the same memory bit for bit and the same number of viscous
sub-steps; the momentum it diffuses is FP32 on the device, so it agrees to FP32 rounding. Over
whole steps the FP32 state drifts from the FP64 one as it does without fronts; the fronts must
still agree on all but a few cells at their edges.
"""
import math

import numpy as np
import pytest

from oracle.oracle import OracleSolver
from wavesim_b200 import Bathymetry, Breaking, Dispersion, EddyViscosity, Ensemble, Grid, Order, Solver, State
from wavesim_b200.model import GHOST
from wavesim_b200.solver import WavecoreError

pytestmark = pytest.mark.gpu


def eddy_dispersion(**kw):
    return Dispersion(breaking=Breaking(viscosity=EddyViscosity(**kw)), tolerance=1e-8)


def dam_break(grid, up=2.0, x0=5.0):
    """A flat bed 1 m deep with `up` metres more water west of x0: the bore it sends east keeps
    breaking by Kennedy's criterion."""
    bed = Bathymetry.flat(grid, 1.0)
    s = State.lake_at_rest(grid, bed, 0.0)
    for i, j in grid.interior():
        if (i - GHOST + 0.5) * grid.dx < x0:
            s.h[grid.idx(i, j)] += up
    s.fill_walls(grid)
    return bed, s


def pair(grid, bed, periodic=False, **kw):
    def make(cls):
        s = cls(grid, bed).with_order(Order.Fifth).with_dispersion(eddy_dispersion(**kw))
        return s.with_periodic_y() if periodic else s
    return make(Solver), make(OracleSolver)


def to_fp32(s: State) -> State:
    r = s.clone()
    for a in (r.h, r.hu, r.hv):
        a[:] = a.astype(np.float32).astype(np.float64)
    return r


def developed(grid, periodic, steps=30):
    """An oracle run of the dam break with followed fronts: a state with fronts, lingering cells
    and nonzero viscosity, its values rounded to FP32."""
    bed, s = dam_break(grid)
    # a ragged front along y, so that both directions and the cross terms take part
    for i, j in grid.interior():
        x = (i - GHOST + 0.5) * grid.dx
        if 5.0 <= x < 5.0 + 0.75 * (1 + math.sin(2 * math.pi * (j - GHOST) / grid.ny)):
            s.h[grid.idx(i, j)] += 2.0
    _, orc = pair(grid, bed, periodic)
    for _ in range(steps):
        orc.step(s, orc.stable_dt(s))
    return bed, to_fp32(s)


@pytest.mark.parametrize("periodic", [False, True])
def test_one_application_matches_the_oracle_bit_for_bit_in_the_memory(periodic):
    grid = Grid(96, 24, 0.25, 0.25)
    bed, s = developed(grid, periodic)
    gpu, orc = pair(grid, bed, periodic)
    mem0 = grid.inner(s.breaking)
    assert (mem0 > 0).any() and (mem0 < 0).any(), "the state has no fronts or no lingering cells"
    a, b = s.clone(), s.clone()
    dt = orc.stable_dt(s)
    ng = gpu.follow_breaking(a, dt)
    no = orc.follow_breaking(b, dt)
    assert ng == no and no >= 1
    ma, mb = grid.inner(a.breaking), grid.inner(b.breaking)
    assert np.array_equal(ma, mb), f"{int((ma != mb).sum())} cells differ"
    for x, y in ((a.hu, b.hu), (a.hv, b.hv)):
        d = np.abs(grid.inner(x) - grid.inner(y)).max()
        assert d <= 2e-6 * (1.0 + np.abs(grid.inner(y)).max()), d
    assert np.array_equal(grid.inner(a.h), grid.inner(b.h))
    # the viscosity changed the momentum
    assert np.abs(grid.inner(b.hu) - grid.inner(s.hu)).max() > 1e-4


def test_the_indicator_reads_breaking_wherever_the_memory_holds_a_front():
    grid = Grid(96, 24, 0.25, 0.25)
    bed, s = developed(grid, False)
    gpu, orc = pair(grid, bed)
    ig = gpu.breaking_indicator(s).reshape(grid.ny, grid.nx)
    io = orc.breaking_indicator(s).reshape(grid.ny, grid.nx)
    held = (grid.inner(s.breaking) != 0.0) & (grid.inner(s.h) >= 0.05)
    assert held.any() and np.all(ig[held] == 1.0) and np.all(io[held] == 1.0)
    assert np.mean((ig >= 0.8) == (io >= 0.8)) > 0.999


def test_steps_with_followed_fronts_track_the_oracle():
    grid = Grid(128, 32, 0.25, 0.25)
    bed, s0 = dam_break(grid)
    gpu, orc = pair(grid, bed)
    sg, so = s0.clone(), s0.clone()
    for _ in range(60):
        dt = orc.stable_dt(so)
        orc.step(so, dt)
        gpu.step(sg, dt)
    eg, eo = grid.inner(sg.h), grid.inner(so.h)
    d = np.abs(eg - eo)
    mg, mo = grid.inner(sg.breaking), grid.inner(so.breaking)
    agree = float(np.mean(np.sign(mg) == np.sign(mo)))
    both = (mg > 0) & (mo > 0)
    print("eta max diff", d.max(), "rms", np.sqrt(np.mean(d * d)), "front-class agreement", agree,
          "front cells", int((mo > 0).sum()), "lingering", int((mo < 0).sum()))
    assert (mo > 0).sum() >= 10 and (mo < 0).sum() >= 10
    assert agree > 0.99
    assert np.abs(mg[both] - mo[both]).max() < 1e-6
    assert d.max() < 2e-3 and np.sqrt(np.mean(d * d)) < 1e-4
    assert abs(sg.volume(grid) - so.volume(grid)) < 1e-6 * so.volume(grid)


def test_still_water_with_followed_fronts_stays_still_on_the_device():
    grid = Grid(64, 32, 1.0, 1.0)
    bed = Bathymetry.plane_beach(grid, 0.05, 2.0)
    bed.b[:] = bed.b.astype(np.float32).astype(np.float64)
    sol = Solver(grid, bed).with_order(Order.Fifth).with_dispersion(eddy_dispersion())
    s = State.lake_at_rest(grid, bed, 0.0)
    h0 = grid.inner(s.h).copy()
    sol.upload(s)
    sol.step_n(20, 5.0)
    sol.synchronize()
    out = s.clone()
    sol.download(out)
    assert np.array_equal(grid.inner(out.h), h0)
    assert np.all(grid.inner(out.hu) == 0.0) and np.all(grid.inner(out.hv) == 0.0)
    assert np.all(out.breaking == 0.0)


def test_the_captured_step_equals_the_launched_one():
    """Device-resident steps replay a captured graph holding the cooperative eddy launch; with
    per-kernel timing on, the same kernels are launched one by one. Both give the same bits."""
    grid = Grid(96, 24, 0.25, 0.25)
    bed, s = developed(grid, False, steps=10)
    a, b = s.clone(), s.clone()
    runs = []
    for profile, st in ((False, a), (True, b)):
        sol, _ = pair(grid, bed)
        sol.upload(st)
        if profile:
            sol.profile(True)
        for _ in range(15):
            sol.step_device(0.004)
        sol.synchronize()
        sol.download(st)
        runs.append(sol.profile_read() if profile else None)
    for x, y in ((a.h, b.h), (a.hu, b.hu), (a.hv, b.hv), (a.breaking, b.breaking)):
        assert np.array_equal(grid.inner(x), grid.inner(y))
    assert runs[1]["eddy"][0] == 15


def test_an_ensemble_does_not_take_followed_fronts():
    grid = Grid(64, 32, 1.0, 1.0)
    bed = Bathymetry.flat(grid, 2.0)
    m = Solver(grid, bed).with_dispersion(eddy_dispersion())
    with pytest.raises(WavecoreError):
        Ensemble([m])


def test_frames_and_the_recorder_read_the_memory():
    """With followed fronts the driver's frame and its per-step breaking statistics read a cell
    whose memory holds a front as breaking (dispersion.rs:149-152 through breaking_into): the
    device recorder against the FP64 restatement of Stage::record fed with the oracle's states and
    breaking indicators (memory included), same inputs and dt."""
    from oracle.record_oracle import Recorder as OracleRecorder
    from wavesim_b200 import Recorder

    grid = Grid(128, 32, 0.25, 0.25)
    bed, s0 = dam_break(grid)
    gpu, orc = pair(grid, bed)
    rec = Recorder(gpu, 0.0, 1.0)
    ref = OracleRecorder(grid.nx * grid.ny, 0.0, 0.0, 1.0)
    sg, so = s0.clone(), s0.clone()
    b = grid.inner(bed.b)
    for _ in range(40):
        dt = orc.stable_dt(so)
        orc.step(so, dt)
        gpu.step(sg, dt)
        ref.record(so.time, dt, (grid.inner(so.h) + b).ravel(), orc.breaking_indicator(so).ravel())
    frac, frac_o = rec.read()["breaking_fraction"].ravel(), ref.breaking_fraction()
    assert frac_o.max() > 0.9, "nothing broke"
    assert np.mean(np.abs(frac - frac_o) < 0.05) > 0.99
    # the frame of the resident state: breaking wherever the memory holds a front
    gpu.upload(sg)
    gpu_state = sg.clone()
    _, brk, _ = gpu.frame(0.0)
    mem, h = grid.inner(gpu_state.breaking), grid.inner(gpu_state.h)
    held = (mem != 0.0) & (h >= 0.05)
    assert held.sum() >= 10 and np.all(brk[held] == 1.0)
    rec.close()
