"""One-way nesting on the device against its FP64 restatement run on two oracle solvers
(same inputs, same step sizes). Tolerance: FP32 against FP64, 5e-5 m on the fine surface."""
import numpy as np
import pytest

from oracle.nest_oracle import Nest as OracleNest
from oracle.oracle import OracleSolver
from wavesim_b200 import Bathymetry, Grid, Nest, Order, Solver, Sponge, State, WaveMaker

pytestmark = pytest.mark.gpu


def runs():
    # a coarse 6 m run with the wave-maker; a 3 m fine grid starting 300 m into it, with a
    # relaxation zone along its offshore edge
    cgrid = Grid(120, 24, 6.0, 6.0)
    fgrid = Grid(160, 40, 3.0, 3.0)
    x0 = 300.0
    bc = Bathymetry.plane_beach(cgrid, 1.0 / 40.0, 12.0)
    Xf, _ = fgrid.centres()
    bf_int = np.maximum(-12.0, (x0 + Xf - 12.0 * 40.0) / 40.0)
    bf = Bathymetry.from_interior(fgrid, bf_int)

    def coarse(cls):
        return (cls(cgrid, bc).with_order(Order.Second).with_manning(0.02)
                .with_sponge(Sponge(5, 1.5).edges(True, False, False, False))
                .with_wavemaker(WaveMaker(x=60.0, amplitude=0.5, period=10.0, angle=0.0, sigma=12.0, ramp_periods=1.0)))

    def fine(cls):
        return cls(fgrid, bf).with_order(Order.Second).with_manning(0.02)

    zones = [Sponge(20, 2.0).edges(True, False, False, False)]
    return cgrid, fgrid, bc, bf, x0, coarse, fine, zones


def test_nested_fine_run_matches_the_restated_driver():
    cgrid, fgrid, bc, bf, x0, coarse, fine, zones = runs()
    sc = State.lake_at_rest(cgrid, bc, 0.0)
    sf = State.lake_at_rest(fgrid, bf, 0.0)
    fine_dt, coarse_dt, steps = 0.12, 0.25, 450
    # FP64: two oracle solvers and the restated nesting
    oc, of = coarse(OracleSolver), fine(OracleSolver)
    on = OracleNest(fgrid, cgrid, zones, x0, 0.0)
    c64, f64 = sc.clone(), sf.clone()
    frm = to = None
    t0 = t1 = 0.0
    for _ in range(steps):
        end = f64.time + fine_dt
        stepped = False
        while c64.time < end - 1e-9:
            before = c64.clone()
            oc.step(c64, coarse_dt)
            stepped = True
        if stepped:
            # lib.rs:1860-1872: both states' ghosts filled as walls before sampling
            t0, frm = before.time, on.sample(before, bc.b)
            t1, to = c64.time, on.sample(c64, bc.b)
        of.step(f64, fine_dt)
        on.apply(f64, bf.b, fine_dt, t0, frm, t1, to, f64.time)
    # device
    gc, gf = coarse(Solver), fine(Solver)
    gc.upload(sc)
    gf.upload(sf)
    nest = Nest(gf, gc, zones, x0, 0.0)
    assert nest.cells == len(on.cells) > 0
    nest.run([fine_dt] * steps, lambda t: coarse_dt)
    gf.synchronize()
    out = sf.clone()
    gf.download(out)
    hg, ho = fgrid.inner(out.h), fgrid.inner(f64.h)
    assert abs(out.time - f64.time) < 1e-9
    assert np.max(np.abs(ho)) > 0 and np.max(np.abs(fgrid.inner(f64.hu))) > 0.05  # waves came in
    d = np.abs(hg - ho)
    j, i = np.unravel_index(np.argmax(d), d.shape)
    print("max", d.max(), "at", (i, j), "h", hg[j, i], ho[j, i], "bed", fgrid.inner(bf.b)[j, i],
          "zone max", d[:, :25].max(), "wet-both max", d[(hg > 1e-3) & (ho > 1e-3)].max())
    assert np.max(np.abs(hg - ho)) < 5e-5
    assert np.max(np.abs(fgrid.inner(out.hu) - fgrid.inner(f64.hu))) < 1e-2  # momentum, FP32 vs FP64 after 54 s
