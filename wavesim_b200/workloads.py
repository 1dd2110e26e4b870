"""Seeded synthetic workloads of the benchmark configurations.

The reference benchmarks nothing on a public suite; these inputs have the configurations' shapes
(grid, cell size, bed family, wave-maker) and are fed bit-identically to the device build and
to the FP64 oracle. Every random draw takes an explicit seed.

Beds: a 1:30 plane beach behind a flat 20 m shelf plus a Gaussian random field
(white noise filtered by exp(-|k|^2 l^2 / 4), i.e. convolved with exp(-r^2/l^2), scaled to the
requested standard deviation; periodic in both directions, so it suits a periodic-y domain);
config 5's reef adds a Gaussian shoal whose crest is 1 m deep and takes a ridged field instead
(`reef_bed`, also the bed of the smaller reef runs the learned preconditioner's training harvests).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .model import Bathymetry, Dispersion, Grid, Order, Sponge, State, WaveMaker, linear_wave


def gaussian_field(nx: int, ny: int, dx: float, dy: float, sigma: float, corr: float, seed: int) -> np.ndarray:
    """A (ny, nx) zero-mean Gaussian random field of standard deviation `sigma` and correlation
    length `corr` metres."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((ny, nx))
    kx = 2.0 * np.pi * np.fft.fftfreq(nx, d=dx)
    ky = 2.0 * np.pi * np.fft.fftfreq(ny, d=dy)
    KX, KY = np.meshgrid(kx, ky)
    filt = np.exp(-(KX**2 + KY**2) * corr * corr / 4.0)
    f = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    f -= f.mean()
    std = f.std()
    return f * (sigma / std) if std > 0 else f


def ridged_field(nx: int, ny: int, dx: float, dy: float, sigma: float, corr: float, seed: int) -> np.ndarray:
    """A ridged (reef-like) field: sigma * (1 - 2|g|) of a unit Gaussian field g, re-centred."""
    g = gaussian_field(nx, ny, dx, dy, 1.0, corr, seed)
    r = 1.0 - 2.0 * np.abs(g)
    r -= r.mean()
    return r * (sigma / r.std())


def shelf_and_beach(grid: Grid, shelf_depth: float, slope: float, shore_x: float) -> np.ndarray:
    """(ny, nx) bed: flat at -shelf_depth, rising at `slope` to still water at x = shore_x."""
    X, _ = grid.centres()
    return np.maximum(-shelf_depth, slope * (X - shore_x))


def snapped_angle(omega: float, depth: float, ly: float, target: float, dispersive: bool):
    """The angle nearest `target` whose alongshore wavenumber fits a periodic domain of length
    ly (k sin(angle) ly = 2 pi n; crates/wavecore/src/solver.rs:421-429). Returns (angle, n)."""
    k = linear_wave(omega, depth, dispersive).k
    best = None
    n = 0
    while True:
        s = 2.0 * math.pi * n / (k * ly)
        if s > 1.0:
            break
        a = math.asin(s)
        if best is None or abs(a - target) < abs(best[0] - target):
            best = (a, n)
        n += 1
    return best


@dataclass
class Workload:
    name: str
    grid: Grid
    bed: Bathymetry
    order: Order
    cfl: float
    manning: float
    periodic_y: bool
    sponges: list
    maker: WaveMaker
    dispersion: Dispersion | None
    steps: int
    meta: dict = field(default_factory=dict)

    def solver(self, cls):
        s = cls(self.grid, self.bed).with_order(self.order).with_manning(self.manning)
        s.cfl = self.cfl
        for sp in self.sponges:
            s = s.with_sponge(sp)
        if self.dispersion is not None:
            s = s.with_dispersion(self.dispersion)
        s = s.with_wavemaker(self.maker)
        if self.periodic_y:
            s = s.with_periodic_y()
        return s

    def interior_cells(self) -> int:
        return self.grid.nx * self.grid.ny


def config1() -> Workload:
    """Plane beach 256x64 at 3 m, 1:30 from 20 m to a dry shore; MC + HLL, SSP-RK2, CFL 0.45,
    no dispersion; maker H=1 m, T=12 s, normal incidence at x=90 m (sigma 2 cells, ramp 4
    periods); 50 m (17-cell) sponges at both x ends at 1.5 /s; Manning 0.02; walls; 2000 steps."""
    grid = Grid(256, 64, 3.0, 3.0)
    bed = Bathymetry.plane_beach(grid, 1.0 / 30.0, 20.0)
    return Workload(
        name="swe_plane_beach_256x64_dx3",
        grid=grid,
        bed=bed,
        order=Order.Second,
        cfl=0.45,
        manning=0.02,
        periodic_y=False,
        sponges=[Sponge(17, 1.5).edges(True, True, False, False)],
        maker=WaveMaker(x=90.0, amplitude=0.5, period=12.0, angle=0.0, sigma=6.0, ramp_periods=4.0),
        dispersion=None,
        steps=2000,
    )


def sgn_beach(nx: int, ny: int, dx: float, seed: int, tolerance: float = 1e-8, height: float = 2.0,
              period: float = 14.0, angle_deg: float = 15.0, sigma_bed: float = 0.5, corr: float = 20.0,
              name: str | None = None, steps: int = 5000, preconditioner: int = 0, periodic: bool = True) -> Workload:
    """Fifth order + SGN by PCG, periodic in y: a 20 m shelf, then a 1:30 beach whose still-water
    shoreline is at 0.85 Lx, plus a Gaussian random field; maker H, T at x = 160 m (0.15 Lx on
    small grids) in ~20 m,
    oblique at the angle nearest `angle_deg` that fits the periodic width; a 100 m sponge at the
    offshore edge; Manning 0.02; CFL 0.4. With `periodic=False` the y ends are walls and the maker
    takes `angle_deg` itself (an oblique maker needs no fit between walls)."""
    grid = Grid(nx, ny, dx, dx)
    lx, ly = nx * dx, ny * dx
    base = shelf_and_beach(grid, 20.0, 1.0 / 30.0, 0.85 * lx)
    b = base + gaussian_field(nx, ny, dx, dx, sigma_bed, corr, seed)
    bed = Bathymetry.from_interior(grid, b)
    maker_x = min(160.0, 0.15 * lx)
    i_m = min(max(int(round(maker_x / dx - 0.5)), 0), nx - 1)
    depth = -b[ny // 2, i_m]
    omega = 2.0 * math.pi / period
    if periodic:
        angle, turns = snapped_angle(omega, depth, ly, math.radians(angle_deg), True)
    else:
        angle, turns = math.radians(angle_deg), None
    maker = WaveMaker(x=maker_x, amplitude=height / 2.0, period=period, angle=angle, sigma=2.0 * dx, ramp_periods=4.0)
    return Workload(
        name=name or f"sgn_beach_{nx}x{ny}_dx{dx:g}",
        grid=grid,
        bed=bed,
        order=Order.Fifth,
        cfl=0.4,
        manning=0.02,
        periodic_y=periodic,
        sponges=[Sponge(int(round(100.0 / dx)), 1.5).edges(True, False, False, False)],
        maker=maker,
        dispersion=Dispersion(tolerance=tolerance, max_iterations=1000, preconditioner=preconditioner),
        steps=steps,
        meta={"seed": seed, "maker_depth_m": depth, "angle_deg": math.degrees(angle), "alongshore_turns": turns,
              "bed": f"20 m shelf + 1:30 beach (shore at 0.85 Lx) + Gaussian field sigma {sigma_bed} m, corr {corr} m"},
    )


def swe_beach(nx: int, ny: int, dx: float, seed: int, name: str | None = None, steps: int = 2000) -> Workload:
    """The non-dispersive stencil at scale: the beach of `sgn_beach` (20 m shelf, 1:30 beach,
    Gaussian field sigma 0.5 m / 20 m, periodic y) with the plain method of the first
    configuration: second order (MUSCL-MC + HLL), SSP-RK2, CFL 0.45, no dispersion, Manning 0.02;
    maker H = 1 m, T = 12 s at normal incidence; a 100 m offshore sponge."""
    grid = Grid(nx, ny, dx, dx)
    lx = nx * dx
    b = shelf_and_beach(grid, 20.0, 1.0 / 30.0, 0.85 * lx) + gaussian_field(nx, ny, dx, dx, 0.5, 20.0, seed)
    bed = Bathymetry.from_interior(grid, b)
    maker_x = min(160.0, 0.15 * lx)
    return Workload(
        name=name or f"swe_beach_{nx}x{ny}_dx{dx:g}",
        grid=grid, bed=bed, order=Order.Second, cfl=0.45, manning=0.02, periodic_y=True,
        sponges=[Sponge(int(round(100.0 / dx)), 1.5).edges(True, False, False, False)],
        maker=WaveMaker(x=maker_x, amplitude=0.5, period=12.0, angle=0.0, sigma=2.0 * dx, ramp_periods=4.0),
        dispersion=None, steps=steps,
        meta={"seed": seed, "bed": "20 m shelf + 1:30 beach (shore at 0.85 Lx) + Gaussian field sigma 0.5 m, corr 20 m"},
    )


def swe_large(seed: int = 7) -> Workload:
    """4096 x 4096 at 2 m of the non-dispersive stencil (16.8 M cells, the size of the largest
    configuration)."""
    return swe_beach(4096, 4096, 2.0, seed, name="swe_beach_4096x4096_dx2")


def reef_bed(grid: Grid, seed: int, shore_x: float, shoal_x: float, shoal_y: float, shoal_radius: float = 150.0,
             sigma: float = 1.0, corr: float = 10.0) -> np.ndarray:
    """(ny, nx) reef-like bed: a 20 m shelf and a 1:30 beach with its still-water shoreline at
    shore_x, a Gaussian shoal centred at (shoal_x, shoal_y) whose crest is 1 m deep (the beach is
    kept where it is shallower), plus a ridged random field (sigma, correlation length)."""
    X, Y = grid.centres()
    base = shelf_and_beach(grid, 20.0, 1.0 / 30.0, shore_x)
    base_at_shoal = float(np.maximum(-20.0, (shoal_x - shore_x) / 30.0))
    shoal = (-1.0 - base_at_shoal) * np.exp(-((X - shoal_x) ** 2 + (Y - shoal_y) ** 2) / (shoal_radius**2))
    return np.maximum(base + shoal, np.minimum(base, -1.0)) + ridged_field(grid.nx, grid.ny, grid.dx, grid.dy,
                                                                          sigma, corr, seed)


def config5(seed: int = 2026, preconditioner: int = 0) -> Workload:
    """4096 x 4096 at 1 m: a 1:30 plane beach behind a 20 m shelf plus a ridged random field
    (sigma 1 m, correlation 10 m) and a Gaussian shoal (radius 150 m) whose crest is 1 m deep;
    fifth order + SGN to 1e-8 with the breaking switch; maker H = 3 m, T = 16 s at the angle
    nearest 10 degrees that fits the periodic width; 10000 steps."""
    nx = ny = 4096
    dx = 1.0
    grid = Grid(nx, ny, dx, dx)
    lx, ly = nx * dx, ny * dx
    b = reef_bed(grid, seed, 0.85 * lx, 0.5 * lx, 0.5 * ly)
    bed = Bathymetry.from_interior(grid, b)
    maker_x = 160.0
    i_m = int(round(maker_x / dx - 0.5))
    depth = -b[ny // 2, i_m]
    omega = 2.0 * math.pi / 16.0
    angle, turns = snapped_angle(omega, depth, ly, math.radians(10.0), True)
    maker = WaveMaker(x=maker_x, amplitude=1.5, period=16.0, angle=angle, sigma=2.0 * dx, ramp_periods=4.0)
    return Workload(
        name="sgn_reef_4096x4096_dx1", grid=grid, bed=bed, order=Order.Fifth, cfl=0.4, manning=0.02,
        periodic_y=True, sponges=[Sponge(100, 1.5).edges(True, False, False, False)], maker=maker,
        dispersion=Dispersion(tolerance=1e-8, max_iterations=1000, preconditioner=preconditioner), steps=10000,
        meta={"seed": seed, "maker_depth_m": depth, "angle_deg": math.degrees(angle), "alongshore_turns": turns,
              "bed": "20 m shelf + 1:30 beach + ridged field sigma 1 m / 10 m + shoal to 1 m depth"},
    )


def sgn_reef(nx: int, ny: int, dx: float, seed: int, height: float = 3.0, period: float = 16.0,
             angle_deg: float = 10.0, name: str | None = None, steps: int = 1000) -> Workload:
    """A smaller run of config 5's family between walls: the reef bed (20 m shelf, 1:30 beach with
    its shoreline at 0.85 Lx, a shoal to 1 m depth at mid-width, a ridged field sigma 1 m /
    10 m), fifth order + SGN to 1e-8, a maker of height H and period T at x = 160 m taking
    `angle_deg` itself, a 100 m offshore sponge, Manning 0.02, CFL 0.4."""
    grid = Grid(nx, ny, dx, dx)
    lx, ly = nx * dx, ny * dx
    b = reef_bed(grid, seed, 0.85 * lx, 0.5 * lx, 0.5 * ly)
    bed = Bathymetry.from_interior(grid, b)
    maker_x = min(160.0, 0.15 * lx)
    i_m = min(max(int(round(maker_x / dx - 0.5)), 0), nx - 1)
    maker = WaveMaker(x=maker_x, amplitude=height / 2.0, period=period, angle=math.radians(angle_deg),
                      sigma=2.0 * dx, ramp_periods=4.0)
    return Workload(
        name=name or f"sgn_reef_{nx}x{ny}_dx{dx:g}", grid=grid, bed=bed, order=Order.Fifth, cfl=0.4, manning=0.02,
        periodic_y=False, sponges=[Sponge(int(round(100.0 / dx)), 1.5).edges(True, False, False, False)],
        maker=maker, dispersion=Dispersion(tolerance=1e-8, max_iterations=1000), steps=steps,
        meta={"seed": seed, "maker_depth_m": -b[ny // 2, i_m], "angle_deg": angle_deg,
              "bed": "20 m shelf + 1:30 beach + ridged field sigma 1 m / 10 m + shoal to 1 m depth"},
    )


def config2(seed: int = 2024) -> Workload:
    """1024x512 at 2 m, fifth order + SGN by Jacobi PCG to 1e-8, periodic y, H=2 m, T=14 s."""
    return sgn_beach(1024, 512, 2.0, seed, name="sgn_beach_1024x512_dx2")


def config3(seed: int = 2025) -> Workload:
    """2048x1024 at 2 m, same physics as config2."""
    return sgn_beach(2048, 1024, 2.0, seed, name="sgn_beach_2048x1024_dx2")


def config4(seed: int = 4, members: int = 64, preconditioner: int = 0):
    """64 runs of uneven grids (nx 512-2048, ny 256-1024, dx 2-3 m) on seeded rough plane beaches
    (20 m shelf, 1:30 beach, Gaussian field sigma 0.5 m / 20 m), reflective y walls; per run the
    swell angle ~ U(-20, 20) deg, T ~ U(8, 18) s, H ~ U(0.5, 4) m and a still-water offset
    ~ U(-1, 1) m applied as a bed shift (as the reference's Bed::bathymetry(tide) does,
    crates/waveio/src/bed.rs:239-246); fifth order + SGN to 1e-8."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(members):
        nx = int(rng.integers(512 // 64, 2048 // 64 + 1)) * 64
        ny = int(rng.integers(256 // 32, 1024 // 32 + 1)) * 32
        dx = float(rng.uniform(2.0, 3.0))
        angle = math.radians(float(rng.uniform(-20.0, 20.0)))
        period = float(rng.uniform(8.0, 18.0))
        height = float(rng.uniform(0.5, 4.0))
        tide = float(rng.uniform(-1.0, 1.0))
        grid = Grid(nx, ny, dx, dx)
        lx = nx * dx
        b = shelf_and_beach(grid, 20.0, 1.0 / 30.0, 0.85 * lx) + gaussian_field(nx, ny, dx, dx, 0.5, 20.0, seed * 1000 + m)
        b = b - tide
        bed = Bathymetry.from_interior(grid, b)
        maker = WaveMaker(x=160.0, amplitude=height / 2.0, period=period, angle=angle, sigma=2.0 * dx, ramp_periods=4.0)
        out.append(Workload(
            name=f"ensemble_member_{m}_{nx}x{ny}",
            grid=grid, bed=bed, order=Order.Fifth, cfl=0.4, manning=0.02, periodic_y=False,
            sponges=[Sponge(int(round(100.0 / dx)), 1.5).edges(True, False, False, False)],
            maker=maker,
            dispersion=Dispersion(tolerance=1e-8, max_iterations=1000, preconditioner=preconditioner),
            steps=3000,
            meta={"dx": dx, "angle_deg": math.degrees(angle), "period": period, "height": height, "tide": tide},
        ))
    return out


def wave_train_state(w: Workload, x_from: float | None = None, x_to: float | None = None) -> State:
    """A start that already holds the swell: still water plus a linear wave train of the maker's
    amplitude, direction and (offshore) wavenumber over the shelf, tapered to zero at both ends,
    with the linear velocity u = (omega/k) eta / h along the direction of travel; the clock
    starts at the end of the maker's ramp. Both the device build and the oracle start from it."""
    grid, bed, m = w.grid, w.bed, w.maker
    s = State.lake_at_rest(grid, bed, 0.0)
    X, Y = grid.centres()
    depth0 = max(1.0, float(-np.median(grid.inner(bed.b)[:, : max(1, grid.nx // 8)])))
    omega = 2.0 * math.pi / m.period
    lw = linear_wave(omega, depth0, w.dispersion is not None)
    kx, ky = lw.k * math.cos(m.angle), lw.k * math.sin(m.angle)
    x_from = m.x + 2.0 * m.sigma if x_from is None else x_from
    x_to = 0.6 * grid.nx * grid.dx if x_to is None else x_to
    width = max(1.0, 0.25 * (x_to - x_from))
    taper = np.clip((X - x_from) / width, 0.0, 1.0) * np.clip((x_to - X) / width, 0.0, 1.0)
    taper = taper * taper * (3.0 - 2.0 * taper)
    eta = m.amplitude * taper * np.cos(kx * X + ky * Y)
    b = grid.inner(bed.b)
    h = np.maximum(eta - b, 0.0)
    wet = h > 0.05
    un = np.where(wet, lw.phase_speed * eta / np.maximum(h, 0.05), 0.0)
    grid.inner(s.h)[:] = h
    grid.inner(s.hu)[:] = h * un * math.cos(m.angle)
    grid.inner(s.hv)[:] = h * un * math.sin(m.angle)
    s.fill_boundaries(grid, w.periodic_y)
    s.time = m.ramp_periods * m.period
    return s
