"""Host-side data types of wavecore, mirrored in Python over numpy.

These restate the reference's plain data and host helpers so that callers and tests read like
the reference's own (`Grid::new`, `Bathymetry::plane_beach`, `State::lake_at_rest`, the
`Sponge`/`WaveMaker`/`Dispersion` builders). None of them advances the water: stepping happens
only in the device library behind `wavesim_b200.solver.Solver`.

References are to mlaegn/wavesim, `crates/wavecore/src/`.
"""
from __future__ import annotations

import copy
import enum
import math
from dataclasses import dataclass, field, replace
from typing import Callable, Optional

import numpy as np

from . import abi

GHOST = abi.GHOST
G = 9.81  # solver.rs:26
H_DRY = 1e-8  # solver.rs:28


class Order(enum.IntEnum):
    """solver.rs:34-50."""

    First = 0
    Second = 1
    Fifth = 2


@dataclass(frozen=True)
class Grid:
    """grid.rs:12-57: a uniform grid with GHOST ghost layers on every side."""

    nx: int
    ny: int
    dx: float
    dy: float

    def __post_init__(self):
        if not (self.nx > 0 and self.ny > 0):
            raise ValueError("grid must have at least one interior cell")
        if not (self.dx > 0.0 and self.dy > 0.0):
            raise ValueError("cell size must be positive")

    def width(self) -> int:
        return self.nx + 2 * GHOST

    def rows(self) -> int:
        return self.ny + 2 * GHOST

    def cells(self) -> int:
        return self.width() * self.rows()

    def idx(self, i: int, j: int) -> int:
        return j * self.width() + i

    def interior(self):
        for j in range(GHOST, GHOST + self.ny):
            for i in range(GHOST, GHOST + self.nx):
                yield i, j

    def centre(self, i: int, j: int):
        return ((i - GHOST) + 0.5) * self.dx, ((j - GHOST) + 0.5) * self.dy

    def centres(self):
        """Interior cell centres as (ny, nx) arrays X, Y."""
        x = (np.arange(self.nx) + 0.5) * self.dx
        y = (np.arange(self.ny) + 0.5) * self.dy
        return np.meshgrid(x, y)

    def to_c(self) -> abi.wc_grid:
        return abi.wc_grid(self.nx, self.ny, float(self.dx), float(self.dy))

    def view(self, a: np.ndarray) -> np.ndarray:
        """A padded flat array as (rows, width)."""
        return a.reshape(self.rows(), self.width())

    def inner(self, a: np.ndarray) -> np.ndarray:
        """The interior of a padded flat array as (ny, nx)."""
        return self.view(a)[GHOST : GHOST + self.ny, GHOST : GHOST + self.nx]


def mirror_ghosts(grid: Grid, a: np.ndarray) -> None:
    """grid.rs:60-75, in place on a padded flat array."""
    v = grid.view(a)
    nx, ny = grid.nx, grid.ny
    for k in range(GHOST):
        v[GHOST : GHOST + ny, GHOST - 1 - k] = v[GHOST : GHOST + ny, GHOST + k]
        v[GHOST : GHOST + ny, GHOST + nx + k] = v[GHOST : GHOST + ny, GHOST + nx - 1 - k]
    for k in range(GHOST):
        v[GHOST - 1 - k, :] = v[GHOST + k, :]
        v[GHOST + ny + k, :] = v[GHOST + ny - 1 - k, :]


def wrap_ghosts_y(grid: Grid, a: np.ndarray) -> None:
    """grid.rs:77-87."""
    v = grid.view(a)
    ny = grid.ny
    for k in range(GHOST):
        v[GHOST - 1 - k, :] = v[GHOST + ny - 1 - k, :]
        v[GHOST + ny + k, :] = v[GHOST + k, :]


class Bathymetry:
    """bathymetry.rs: the padded bed `b`, negative under water."""

    def __init__(self, b: np.ndarray):
        self.b = np.ascontiguousarray(b, dtype=np.float64)

    def clone(self) -> "Bathymetry":
        return Bathymetry(self.b.copy())

    @staticmethod
    def from_fn(grid: Grid, f: Callable) -> "Bathymetry":
        """bathymetry.rs:11-19. `f(x, y)` may take arrays (vectorised) or scalars."""
        b = np.zeros(grid.cells())
        X, Y = grid.centres()
        try:
            vals = np.asarray(f(X, Y), dtype=np.float64)
            if vals.shape != X.shape:
                vals = np.broadcast_to(vals, X.shape)
        except Exception:
            vals = np.vectorize(f, otypes=[np.float64])(X, Y)
        grid.inner(b)[:] = vals
        mirror_ghosts(grid, b)
        return Bathymetry(b)

    @staticmethod
    def from_interior(grid: Grid, values) -> "Bathymetry":
        """bathymetry.rs:21-38."""
        values = np.asarray(values, dtype=np.float64).ravel()
        if values.size != grid.nx * grid.ny:
            raise ValueError(f"bed has {values.size} values, grid needs {grid.nx * grid.ny}")
        b = np.zeros(grid.cells())
        grid.inner(b)[:] = values.reshape(grid.ny, grid.nx)
        mirror_ghosts(grid, b)
        return Bathymetry(b)

    @staticmethod
    def flat(grid: Grid, depth: float) -> "Bathymetry":
        """bathymetry.rs:40-43."""
        return Bathymetry.from_fn(grid, lambda x, y: np.full_like(x, -depth))

    @staticmethod
    def plane_beach(grid: Grid, slope: float, offshore_depth: float) -> "Bathymetry":
        """bathymetry.rs:45-49."""
        return Bathymetry.from_fn(grid, lambda x, y: -offshore_depth + slope * x + 0.0 * y)

    @staticmethod
    def rough(grid: Grid, mean_depth: float, amplitude: float) -> "Bathymetry":
        """bathymetry.rs:51-62."""
        lx = grid.nx * grid.dx
        ly = grid.ny * grid.dy
        tau = 2.0 * math.pi

        def f(x, y):
            s = 0.6 * np.sin(tau * 3.0 * x / lx) * np.cos(tau * 2.0 * y / ly) + 0.4 * np.sin(
                tau * 7.0 * x / lx + 1.3
            )
            return -mean_depth + amplitude * s

        return Bathymetry.from_fn(grid, f)


class State:
    """state.rs: padded depth and momentum, the breaking memory, and the time."""

    def __init__(self, h, hu, hv, breaking, time: float = 0.0):
        self.h = np.ascontiguousarray(h, dtype=np.float64)
        self.hu = np.ascontiguousarray(hu, dtype=np.float64)
        self.hv = np.ascontiguousarray(hv, dtype=np.float64)
        self.breaking = np.ascontiguousarray(breaking, dtype=np.float64)
        self.time = float(time)

    @staticmethod
    def zeros(grid: Grid) -> "State":
        n = grid.cells()
        return State(np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n), 0.0)

    @staticmethod
    def lake_at_rest(grid: Grid, bed: Bathymetry, eta: float) -> "State":
        """state.rs:31-40."""
        s = State.zeros(grid)
        grid.inner(s.h)[:] = np.maximum(eta - grid.inner(bed.b), 0.0)
        s.fill_walls(grid)
        return s

    def clone(self) -> "State":
        return State(self.h.copy(), self.hu.copy(), self.hv.copy(), self.breaking.copy(), self.time)

    def fill_walls(self, grid: Grid) -> None:
        """state.rs:42-62."""
        for a in (self.h, self.hu, self.hv, self.breaking):
            mirror_ghosts(grid, a)
        vu = grid.view(self.hu)
        vv = grid.view(self.hv)
        nx, ny = grid.nx, grid.ny
        for k in range(GHOST):
            vu[:, GHOST - 1 - k] *= -1.0
            vu[:, GHOST + nx + k] *= -1.0
            vv[GHOST - 1 - k, :] *= -1.0
            vv[GHOST + ny + k, :] *= -1.0

    def fill_boundaries(self, grid: Grid, periodic_y: bool) -> None:
        """state.rs:64-76."""
        self.fill_walls(grid)
        if periodic_y:
            for a in (self.h, self.hu, self.hv, self.breaking):
                wrap_ghosts_y(grid, a)

    def volume(self, grid: Grid) -> float:
        """state.rs:78-85 (one running sum, in interior order)."""
        return float(np.cumsum(grid.inner(self.h).ravel())[-1]) * grid.dx * grid.dy

    def max_abs_momentum(self, grid: Grid) -> float:
        """state.rs:87-95."""
        return float(np.max(np.maximum(np.abs(grid.inner(self.hu)), np.abs(grid.inner(self.hv)))))

    def min_depth(self, grid: Grid) -> float:
        """state.rs:97-102."""
        return float(np.min(grid.inner(self.h)))

    def eta(self, grid: Grid, bed: Bathymetry) -> np.ndarray:
        """The free surface h + b over the interior, (ny, nx)."""
        return grid.inner(self.h) + grid.inner(bed.b)


@dataclass
class Sponge:
    """forcing.rs:146-206."""

    width: int
    strength: float
    level: float = 0.0
    west: bool = False
    east: bool = False
    south: bool = False
    north: bool = False

    def edges(self, west: bool, east: bool, south: bool, north: bool) -> "Sponge":
        return replace(self, west=west, east=east, south=south, north=north)

    def to_c(self) -> abi.wc_sponge:
        return abi.wc_sponge(
            int(self.width),
            float(self.strength),
            float(self.level),
            int(self.west),
            int(self.east),
            int(self.south),
            int(self.north),
        )


@dataclass
class WaveMaker:
    """forcing.rs:18-33."""

    x: float
    amplitude: float
    period: float
    angle: float
    sigma: float
    ramp_periods: float

    def to_c(self) -> abi.wc_wavemaker:
        return abi.wc_wavemaker(
            float(self.x),
            float(self.amplitude),
            float(self.period),
            float(self.angle),
            float(self.sigma),
            float(self.ramp_periods),
        )


@dataclass
class EddyViscosity:
    """eddy.rs:62-90: how breaking fronts are followed, Kennedy et al.'s (2000) coefficients by
    default. `initial`, `settled`: rates of rise in sqrt(g h); `duration`, `linger`: times in
    sqrt(h / g); `mixing`: the mixing length in depths (0 follows fronts without viscosity)."""

    initial: float = 0.65
    settled: float = 0.15
    duration: float = 5.0
    mixing: float = 1.2
    linger: float = 5.0

    def to_c(self) -> abi.wc_eddy:
        return abi.wc_eddy(float(self.initial), float(self.settled), float(self.duration), float(self.mixing),
                           float(self.linger))


@dataclass
class Breaking:
    """dispersion.rs:44-74. `viscosity` None reads the switch afresh every step (the default);
    an EddyViscosity follows breaking fronts in the state's breaking memory (eddy.rs)."""

    eta_ratio: tuple = (0.30, 0.55)
    slope: tuple = (0.40, 0.65)
    viscosity: Optional[EddyViscosity] = None

    def to_c(self) -> abi.wc_breaking:
        return abi.wc_breaking(
            float(self.eta_ratio[0]), float(self.eta_ratio[1]), float(self.slope[0]), float(self.slope[1]),
            1 if self.viscosity is not None else 0, (self.viscosity or EddyViscosity()).to_c(),
        )


@dataclass
class Dispersion:
    """dispersion.rs:76-97. `preconditioner` selects Jacobi (the reference's) or the learned one."""

    breaking: Breaking = field(default_factory=Breaking)
    nonlinear: bool = True
    tolerance: float = 1e-4
    max_iterations: int = 200
    preconditioner: int = abi.WC_PC_JACOBI

    def to_c(self) -> abi.wc_dispersion:
        return abi.wc_dispersion(
            self.breaking.to_c(),
            int(self.nonlinear),
            float(self.tolerance),
            int(self.max_iterations),
            int(self.preconditioner),
        )


@dataclass
class DispersionStats:
    """dispersion.rs:99-106."""

    solves: int = 0
    iterations: int = 0
    unconverged: int = 0


@dataclass
class Limiting:
    """solver.rs:248-258."""

    i: int
    j: int
    depth: float
    speed: float


@dataclass
class LinearWave:
    """forcing.rs:35-44."""

    k: float
    phase_speed: float
    group_speed: float


def linear_wave(omega: float, h: float, dispersive: bool) -> LinearWave:
    """forcing.rs:46-75."""
    if not dispersive:
        c = math.sqrt(G * h)
        return LinearWave(omega / c, c, c)
    nu = omega * omega * h / G
    if not nu < 3.0:
        raise ValueError(
            f"a wave of angular frequency {omega} is too short for the dispersive model in {h} m of water"
        )
    kh = math.sqrt(nu / (1.0 - nu / 3.0))
    k = kh / h
    phase_speed = omega / k
    return LinearWave(k, phase_speed, phase_speed / (1.0 + kh * kh / 3.0))


def manning_factor(h: float, speed: float, dt: float, n: float) -> float:
    """forcing.rs:288-297."""
    k = G * n * n / h ** (4.0 / 3.0)
    return 1.0 / (1.0 + dt * k * speed)


class SolverConfig:
    """The builder half of `Solver` (solver.rs:260-429), independent of the engine.

    Builders mutate and return `self`, as the reference's consuming builders do; the engine
    is created on first use. `with_periodic_y` wraps the bed's ghost rows as the reference does.
    """

    def __init__(self, grid: Grid, bed: Bathymetry):
        self.grid = grid
        self.bed = bed.clone()
        self.cfl = 0.4
        self.order = Order.Second
        self.manning = 0.0
        self.periodic_y = False
        self.sponges: list = []
        self.wavemaker: Optional[WaveMaker] = None
        self._dispersion: Optional[Dispersion] = None
        self.shallow: Optional[np.ndarray] = None
        self._handle = None

    def _changed(self):
        self._release()

    def _release(self):
        pass

    def with_order(self, order: Order):
        self.order = Order(order)
        self._changed()
        return self

    def with_manning(self, n: float):
        self.manning = float(n)
        self._changed()
        return self

    def with_sponge(self, sponge: Sponge):
        self.sponges.append(sponge)
        self._changed()
        return self

    def with_wavemaker(self, spec: WaveMaker):
        self.wavemaker = spec
        self._changed()
        return self

    def with_dispersion(self, dispersion: Dispersion):
        self._dispersion = copy.deepcopy(dispersion)
        self._changed()
        return self

    def with_periodic_y(self):
        self.periodic_y = True
        wrap_ghosts_y(self.grid, self.bed.b)
        self._changed()
        return self

    def with_shallow_cells(self, cells):
        cells = np.asarray(cells, dtype=bool).ravel()
        if cells.size != self.grid.nx * self.grid.ny:
            raise ValueError("one entry per interior cell")
        self.shallow = np.ascontiguousarray(cells.astype(np.uint8))
        self._changed()
        return self

    def dispersion(self) -> Optional[Dispersion]:
        return self._dispersion

    def _c_config(self):
        """A wc_config plus the objects that keep its pointers alive."""
        keep = []
        cfg = abi.wc_config()
        cfg.cfl = float(self.cfl)
        cfg.order = int(self.order)
        cfg.manning = float(self.manning)
        cfg.periodic_y = int(self.periodic_y)
        if self.sponges:
            arr = (abi.wc_sponge * len(self.sponges))(*[s.to_c() for s in self.sponges])
            keep.append(arr)
            cfg.sponges = arr
            cfg.n_sponges = len(self.sponges)
        if self.wavemaker is not None:
            wm = self.wavemaker.to_c()
            keep.append(wm)
            cfg.wavemaker = abi.C.pointer(wm)
        if self._dispersion is not None:
            d = self._dispersion.to_c()
            keep.append(d)
            cfg.dispersion = abi.C.pointer(d)
        if self.shallow is not None:
            keep.append(self.shallow)
            cfg.shallow_cells = self.shallow.ctypes.data_as(abi.C.POINTER(abi.C.c_uint8))
        return cfg, keep
