"""wavesim_b200 — wavecore's time step (mlaegn/wavesim) rebuilt for NVIDIA B200.

The step — the well-balanced SSP-RK2 finite-volume shallow-water update and the
Serre-Green-Naghdi dispersion solve by preconditioned conjugate gradients — runs in hand-written
sm_100a CUDA behind the C ABI of include/wavecore_c.h. This package mirrors the reference's
Rust API in Python over that ABI:

    from wavesim_b200 import Grid, Bathymetry, State, Solver, Order, Dispersion
    grid = Grid(64, 48, 3.0, 3.0)
    bed = Bathymetry.plane_beach(grid, 0.02, 8.0)
    s = State.lake_at_rest(grid, bed, 0.0)
    solver = Solver(grid, bed)
    solver.step(s, solver.stable_dt(s))
"""
from .model import (  # noqa: F401
    G,
    GHOST,
    H_DRY,
    Bathymetry,
    Breaking,
    Dispersion,
    DispersionStats,
    EddyViscosity,
    Grid,
    Limiting,
    LinearWave,
    Order,
    Sponge,
    State,
    WaveMaker,
    linear_wave,
    manning_factor,
)
from .solver import Ensemble, LearnedPreconditioner, Nest, Recorder, Solver, WavecoreError  # noqa: F401
