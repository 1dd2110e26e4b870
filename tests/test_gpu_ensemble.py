"""Ensembles: members advanced together by one persistent launch per step match the same runs
done one at a time by standalone solvers (same inputs, same adaptive stepping)."""
import math

import numpy as np
import pytest

from wavesim_b200 import Bathymetry, Ensemble, Grid, Order, Solver, State
from wavesim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _members():
    a = W.sgn_beach(160, 96, 2.0, seed=21, name="m0")          # fifth order + SGN, periodic
    b = W.sgn_beach(96, 64, 3.0, seed=22, name="m1", tolerance=1e-6)
    c = W.config1()                                              # second order shallow water
    return [a, b, c]


def test_ensemble_members_match_standalone_runs():
    ws = _members()
    ens = Ensemble([w.solver(Solver) for w in ws])
    starts = [W.wave_train_state(w) if w.dispersion else State.lake_at_rest(w.grid, w.bed, 0.0) for w in ws]
    for m, s0 in enumerate(starts):
        ens.upload(m, s0)
    choice, ms = ens.autotune(2)
    assert 0 <= choice < 5 and ms[choice] > 0 and ms[4] > 0
    ens.step_n(25)
    ens.synchronize()
    for m, (w, s0) in enumerate(zip(ws, starts)):
        ref = w.solver(Solver)
        ref.upload(s0)
        ref.step_n(25)
        ref.synchronize()
        a, b = s0.clone(), s0.clone()
        ens.download(m, a)
        ref.download(b)
        g = w.grid
        # Same kernels; the dot products are split over a different number of CTAs, so FP64
        # partial sums round differently: agreement to FP32 level, not bitwise.
        assert abs(a.time - b.time) < 1e-9 * max(1.0, b.time), (m, a.time, b.time)
        assert np.max(np.abs(g.inner(a.h) - g.inner(b.h))) < 1e-5, m
        st, t = ens.member_stats(m)
        if w.dispersion:
            assert st.solves == 50 and st.unconverged == 0


def test_ensemble_members_stop_at_their_end_time():
    ws = _members()[1:]
    ens = Ensemble([w.solver(Solver) for w in ws])
    for m, w in enumerate(ws):
        ens.upload(m, W.wave_train_state(w) if w.dispersion else State.lake_at_rest(w.grid, w.bed, 0.0))
    ens.step_n(100000, t_end=57.0)
    ens.synchronize()
    for m in range(len(ws)):
        _, t = ens.member_stats(m)
        assert abs(t - 57.0) < 1e-9


def test_learned_ensemble_members_match_standalone_learned_runs():
    """With the learned preconditioner attached, every member steps through its own captured step
    on its own stream: the same kernels as a standalone solver with the same network, so the same
    bits."""
    from wavesim_b200 import LearnedPreconditioner
    from wavesim_b200.lpc import UNetSpec

    net = LearnedPreconditioner(UNetSpec(), seed=3)
    ws = _members()
    ens = Ensemble([w.solver(Solver) for w in ws])
    ens.set_preconditioner(net)
    starts = [W.wave_train_state(w) if w.dispersion else State.lake_at_rest(w.grid, w.bed, 0.0) for w in ws]
    for m, s0 in enumerate(starts):
        ens.upload(m, s0)
    choice, ms = ens.autotune(2)
    assert choice == 4 and ms[4] > 0 and ms[:4] == [-1.0] * 4
    ens.step_n(20)
    ens.synchronize()
    for m, (w, s0) in enumerate(zip(ws, starts)):
        ref = w.solver(Solver)
        if w.dispersion:
            ref.set_preconditioner(net)
        ref.upload(s0)
        ref.step_n(20)
        ref.synchronize()
        a, b = s0.clone(), s0.clone()
        ens.download(m, a)
        ref.download(b)
        assert a.time == b.time, m
        assert np.array_equal(a.h, b.h) and np.array_equal(a.hu, b.hu) and np.array_equal(a.hv, b.hv), m
        st, _ = ens.member_stats(m)
        if w.dispersion:
            assert st.solves == 40 and st.unconverged == 0
    assert ens.launch_count() > 0
