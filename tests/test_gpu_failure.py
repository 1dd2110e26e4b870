"""Failure handling of the persistent kernels' bounded waits, without any GPU fault.

Every device-side wait (a grid barrier of the dispersive solve's cooperative kernel) is bounded
in time; when the limit runs out the kernel sets an error bit and every CTA returns, and the host
reports WC_ETIMEOUT with the context still usable. A limit of 1 ns makes the first barrier's
waiters run out on a small solve; nothing traps, faults or spins without bound.
"""
import numpy as np
import pytest

from wavesim_b200 import Solver, WavecoreError, abi
from wavesim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_a_barrier_wait_that_runs_out_reports_timeout_and_leaves_the_gpu_usable():
    w = W.sgn_beach(192, 96, 2.0, seed=11, name="sgn_small")  # 36 tiles: many CTAs at each barrier
    s0 = W.wave_train_state(w)
    sol = w.solver(Solver)
    dt = sol.stable_dt(s0)
    sol.set_wait_limit(1)
    with pytest.raises(WavecoreError) as e:
        sol.step(s0.clone(), dt)
    assert e.value.status == abi.WC_ETIMEOUT
    # The same solver with the default limit again, and a fresh one: normal steps. The stopped
    # solve may have left a different warm start behind, so the two agree to the solve's
    # tolerance, not bit for bit.
    sol.set_wait_limit(0)
    a, b = s0.clone(), s0.clone()
    sol.step(a, dt)
    fresh = w.solver(Solver)
    fresh.step(b, dt)
    g = w.grid
    assert np.max(np.abs(g.inner(a.h) - g.inner(b.h))) < 1e-5
    assert np.max(np.abs(g.inner(a.hu) - g.inner(b.hu))) < 1e-4
    assert fresh.dispersion_stats().unconverged == 0
