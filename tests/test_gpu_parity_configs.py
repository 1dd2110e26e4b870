"""Parity with the FP64 oracle at the benchmark configurations' own sizes, the true FP64 residual
of the device's dispersive solves, and ensemble members against the oracle.

Tolerances are FP32 against FP64 and stated per test. The true residual: the device stops on its
recursively updated FP32 residual, ||r|| <= tol ||b|| + 1e-10 with tol = 1e-8, the reference's rule
(crates/wavecore/src/dispersion.rs:510-523); the residual of the stored FP32 solution itself,
||b - A w|| / ||b|| computed in FP64, cannot go below what rounding an exact solution to FP32
leaves, so each test measures that floor on the same system (the oracle's FP64 solve rounded to
FP32) and bounds the device's true residual by a small multiple of it.
"""
import math

import numpy as np
import pytest

from oracle.oracle import OracleSolver, pcg_solve, set_threads, true_relative_residual
from parity import compare, record, surface_metrics
from wavesim_b200 import Ensemble, Solver, State
from wavesim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def residuals(w, gpu):
    """True FP64 residuals of the device's last solve, the oracle's FP64 solve of the same system
    from zero, and that solution rounded to FP32 (the storage floor)."""
    sysd = gpu.dispersion_system()
    dev = true_relative_residual(w.grid, w.periodic_y, sysd)
    wx, wy, it, conv = pcg_solve(w.grid, w.periodic_y, sysd, w.dispersion.tolerance, 2000)
    orc = true_relative_residual(w.grid, w.periodic_y, {**sysd, "wx": wx, "wy": wy})
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    floor = true_relative_residual(w.grid, w.periodic_y, {**sysd, "wx": f32(wx), "wy": f32(wy)})
    return {"device_true_rel_residual": dev, "oracle_true_rel_residual": orc, "oracle_iterations_from_zero": it,
            "oracle_converged": bool(conv), "fp32_solution_floor": floor}


def test_config2_full_size_matches_the_oracle():
    """1024x512 at 2 m, fifth order + SGN by Jacobi PCG to 1e-8, periodic, oblique maker: 20 steps
    from the wave-train start."""
    w = W.config2()
    m, sg, so, gpu = compare(w, W.wave_train_state(w), 20)
    m.update(residuals(w, gpu))
    record("config2_1024x512_20steps", m)
    # FP32 state against FP64 after 20 steps of 2 m swell.
    assert m["eta_max_abs_diff_m"] < 3e-5
    assert m["eta_rms_diff_m"] < 3e-6
    assert m["wet_mask_agreement"] > 0.999
    assert m["breaking_mask_agreement"] > 0.995
    assert m["volume_rel_diff"] < 1e-6
    assert m["oracle_converged"] and m["oracle_true_rel_residual"] < 1.2e-8
    assert m["device_true_rel_residual"] < max(20.0 * m["fp32_solution_floor"], 1.2e-8)


def test_config3_full_size_matches_the_oracle():
    """2048x1024 at 2 m (the benchmark's default workload): 6 steps from the wave-train start."""
    w = W.config3()
    m, sg, so, gpu = compare(w, W.wave_train_state(w), 6)
    m.update(residuals(w, gpu))
    record("config3_2048x1024_6steps", m)
    assert m["eta_max_abs_diff_m"] < 2e-5
    assert m["eta_rms_diff_m"] < 2e-6
    assert m["wet_mask_agreement"] > 0.999
    assert m["breaking_mask_agreement"] > 0.995
    assert m["device_true_rel_residual"] < max(20.0 * m["fp32_solution_floor"], 1.2e-8)


def test_config5_reef_matches_the_oracle():
    """4096x4096 at 1 m, the reef with its shoal: 5 steps from the wave-train start."""
    w = W.config5()
    m, sg, so, gpu = compare(w, W.wave_train_state(w), 5)
    record("config5_4096x4096_5steps", m)
    assert m["eta_max_abs_diff_m"] < 2e-5
    assert m["eta_rms_diff_m"] < 2e-6
    assert m["wet_mask_agreement"] > 0.999
    assert m["breaking_mask_agreement"] > 0.995


def test_ensemble_members_match_the_oracle():
    """The two smallest members of the 64-run ensemble, advanced together by the ensemble's
    persistent launches and, separately, by the oracle, both with adaptive steps to the same end
    time."""
    members = sorted(W.config4(), key=lambda w: w.grid.nx * w.grid.ny)[:2]
    ens = Ensemble([w.solver(Solver) for w in members])
    starts = [W.wave_train_state(w) for w in members]
    for k, s0 in enumerate(starts):
        ens.upload(k, s0)
    t_end = max(s.time for s in starts) + 4.0
    ens.step_n(100000, t_end=t_end)
    ens.synchronize()
    set_threads(0)
    for k, (w, s0) in enumerate(zip(members, starts)):
        orc = w.solver(OracleSolver)
        so = s0.clone()
        steps = 0
        while so.time < t_end:
            dt = min(orc.stable_dt(so), t_end - so.time)
            assert math.isfinite(dt) and dt > 0
            orc.step(so, dt)
            steps += 1
        sg = s0.clone()
        ens.download(k, sg)
        st, t = ens.member_stats(k)
        m = {"member": w.name, "oracle_steps": steps, "device_solves": st.solves, **surface_metrics(w, sg, so)}
        record(f"ensemble_{w.name}", m)
        assert abs(t - t_end) < 1e-9 and abs(so.time - t_end) < 1e-9
        assert st.unconverged == 0
        assert m["eta_max_abs_diff_m"] < 3e-5
        assert m["eta_rms_diff_m"] < 3e-6
        assert m["wet_mask_agreement"] > 0.999
