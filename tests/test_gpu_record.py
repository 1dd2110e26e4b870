"""The device recorder (per-step statistics) and frames against the FP64 restatement of the
reference driver's `Stage::record` run on the FP64 oracle's states (same inputs, same dt).

Tolerances (FP32 state against FP64): surface statistics 3e-5 m, harmonic 3e-5 m, breaking
fractions within 0.02 on 99.5 % of the cells.
"""
import math

import numpy as np
import pytest

from oracle.oracle import OracleSolver
from oracle.record_oracle import Recorder as OracleRecorder
from oracle.record_oracle import frame_rise
from wavesim_b200 import Recorder, Solver
from wavesim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run_both(w, steps, start_from_offset):
    s0 = W.wave_train_state(w)
    g = w.grid
    gpu = w.solver(Solver)
    orc = w.solver(OracleSolver)
    sg, so = s0.clone(), s0.clone()
    period = w.maker.period
    rec = Recorder(gpu, s0.time + start_from_offset, period)
    ref = OracleRecorder(g.nx * g.ny, s0.time, s0.time + start_from_offset, period)
    b = g.inner(w.bed.b)
    for _ in range(steps):
        dt = orc.stable_dt(so)
        orc.step(so, dt)
        gpu.step(sg, dt)
        eta = (g.inner(so.h) + b).ravel()
        ref.record(so.time, dt, eta, orc.breaking_indicator(so).ravel())
    return gpu, rec, ref, sg, so


def test_recorder_matches_the_restated_driver_statistics():
    w = W.config1()
    gpu, rec, ref, sg, so = run_both(w, 700, 2.0)
    out = rec.read()
    g = w.grid
    assert out["waves"] == len(ref.waves) >= 2
    assert abs(out["seconds"] - ref.seconds) < 1e-9 * ref.seconds
    for k, v in (("eta_max", ref.eta_max), ("eta_min", ref.eta_min), ("wave_height", ref.wave_height())):
        d = np.abs(out[k].ravel() - v)
        assert d.max() < 3e-5, (k, d.max())
    amp = ref.harmonic.amplitudes()
    assert out["harmonic"] is not None and amp is not None
    h = out["harmonic"].ravel()
    assert np.max(np.abs(h.real - amp[:, 0])) < 3e-5 and np.max(np.abs(h.imag - amp[:, 1])) < 3e-5
    bf = np.abs(out["breaking_fraction"].ravel() - ref.breaking_fraction())
    assert np.mean(bf < 0.02) > 0.995
    u_ref = ref.unsettled(g.nx, g.ny)
    assert (out["unsettled"] is None) == (u_ref is None)
    if u_ref is not None:
        assert abs(out["unsettled"] - u_ref) < 1e-3


def test_frame_matches_the_oracle_state():
    w = W.sgn_beach(128, 64, 2.0, seed=5, name="frame")
    gpu, rec, ref, sg, so = run_both(w, 40, 0.0)
    gpu.upload(sg)
    eta, brk, rise = gpu.frame(0.0)
    g = w.grid
    eta_o = g.inner(so.h) + g.inner(w.bed.b)
    assert np.max(np.abs(eta - eta_o)) < 3e-5
    brk_o = np.asarray(w.solver(OracleSolver).breaking_indicator(so)).reshape(brk.shape)
    assert np.mean(np.abs(brk - brk_o) < 0.02) > 0.995
    assert abs(rise - frame_rise(eta_o.ravel(), g.inner(so.h).ravel(), 0.0)) < 3e-5
    assert eta.dtype == np.float32 and brk.dtype == np.float32


def test_device_resident_steps_record_like_host_steps():
    w = W.sgn_beach(128, 64, 2.0, seed=6, name="resident_rec")
    s0 = W.wave_train_state(w)
    a, b = w.solver(Solver), w.solver(Solver)
    ra = Recorder(a, s0.time, w.maker.period)
    rb = Recorder(b, s0.time, w.maker.period)
    sa = s0.clone()
    dts = []
    for _ in range(30):
        dt = a.stable_dt(sa)
        dts.append(dt)
        a.step(sa, dt)
    b.upload(s0)
    for dt in dts:
        b.step_device(dt)
    b.synchronize()
    oa, ob = ra.read(), rb.read()
    assert oa["seconds"] == pytest.approx(ob["seconds"], rel=1e-12)
    assert np.max(np.abs(oa["eta_max"] - ob["eta_max"])) < 1e-9
    assert math.isfinite(oa["seconds"])


def test_a_recorded_run_reads_back_in_the_reference_format(tmp_path):
    from wavesim_b200.runio import Run, RunWriter, record_frame, record_stats

    w = W.config1()
    s0 = W.wave_train_state(w)
    sol = w.solver(Solver)
    sol.upload(s0)
    rec = Recorder(sol, s0.time, w.maker.period)
    g = w.grid
    writer = RunWriter(str(tmp_path / "run"), "swe", g.inner(w.bed.b), g.dx, g.dy,
                       waves={"height_m": 2 * w.maker.amplitude, "period_s": w.maker.period})
    frames = []
    for _ in range(4):
        sol.step_n(150)
        sol.synchronize()
        t = sol.time_device()
        record_frame(writer, sol, t)
        frames.append((t, *sol.frame(0.0)[:2]))
    record_stats(writer, rec, s0.time, sol.time_device())
    writer.finish()
    run = Run(str(tmp_path / "run"))
    assert run.header["frame_count"] == 4 and run.header["times"] == [f[0] for f in frames]
    for k, (t, eta, brk) in enumerate(frames):
        assert np.array_equal(run.field("eta", k), eta) and np.array_equal(run.field("breaking", k), brk)
    out = rec.read()
    assert np.array_equal(run.stat("eta_max"), out["eta_max"].astype(np.float32))
    assert run.header["stats"]["fields"][:3] == ["break_fraction", "eta_max", "eta_min"]
