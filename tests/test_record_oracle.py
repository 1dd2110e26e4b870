"""The FP64 restatement of the driver's per-step statistics (CPU only)."""
import math

import numpy as np

from oracle.record_oracle import FirstHarmonic, Recorder, frame_rise


def test_first_harmonic_recovers_a_sinusoid_exactly():
    # lib.rs:1095-1169: eta = m + a cos wt + b sin wt reads (a, -b), whatever the weights.
    period, m, a, b = 12.0, 0.3, 0.7, -0.4
    fh = FirstHarmonic(period, 1)
    rng = np.random.default_rng(0)
    t = 5.0
    while t < 5.0 + 1.5 * period:
        dt = float(rng.uniform(0.05, 0.3))
        t += dt
        eta = m + a * math.cos(fh.omega * t) + b * math.sin(fh.omega * t)
        fh.add_all(np.array([eta]), fh.weights(t, dt))
    amp = fh.amplitudes()
    assert abs(amp[0, 0] - a) < 1e-12 and abs(amp[0, 1] + b) < 1e-12


def test_first_harmonic_needs_enough_of_a_period():
    fh = FirstHarmonic(12.0, 1)
    for k in range(10):
        t = 0.1 * k
        fh.add_all(np.array([1.0]), fh.weights(t, 0.1))
    assert fh.amplitudes() is None


def test_wave_heights_breaking_time_and_the_start():
    period, amp = 10.0, 0.5
    rec = Recorder(cells=2, start=0.0, start_from=2.0, period=period)
    t, dt = 0.0, 0.01
    while t < 4.5 * period:
        t += dt
        eta = np.array([amp * math.sin(2 * math.pi * t / period), 0.0])
        now = np.array([1.0 if math.sin(2 * math.pi * t / period) > 0 else 0.0, 0.0])
        rec.record(t, dt, eta, now)
    assert abs(rec.seconds - (t - 2.0)) < 1e-9  # nothing before `from`
    assert len(rec.waves) == 4  # waves close at 12, 22, 32, 42 s
    h = rec.wave_height()
    assert abs(h[0] - 2 * amp) < 1e-3 and h[1] == 0.0
    assert abs(rec.breaking_fraction()[0] - 0.5) < 0.05  # 4.3 periods: not exactly half
    assert rec.unsettled(2, 1) is None or rec.unsettled(2, 1) < 1e-3


def test_frame_rise_counts_wet_cells_only():
    eta = np.array([0.5, 3.0, 1.0])
    depth = np.array([1.0, 0.0005, 2.0])
    assert frame_rise(eta, depth, 0.2) == 0.8
