"""FP64 restatement of the reference driver's per-step statistics (TEST INFRASTRUCTURE ONLY).

Follows crates/wavesim/src/lib.rs: `Stats` and `Stats::close_wave` (:899-931), `Stage::record`
(:1276-1301), `wave_height` (:1303-1314), `unsettled` (:1316-1338), `breaking_fraction`
(:1340-1344), the frame's rise check (:1348-1366) and `FirstHarmonic` (:1095-1169), on states of
the FP64 oracle. Only tests/ import it; it checks the device recorder (`wc_recorder_*`).
"""
from __future__ import annotations

import math

import numpy as np

BREAKING = 0.8  # lib.rs:1222


class FirstHarmonic:
    """lib.rs:1095-1169: least-squares fit of eta = m + a cos(wt) + b sin(wt) per cell."""

    def __init__(self, period: float, cells: int):
        self.omega = 2.0 * math.pi / period
        self.moments = np.zeros(6)
        self.sums = np.zeros((3, cells))

    def weights(self, t: float, w: float):
        s, c = math.sin(self.omega * t), math.cos(self.omega * t)
        self.moments += w * np.array([1.0, c, s, c * c, c * s, s * s])
        return w, w * c, w * s

    def add_all(self, eta: np.ndarray, weights) -> None:
        for k in range(3):
            self.sums[k] += weights[k] * eta

    def amplitudes(self):
        """(a, -b) per cell as an (cells, 2) array, or None when the samples cannot separate a
        mean, a cosine and a sine."""
        s, c, n, cc, cs, ss = self.moments
        m = np.array([[s, c, n], [c, cc, cs], [n, cs, ss]])

        def cof(r, k):
            r1, r2 = (r + 1) % 3, (r + 2) % 3
            k1, k2 = (k + 1) % 3, (k + 2) % 3
            return m[r1][k1] * m[r2][k2] - m[r1][k2] * m[r2][k1]

        det = sum(m[0][k] * cof(0, k) for k in range(3))
        if math.isnan(det) or det <= 1e-3 * s * s * s / 4.0:
            return None
        inv = np.array([[cof(k, r) / det for k in range(3)] for r in range(3)])
        rows = inv @ self.sums
        return np.stack([rows[1], -rows[2]], axis=1)


class Recorder:
    """`Stats` of one stage, fed with interior eta and the breaking indicator after every step."""

    def __init__(self, cells: int, start: float, start_from: float, period: float):
        self.from_ = start_from
        self.seconds = 0.0
        self.breaking_seconds = np.zeros(cells)
        self.eta_max = np.full(cells, -np.inf)
        self.eta_min = np.full(cells, np.inf)
        self.period = period
        self.next_wave = max(start_from, start) + period
        self.wave_max = np.full(cells, -np.inf)
        self.wave_min = np.full(cells, np.inf)
        self.waves = []
        self.harmonic = FirstHarmonic(period, cells)

    def close_wave(self):
        heights = np.where(np.isfinite(self.wave_max), self.wave_max - self.wave_min, 0.0)
        self.waves.append(heights)
        self.wave_max[:] = -np.inf
        self.wave_min[:] = np.inf
        self.next_wave += self.period

    def record(self, time: float, dt: float, eta: np.ndarray, now: np.ndarray) -> None:
        """A step of `dt` that ended at `time`; eta and the breaking indicator `now` per cell."""
        inside = min(dt, time - self.from_)
        if inside <= 0.0:
            return
        if time > self.next_wave + 1e-9:
            self.close_wave()
        w = self.harmonic.weights(time, inside)
        self.harmonic.add_all(eta, w)
        self.eta_max = np.maximum(self.eta_max, eta)
        self.eta_min = np.minimum(self.eta_min, eta)
        self.wave_max = np.maximum(self.wave_max, eta)
        self.wave_min = np.minimum(self.wave_min, eta)
        self.breaking_seconds += np.where(now >= BREAKING, inside, 0.0)
        self.seconds += inside

    def wave_height(self):
        if not self.waves:
            return None
        return sum(self.waves) / len(self.waves)

    def unsettled(self, nx: int, ny: int):
        if len(self.waves) < 2:
            return None
        first, last = self.waves[0], self.waves[-1]
        change = []
        for j in range(ny // 4, ny - ny // 4):
            for i in range(nx):
                n = j * nx + i
                if first[n] > 0.3:
                    change.append(abs(last[n] / first[n] - 1.0) / (len(self.waves) - 1))
        if not change:
            return None
        change.sort()
        return change[len(change) // 2]

    def breaking_fraction(self):
        return self.breaking_seconds / max(self.seconds, np.finfo(float).tiny)


def frame_rise(eta: np.ndarray, depth: np.ndarray, tide: float) -> float:
    """lib.rs:1352-1358: the highest surface above still water among cells deeper than 1 mm."""
    wet = depth > 1e-3
    return float(max(0.0, np.max(eta[wet] - tide))) if wet.any() else 0.0
