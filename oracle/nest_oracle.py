"""FP64 restatement of one-way nesting (TEST INFRASTRUCTURE ONLY).

Follows crates/wavecore/src/forcing.rs:180-283 (Sponge::rate, relax_cell, Relaxation) and
crates/wavesim/src/lib.rs:1554-1605 (Sampler) and :1846-1896 (the nested step: the coarse run
stepped until it brackets the fine step's end, targets sampled from the states around it and
interpolated in time, the fine step, then the relaxation). Works on oracle states (padded FP64
arrays). Only tests/ import it.
"""
from __future__ import annotations

import math

import numpy as np

GHOST = 3
H_DRY = 1e-8


def sponge_rate(sp, nx: int, ny: int, a: int, b: int) -> float:
    """forcing.rs:180-206 at interior cell (a, b)."""
    w = float(sp.width)

    def ramp(d):
        if d < sp.width:
            f = (w - d) / w
            return f * f
        return 0.0

    r = 0.0
    if sp.west:
        r = max(r, ramp(a))
    if sp.east:
        r = max(r, ramp(nx - 1 - a))
    if sp.south:
        r = max(r, ramp(b))
    if sp.north:
        r = max(r, ramp(ny - 1 - b))
    return sp.strength * r


def _reflect(i: int, n: int) -> int:
    if 0 <= i < n:
        return i
    p = 2 * n
    t = i % p
    return t if t < n else p - 1 - t


class Nest:
    def __init__(self, fine_grid, coarse_grid, zones, x_offset: float, y_offset: float):
        self.cells = []
        fg, cg = fine_grid, coarse_grid
        for b in range(fg.ny):
            for a in range(fg.nx):
                rate = max([sponge_rate(z, fg.nx, fg.ny, a, b) for z in zones] + [0.0])
                if rate <= 0.0:
                    continue
                x = x_offset + (a + 0.5) * fg.dx
                y = y_offset + (b + 0.5) * fg.dy
                cx, cy = x / cg.dx - 0.5, y / cg.dy - 0.5
                ix, iy = math.floor(cx), math.floor(cy)
                wx, wy = cx - ix, cy - iy
                corners = []
                for di, dj, w in ((0, 0, (1 - wx) * (1 - wy)), (1, 0, wx * (1 - wy)), (0, 1, (1 - wx) * wy), (1, 1, wx * wy)):
                    pi = min(max(ix + di, -1), cg.nx)
                    pj = min(max(iy + dj, -1), cg.ny)
                    corners.append((pi, pj, w))
                self.cells.append(((a, b), rate, corners))
        self.fg, self.cg = fg, cg

    def sample(self, s, bed_b):
        """Sampler::sample on the coarse state filled as walls (lib.rs:1863-1864, 1590-1605)."""
        cg = self.cg
        W = cg.nx + 2 * GHOST
        out = []
        for _, _, corners in self.cells:
            eta = u = v = wt = 0.0
            for pi, pj, w in corners:
                mi, mj = _reflect(pi, cg.nx), _reflect(pj, cg.ny)
                k = (mj + GHOST) * W + (mi + GHOST)
                sx = 1.0 if 0 <= pi < cg.nx else -1.0
                sy = 1.0 if 0 <= pj < cg.ny else -1.0
                h = s.h[k]
                if h > 1e-3 and w > 0.0:
                    eta += w * (h + bed_b[k])
                    u += w * sx * s.hu[k] / h
                    v += w * sy * s.hv[k] / h
                    wt += w
            out.append((eta / wt, u / wt, v / wt) if wt > 0.0 else (-math.inf, 0.0, 0.0))
        return out

    def apply(self, s, bed_b, dt, t0, frm, t1, to, end):
        """The time interpolation of lib.rs:1875-1893, then Relaxation::apply (forcing.rs:259-282)."""
        w = min(max((end - t0) / (t1 - t0), 0.0), 1.0) if t1 != t0 else 1.0
        W = self.fg.nx + 2 * GHOST
        for m, ((a, b), rate, _) in enumerate(self.cells):
            x, y = frm[m], to[m]
            if math.isfinite(x[0]) and math.isfinite(y[0]):
                tgt = tuple(x[i] + w * (y[i] - x[i]) for i in range(3))
            else:
                tgt = x if w < 0.5 else y
            k = (b + GHOST) * W + (a + GHOST)
            f = math.exp(-rate * dt)
            ht = max(tgt[0] - bed_b[k], 0.0)
            s.h[k] = f * s.h[k] + (1.0 - f) * ht
            s.hu[k] = f * s.hu[k] + (1.0 - f) * ht * tgt[1]
            s.hv[k] = f * s.hv[k] + (1.0 - f) * ht * tgt[2]
            if s.h[k] < H_DRY:
                s.h[k] = max(s.h[k], 0.0)
                s.hu[k] = 0.0
                s.hv[k] = 0.0
