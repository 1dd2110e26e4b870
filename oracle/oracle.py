"""Python binding of the FP64 oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the parity checker of the device build and its timed CPU baseline: a line-faithful
FP64 C restatement of wavecore's step (mlaegn/wavesim, crates/wavecore/src/). Only tests/,
`__graft_entry__.smoke()` and bench.py's CPU-baseline leg use it; the product never imports it.

`OracleSolver` has the same builder API as the product's `wavesim_b200.Solver`, so one test body
runs against either.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

from wavesim_b200 import abi
from wavesim_b200.model import DispersionStats, Limiting, SolverConfig, State

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwavecore_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off, OpenMP)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        D = abi.DPTR
        L.or_set_threads.argtypes = [C.c_int]
        L.or_set_threads.restype = C.c_int
        L.or_solver_create.argtypes = [C.POINTER(abi.wc_grid), D, C.POINTER(abi.wc_config), C.POINTER(C.c_void_p)]
        L.or_solver_create.restype = C.c_int
        L.or_solver_destroy.argtypes = [C.c_void_p]
        L.or_last_error.restype = C.c_char_p
        L.or_solver_bed.argtypes = [C.c_void_p]
        L.or_solver_bed.restype = D
        L.or_step.argtypes = [C.c_void_p, D, D, D, D, D, C.c_double]
        L.or_stable_dt.argtypes = [C.c_void_p, D, D, D]
        L.or_stable_dt.restype = C.c_double
        L.or_limiting_cell.argtypes = [C.c_void_p, D, D, D, C.POINTER(abi.wc_limiting)]
        L.or_limiting_cell.restype = C.c_int
        L.or_breaking_indicator.argtypes = [C.c_void_p, D, D, D, D, D]
        L.or_dispersion_stats.argtypes = [C.c_void_p, C.POINTER(abi.wc_stats)]
        L.or_dispersion_stats.restype = C.c_int
        L.or_drive.argtypes = [C.c_void_p, D, D, D]
        L.or_drive.restype = C.c_int
        L.or_face_values.argtypes = [D, C.c_double, D, D]
        L.or_smoothstep.argtypes = [C.c_double, C.c_double, C.c_double]
        L.or_smoothstep.restype = C.c_double
        L.or_linear_wave.argtypes = [C.c_double, C.c_double, C.c_int, D, D, D]
        L.or_linear_wave.restype = C.c_int
        L.or_manning_factor.argtypes = [C.c_double] * 4
        L.or_manning_factor.restype = C.c_double
        L.or_mirror_ghosts.argtypes = [C.POINTER(abi.wc_grid), D]
        L.or_wrap_ghosts_y.argtypes = [C.POINTER(abi.wc_grid), D]
        L.or_fill_boundaries.argtypes = [C.POINTER(abi.wc_grid), C.c_int, D, D, D, D]
        L.or_matvec.argtypes = [C.POINTER(abi.wc_grid), C.c_int, D, D, D, D, D, D, D]
        L.or_dot.argtypes = [C.POINTER(abi.wc_grid), D, D, D, D]
        L.or_dot.restype = C.c_double
        L.or_dispersion_apply.argtypes = [
            C.POINTER(abi.wc_grid), C.c_int, C.POINTER(abi.wc_dispersion), D, D, D, D, D, D, D,
        ]
        L.or_eddy_threshold.argtypes = [C.POINTER(abi.wc_eddy), C.c_double, C.c_double]
        L.or_eddy_threshold.restype = C.c_double
        L.or_eddy_follow.argtypes = [C.POINTER(abi.wc_grid), C.POINTER(abi.wc_eddy), D, D, D, D, D, C.c_double, D]
        L.or_eddy_diffuse.argtypes = [C.POINTER(abi.wc_grid), C.c_int, D, D, D, D, D, C.c_double]
        L.or_eddy_diffuse.restype = C.c_int
        L.or_follow_breaking.argtypes = [C.c_void_p, D, D, D, D, C.c_double]
        L.or_follow_breaking.restype = C.c_int
        L.or_volume.argtypes = [C.POINTER(abi.wc_grid), D]
        L.or_volume.restype = C.c_double
        L.or_max_abs_momentum.argtypes = [C.POINTER(abi.wc_grid), D, D]
        L.or_max_abs_momentum.restype = C.c_double
        L.or_min_depth.argtypes = [C.POINTER(abi.wc_grid), D]
        L.or_min_depth.restype = C.c_double
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    """OpenMP threads for the oracle's row loops (results are identical for any count)."""
    return lib().or_set_threads(int(n))


class OracleError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class OracleSolver(SolverConfig):
    """The reference's `Solver` (solver.rs:260-733), computed by the FP64 oracle."""

    def _release(self):
        if getattr(self, "_handle", None):
            lib().or_solver_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    def _h(self):
        if self._handle is None:
            cfg, keep = self._c_config()
            g = self.grid.to_c()
            out = C.c_void_p()
            st = lib().or_solver_create(C.byref(g), abi.dptr(self.bed.b), C.byref(cfg), C.byref(out))
            if st != abi.WC_OK:
                raise OracleError(st, lib().or_last_error().decode())
            self._handle = out
        return self._handle

    def check(self):
        """Create the engine now, raising where the reference's builders would panic."""
        self._h()
        return self

    def step(self, s: State, dt: float) -> None:
        t = C.c_double(s.time)
        lib().or_step(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), abi.dptr(s.breaking), C.byref(t), float(dt))
        s.time = t.value

    def stable_dt(self, s: State) -> float:
        return lib().or_stable_dt(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv))

    def limiting_cell(self, s: State):
        out = abi.wc_limiting()
        if not lib().or_limiting_cell(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), C.byref(out)):
            return None
        return Limiting(out.i, out.j, out.depth, out.speed)

    def breaking_indicator(self, s: State) -> np.ndarray:
        out = np.zeros(self.grid.nx * self.grid.ny)
        lib().or_breaking_indicator(
            self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), abi.dptr(s.breaking), abi.dptr(out)
        )
        return out

    def follow_breaking(self, s: State, dt: float) -> int:
        """solver.rs:509-532 on `s` in place; returns the viscous sub-steps taken."""
        return lib().or_follow_breaking(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv),
                                        abi.dptr(s.breaking), float(dt))

    def dispersion_stats(self):
        st = abi.wc_stats()
        if not lib().or_dispersion_stats(self._h(), C.byref(st)):
            return None
        return DispersionStats(st.solves, st.iterations, st.unconverged)

    def drive(self):
        om, ky, stg = C.c_double(), C.c_double(), C.c_double()
        if not lib().or_drive(self._h(), C.byref(om), C.byref(ky), C.byref(stg)):
            return None
        return om.value, ky.value, stg.value


# ---- pieces of the reference exposed for its unit tests -------------------------------------


def face_values(v, blend):
    v = np.ascontiguousarray(v, dtype=np.float64)
    lo, hi = C.c_double(), C.c_double()
    lib().or_face_values(abi.dptr(v), float(blend), C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def smoothstep(lo, hi, x):
    return lib().or_smoothstep(lo, hi, x)


def linear_wave(omega, h, dispersive):
    k, c, cg = C.c_double(), C.c_double(), C.c_double()
    st = lib().or_linear_wave(omega, h, int(dispersive), C.byref(k), C.byref(c), C.byref(cg))
    if st != abi.WC_OK:
        raise OracleError(st, lib().or_last_error().decode())
    return k.value, c.value, cg.value


def manning_factor(h, speed, dt, n):
    return lib().or_manning_factor(h, speed, dt, n)


def matvec(grid, periodic, heff, mask, c, px, py):
    """A p of dispersion.rs:269-317; px/py are copied (their ghosts get filled)."""
    px = np.array(px, dtype=np.float64)
    py = np.array(py, dtype=np.float64)
    ax = np.zeros(grid.cells())
    ay = np.zeros(grid.cells())
    g = grid.to_c()
    lib().or_matvec(
        C.byref(g), int(periodic), abi.dptr(np.ascontiguousarray(heff)), abi.dptr(np.ascontiguousarray(mask)),
        abi.dptr(np.ascontiguousarray(c)), abi.dptr(px), abi.dptr(py), abi.dptr(ax), abi.dptr(ay),
    )
    return ax, ay


def true_relative_residual(grid, periodic, system) -> float:
    """||b - A w||_2 / ||b||_2 in FP64 (dispersion.rs:269-317 for A) of a system given as (ny, nx)
    arrays c, heff, bx, by, wx, wy, e.g. a device solve's (`Solver.dispersion_system`). The ring
    of c outside the interior follows the boundaries (mirrored at walls, wrapped when periodic),
    as the reference's c, computed from ghost-filled depths, does; a cell takes part where its
    FP32 heff is at least 0.05, as on the device. Compared with the recursively updated residual
    the stopping rule reads, this is the residual of the stored solution itself."""
    def padded(a):
        out = np.zeros(grid.cells())
        grid.inner(out)[:] = a
        return out

    c = padded(system["c"])
    mirror_ghosts(grid, c)
    if periodic:
        wrap_ghosts_y(grid, c)
    heff = padded(system["heff"])
    mask = padded((np.asarray(system["heff"], dtype=np.float32) >= np.float32(0.05)).astype(np.float64))
    ax, ay = matvec(grid, periodic, heff, mask, c, padded(system["wx"]), padded(system["wy"]))
    rx = np.asarray(system["bx"]) - grid.inner(ax)
    ry = np.asarray(system["by"]) - grid.inner(ay)
    nb = math.sqrt(float(np.sum(np.square(system["bx"])) + np.sum(np.square(system["by"]))))
    return math.sqrt(float(np.sum(rx * rx) + np.sum(ry * ry))) / nb if nb > 0 else 0.0


def pcg_solve(grid, periodic, system, tolerance, max_iterations, w0=None):
    """The reference's Jacobi PCG (dispersion.rs:440-545) in FP64 on a given system (the (ny, nx)
    arrays c, heff, bx, by of `true_relative_residual`), from w0 (zero if None) with its stopping
    rule ||r|| <= tol ||b|| + 1e-10. Returns (wx, wy, iterations, converged)."""
    def padded(a):
        out = np.zeros(grid.cells())
        grid.inner(out)[:] = a
        return out

    c = padded(system["c"])
    mirror_ghosts(grid, c)
    if periodic:
        wrap_ghosts_y(grid, c)
    heff_i = np.asarray(system["heff"], dtype=np.float64)
    m_i = (np.asarray(system["heff"], dtype=np.float32) >= np.float32(0.05)).astype(np.float64)
    heff, mask = padded(heff_i), padded(m_i)
    cv = grid.view(c)
    g3 = 3
    ci = cv[g3:g3 + grid.ny, g3:g3 + grid.nx]
    q = 0.25 / (grid.dx * grid.dx)
    dgx = np.where(m_i > 0, heff_i + (cv[g3:g3 + grid.ny, g3 + 1:g3 + grid.nx + 1] + cv[g3:g3 + grid.ny, g3 - 1:g3 + grid.nx - 1]) * q, 1.0)
    q = 0.25 / (grid.dy * grid.dy)
    dgy = np.where(m_i > 0, heff_i + (cv[g3 + 1:g3 + grid.ny + 1, g3:g3 + grid.nx] + cv[g3 - 1:g3 + grid.ny - 1, g3:g3 + grid.nx]) * q, 1.0)
    del ci
    bx, by = np.asarray(system["bx"], dtype=np.float64), np.asarray(system["by"], dtype=np.float64)
    wx = np.zeros_like(bx) if w0 is None else np.array(w0[0], dtype=np.float64) * m_i
    wy = np.zeros_like(by) if w0 is None else np.array(w0[1], dtype=np.float64) * m_i

    def A(px, py):
        ax, ay = matvec(grid, periodic, heff, mask, c, padded(px), padded(py))
        return grid.inner(ax).copy(), grid.inner(ay).copy()

    ax, ay = A(wx, wy)
    rx, ry = bx - ax, by - ay
    zx, zy = rx / dgx, ry / dgy
    px, py = zx.copy(), zy.copy()
    target = math.sqrt(float(np.sum(bx * bx) + np.sum(by * by))) * tolerance + 1e-10
    rz = float(np.sum(rx * zx) + np.sum(ry * zy))
    it = 0
    converged = math.sqrt(float(np.sum(rx * rx) + np.sum(ry * ry))) <= target
    while not converged and it < max_iterations:
        ax, ay = A(px, py)
        alpha = rz / float(np.sum(px * ax) + np.sum(py * ay))
        wx += alpha * px
        wy += alpha * py
        rx -= alpha * ax
        ry -= alpha * ay
        zx, zy = rx / dgx, ry / dgy
        it += 1
        converged = math.sqrt(float(np.sum(rx * rx) + np.sum(ry * ry))) <= target
        rz_next = float(np.sum(rx * zx) + np.sum(ry * zy))
        beta = rz_next / rz
        rz = rz_next
        px, py = zx + beta * px, zy + beta * py
    return wx, wy, it, converged


def diagnostics(grid, s: State):
    """(volume, max |momentum|, min depth) of a state: state.rs:78-102 (or_volume,
    or_max_abs_momentum, or_min_depth)."""
    g = grid.to_c()
    L = lib()
    return (L.or_volume(C.byref(g), abi.dptr(s.h)), L.or_max_abs_momentum(C.byref(g), abi.dptr(s.hu), abi.dptr(s.hv)),
            L.or_min_depth(C.byref(g), abi.dptr(s.h)))


def dot(grid, ax, ay, bx, by):
    g = grid.to_c()
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (ax, ay, bx, by)]
    return lib().or_dot(C.byref(g), *[abi.dptr(a) for a in arrs])


def dispersion_apply(grid, periodic, dispersion, s: State, lh, lhu, lhv, phi):
    g = grid.to_c()
    d = dispersion.to_c()
    lhu = np.array(lhu, dtype=np.float64)
    lhv = np.array(lhv, dtype=np.float64)
    lib().or_dispersion_apply(
        C.byref(g), int(periodic), C.byref(d), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv),
        abi.dptr(np.ascontiguousarray(lh, dtype=np.float64)), abi.dptr(lhu), abi.dptr(lhv),
        abi.dptr(np.ascontiguousarray(phi, dtype=np.float64)),
    )
    return lhu, lhv


def mirror_ghosts(grid, a):
    g = grid.to_c()
    lib().or_mirror_ghosts(C.byref(g), abi.dptr(a))


def wrap_ghosts_y(grid, a):
    g = grid.to_c()
    lib().or_wrap_ghosts_y(C.byref(g), abi.dptr(a))


def eddy_threshold(eddy, age, h):
    """eddy.rs:114-124."""
    e = eddy.to_c()
    return lib().or_eddy_threshold(C.byref(e), float(age), float(h))


def eddy_follow(grid, eddy, s: State, phi, dt):
    """eddy.rs:155-219 on a ghost-filled state: replaces s.breaking; returns nu (padded)."""
    g, e = grid.to_c(), eddy.to_c()
    nu = np.zeros(grid.cells())
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    lib().or_eddy_follow(C.byref(g), C.byref(e), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv),
                         abi.dptr(s.breaking), abi.dptr(phi), float(dt), abi.dptr(nu))
    return nu


def eddy_diffuse(grid, s: State, nu, dt, periodic=False):
    """eddy.rs:221-302 on `s` in place; returns the sub-steps taken."""
    g = grid.to_c()
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    return lib().or_eddy_diffuse(C.byref(g), int(periodic), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv),
                                 abi.dptr(s.breaking), abi.dptr(nu), float(dt))
