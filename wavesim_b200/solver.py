"""`Solver`: wavecore's solver API over the device library (include/wavecore_c.h).

The step runs only on the GPU, in `libwavecore_b200.so`; there is no CPU path. If the library or
a CUDA device is missing, creating a solver raises.

Builders follow the reference (`Solver::new(grid, bed).with_order(..).with_dispersion(..)`,
crates/wavecore/src/solver.rs:283-419); `step`, `stable_dt`, `limiting_cell`,
`breaking_indicator` and `dispersion_stats` take and return host FP64 arrays like the reference.
The device-resident methods (`upload`, `step_device`, `step_n`, `download`, ...) are the
throughput path and have no counterpart in the reference.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import warnings

import numpy as np

from . import abi
from .model import DispersionStats, Limiting, SolverConfig, State

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwavecore_b200.so")
_lib = None

EXPORTS = [
    "wc_config_default",
    "wc_dispersion_default",
    "wc_eddy_default",
    "wc_solver_create",
    "wc_solver_destroy",
    "wc_step",
    "wc_stable_dt",
    "wc_limiting_cell",
    "wc_breaking_indicator",
    "wc_dispersion_stats",
    "wc_state_upload",
    "wc_state_download",
    "wc_breaking_upload",
    "wc_breaking_download",
    "wc_follow_breaking",
    "wc_step_device",
    "wc_step_n",
    "wc_stable_dt_device",
    "wc_diagnostics_device",
    "wc_dispersion_system",
    "wc_time_device",
    "wc_synchronize",
    "wc_set_stream",
    "wc_set_wait_limit",
    "wc_profile_enable",
    "wc_profile_read",
    "wc_launch_count",
    "wc_last_error",
    "wc_stable_dt_noalloc",
    "wc_ensemble_create",
    "wc_ensemble_destroy",
    "wc_ensemble_upload",
    "wc_ensemble_download",
    "wc_ensemble_step_n",
    "wc_ensemble_autotune",
    "wc_ensemble_set_lpc",
    "wc_ensemble_synchronize",
    "wc_ensemble_member_stats",
    "wc_ensemble_launch_count",
    "wc_lpc_create",
    "wc_lpc_destroy",
    "wc_lpc_num_params",
    "wc_lpc_set_params",
    "wc_lpc_get_params",
    "wc_lpc_set_rounding",
    "wc_lpc_forward_backward",
    "wc_lpc_loss_grad",
    "wc_lpc_forward",
    "wc_lpc_harvest",
    "wc_lpc_num_systems",
    "wc_lpc_train",
    "wc_solver_set_lpc",
    "wc_recorder_create",
    "wc_recorder_destroy",
    "wc_recorder_read",
    "wc_frame",
    "wc_nest_create",
    "wc_nest_destroy",
    "wc_nest_cells",
    "wc_nest_sample",
    "wc_nest_step",
]


class WavecoreError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def load(path: str = LIB_PATH):
    """Load the device library (it must have been built: `python -m wavesim_b200.build`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m wavesim_b200.build` (there is no CPU fallback)"
        )
    L = C.CDLL(path)
    D = abi.DPTR
    V = C.c_void_p
    L.wc_config_default.argtypes = [C.POINTER(abi.wc_config)]
    L.wc_dispersion_default.argtypes = [C.POINTER(abi.wc_dispersion)]
    L.wc_solver_create.argtypes = [C.POINTER(abi.wc_grid), D, C.POINTER(abi.wc_config), C.POINTER(V)]
    L.wc_solver_destroy.argtypes = [V]
    L.wc_step.argtypes = [V, D, D, D, D, D, C.c_double]
    L.wc_stable_dt.argtypes = [V, D, D, D, D]
    L.wc_limiting_cell.argtypes = [V, D, D, D, C.POINTER(abi.wc_limiting), C.POINTER(C.c_int32)]
    L.wc_breaking_indicator.argtypes = [V, D, D, D, D, D]
    L.wc_eddy_default.argtypes = [C.POINTER(abi.wc_eddy)]
    L.wc_eddy_default.restype = None
    L.wc_breaking_upload.argtypes = [V, D]
    L.wc_breaking_download.argtypes = [V, D]
    L.wc_follow_breaking.argtypes = [V, D, D, D, D, C.c_double, C.POINTER(C.c_int32)]
    L.wc_dispersion_stats.argtypes = [V, C.POINTER(abi.wc_stats), C.POINTER(C.c_int32)]
    L.wc_state_upload.argtypes = [V, D, D, D, C.c_double]
    L.wc_state_download.argtypes = [V, D, D, D, D]
    L.wc_step_device.argtypes = [V, C.c_double]
    L.wc_step_n.argtypes = [V, C.c_uint64, C.c_double]
    L.wc_stable_dt_device.argtypes = [V, D]
    L.wc_diagnostics_device.argtypes = [V, C.POINTER(abi.wc_diagnostics)]
    L.wc_dispersion_system.argtypes = [V, D, D, D, D, D, D]
    L.wc_time_device.argtypes = [V, D]
    L.wc_synchronize.argtypes = [V]
    L.wc_set_stream.argtypes = [V, V]
    L.wc_set_wait_limit.argtypes = [V, C.c_uint64]
    L.wc_profile_enable.argtypes = [V, C.c_int32]
    L.wc_profile_read.argtypes = [V, C.POINTER(abi.wc_kernel_time)]
    L.wc_ensemble_create.argtypes = [C.c_uint64, C.POINTER(abi.wc_grid), C.POINTER(D), C.POINTER(abi.wc_config), C.POINTER(V)]
    L.wc_ensemble_destroy.argtypes = [V]
    L.wc_ensemble_destroy.restype = None
    L.wc_ensemble_upload.argtypes = [V, C.c_uint64, D, D, D, C.c_double]
    L.wc_ensemble_download.argtypes = [V, C.c_uint64, D, D, D, D]
    L.wc_ensemble_step_n.argtypes = [V, C.c_uint64, C.c_double]
    L.wc_ensemble_autotune.argtypes = [V, C.c_uint32, C.POINTER(C.c_int32), D]
    L.wc_ensemble_synchronize.argtypes = [V]
    L.wc_ensemble_set_lpc.argtypes = [V, V]
    L.wc_ensemble_member_stats.argtypes = [V, C.c_uint64, C.POINTER(abi.wc_stats), D]
    L.wc_ensemble_launch_count.argtypes = [V]
    L.wc_ensemble_launch_count.restype = C.c_uint64
    for name in ("wc_ensemble_create", "wc_ensemble_upload", "wc_ensemble_download", "wc_ensemble_step_n",
                 "wc_ensemble_autotune", "wc_ensemble_synchronize", "wc_ensemble_member_stats",
                 "wc_ensemble_set_lpc"):
        getattr(L, name).restype = C.c_int
    L.wc_stable_dt_noalloc.argtypes = [C.POINTER(abi.wc_grid), C.c_double, V, V, V, V, D]
    L.wc_stable_dt_noalloc.restype = C.c_int
    F = C.POINTER(C.c_float)
    L.wc_lpc_create.argtypes = [C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.c_uint64, C.POINTER(V)]
    L.wc_lpc_destroy.argtypes = [V]
    L.wc_lpc_destroy.restype = None
    L.wc_lpc_num_params.argtypes = [V]
    L.wc_lpc_num_params.restype = C.c_uint64
    L.wc_lpc_set_params.argtypes = [V, F, C.c_uint64]
    L.wc_lpc_get_params.argtypes = [V, F, C.c_uint64]
    L.wc_lpc_set_rounding.argtypes = [V, C.c_int32]
    L.wc_lpc_forward_backward.argtypes = [V, C.c_int32, C.c_int32, C.c_int32, F, F, F, F, F, F]
    L.wc_lpc_loss_grad.argtypes = [V, C.c_int32, C.c_int32, C.c_int32, F, F, F, F, C.c_double, C.c_double, D, F]
    L.wc_lpc_forward.argtypes = [V, C.c_int32, C.c_int32, C.c_int32, F, F, C.c_int32, F]
    L.wc_lpc_harvest.argtypes = [V, V]
    L.wc_lpc_num_systems.argtypes = [V]
    L.wc_lpc_num_systems.restype = C.c_uint64
    L.wc_lpc_train.argtypes = [V, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_uint64, D]
    L.wc_solver_set_lpc.argtypes = [V, V]
    for name in ("wc_lpc_create", "wc_lpc_set_params", "wc_lpc_get_params", "wc_lpc_set_rounding",
                 "wc_lpc_forward_backward", "wc_lpc_loss_grad", "wc_lpc_forward", "wc_lpc_harvest", "wc_lpc_train",
                 "wc_solver_set_lpc"):
        getattr(L, name).restype = C.c_int
    L.wc_recorder_create.argtypes = [V, C.c_double, C.c_double, C.POINTER(V)]
    L.wc_recorder_destroy.argtypes = [V]
    L.wc_recorder_destroy.restype = None
    L.wc_recorder_read.argtypes = [V, C.POINTER(abi.wc_record_summary), D, D, D, D, D]
    L.wc_frame.argtypes = [V, C.c_double, F, F, D]
    for name in ("wc_recorder_create", "wc_recorder_read", "wc_frame"):
        getattr(L, name).restype = C.c_int
    L.wc_nest_create.argtypes = [V, V, C.POINTER(abi.wc_sponge), C.c_uint64, C.c_double, C.c_double, C.POINTER(V)]
    L.wc_nest_destroy.argtypes = [V]
    L.wc_nest_destroy.restype = None
    L.wc_nest_cells.argtypes = [V]
    L.wc_nest_cells.restype = C.c_uint64
    L.wc_nest_sample.argtypes = [V, C.c_int32]
    L.wc_nest_step.argtypes = [V, C.c_double]
    for name in ("wc_nest_create", "wc_nest_sample", "wc_nest_step"):
        getattr(L, name).restype = C.c_int
    L.wc_launch_count.argtypes = [V]
    L.wc_launch_count.restype = C.c_uint64
    L.wc_last_error.restype = C.c_char_p
    for name in (
        "wc_solver_create", "wc_step", "wc_stable_dt", "wc_limiting_cell", "wc_breaking_indicator",
        "wc_dispersion_stats", "wc_state_upload", "wc_state_download", "wc_step_device", "wc_step_n",
        "wc_stable_dt_device", "wc_diagnostics_device", "wc_dispersion_system", "wc_time_device", "wc_synchronize",
        "wc_set_stream", "wc_set_wait_limit", "wc_profile_enable", "wc_profile_read", "wc_breaking_upload", "wc_breaking_download",
        "wc_follow_breaking",
    ):
        getattr(L, name).restype = C.c_int
    L.wc_config_default.restype = None
    L.wc_dispersion_default.restype = None
    L.wc_solver_destroy.restype = None
    _lib = L
    return L


def _check(status: int, allow=(abi.WC_OK,)):
    if status in allow:
        return status
    if status == abi.WC_EUNCONVERGED:
        warnings.warn(load().wc_last_error().decode(), RuntimeWarning, stacklevel=3)
        return status
    raise WavecoreError(status, load().wc_last_error().decode())


def stable_dt_noalloc(grid, cfl: float, d_h: int, d_hu: int, d_hv: int, stream: int = 0) -> float:
    """`wc_stable_dt_noalloc`: the time-step limit of a state held in the caller's device memory
    (padded FP64 arrays given as device addresses), computed without allocating anything. For
    callers whose device memory all belongs to their own allocator, or that must not allocate per
    step. The call waits on `stream` and returns the result on the host."""
    g = grid.to_c()
    out = C.c_double()
    _check(
        load().wc_stable_dt_noalloc(C.byref(g), float(cfl), C.c_void_p(d_h), C.c_void_p(d_hu), C.c_void_p(d_hv),
                                    C.c_void_p(stream or None), C.byref(out)),
        allow=(abi.WC_OK, abi.WC_ENAN),
    )
    return out.value


class Solver(SolverConfig):
    """wavecore's `Solver` (solver.rs:260-733) on a B200."""

    def _release(self):
        if getattr(self, "_handle", None):
            load().wc_solver_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    def _h(self):
        if self._handle is None:
            L = load()
            cfg, keep = self._c_config()
            g = self.grid.to_c()
            out = C.c_void_p()
            _check(L.wc_solver_create(C.byref(g), abi.dptr(self.bed.b), C.byref(cfg), C.byref(out)))
            self._handle = out
        return self._handle

    def check(self):
        """Create the device solver now, raising where the reference's builders would panic."""
        self._h()
        return self

    # ---- the reference's host-array API -------------------------------------------------

    def step(self, s: State, dt: float) -> None:
        """solver.rs:479-507: one step of size dt, in place on the host state."""
        t = C.c_double(s.time)
        _check(
            load().wc_step(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), abi.dptr(s.breaking), C.byref(t), float(dt))
        )
        s.time = t.value

    def stable_dt(self, s: State) -> float:
        """solver.rs:431-450 (NaN when a cell is not a number, inf when nothing moves)."""
        out = C.c_double()
        _check(load().wc_stable_dt(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), C.byref(out)),
               allow=(abi.WC_OK, abi.WC_ENAN))
        return out.value

    def limiting_cell(self, s: State):
        """solver.rs:452-477."""
        out = abi.wc_limiting()
        found = C.c_int32()
        _check(load().wc_limiting_cell(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), C.byref(out), C.byref(found)))
        if not found.value:
            return None
        return Limiting(out.i, out.j, out.depth, out.speed)

    def breaking_indicator(self, s: State) -> np.ndarray:
        """solver.rs:336-349: nx*ny values, y outer."""
        out = np.zeros(self.grid.nx * self.grid.ny)
        _check(load().wc_breaking_indicator(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv),
                                            abi.dptr(s.breaking), abi.dptr(out)))
        return out

    def follow_breaking(self, s: State, dt: float) -> int:
        """solver.rs:509-532 (private in the reference, exported for parity checks of eddy.rs):
        the fronts in s.breaking followed on to the state and their eddy viscosity applied over
        dt, in place. Returns the viscous sub-steps taken; a no-op without followed fronts."""
        n = C.c_int32()
        _check(load().wc_follow_breaking(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv),
                                         abi.dptr(s.breaking), float(dt), C.byref(n)))
        return n.value

    def dispersion_stats(self):
        """solver.rs:391-396."""
        st = abi.wc_stats()
        has = C.c_int32()
        _check(load().wc_dispersion_stats(self._h(), C.byref(st), C.byref(has)))
        if not has.value:
            return None
        return DispersionStats(st.solves, st.iterations, st.unconverged)

    # ---- the device-resident throughput path --------------------------------------------

    def upload(self, s: State) -> None:
        """The state onto the device, its breaking memory included (kept only with followed
        fronts)."""
        _check(load().wc_state_upload(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), float(s.time)))
        _check(load().wc_breaking_upload(self._h(), abi.dptr(s.breaking)))

    def download(self, s: State) -> None:
        t = C.c_double()
        _check(load().wc_state_download(self._h(), abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), C.byref(t)))
        if self.follows_fronts:  # otherwise the memory is carried unchanged, as a step does
            _check(load().wc_breaking_download(self._h(), abi.dptr(s.breaking)))
        s.time = t.value

    @property
    def follows_fronts(self) -> bool:
        """Breaking::viscosity is set (and read: only with dispersion, solver.rs:512-518)."""
        d = self.dispersion()
        return d is not None and d.breaking.viscosity is not None

    def step_device(self, dt: float) -> None:
        _check(load().wc_step_device(self._h(), float(dt)))

    def step_n(self, n: int, t_end: float = math.inf) -> None:
        _check(load().wc_step_n(self._h(), int(n), float(t_end)))

    def set_stream(self, stream_handle: int) -> None:
        """Queue work on the caller's CUDA stream (an integer cudaStream_t; 0 = own stream)."""
        _check(load().wc_set_stream(self._h(), C.c_void_p(int(stream_handle) or None)))

    def profile(self, on: bool) -> None:
        """Start (clearing earlier records) or stop per-kernel device timing."""
        _check(load().wc_profile_enable(self._h(), int(bool(on))))

    def profile_read(self) -> dict:
        """{kind: (launches, total device ms)} since profiling was enabled."""
        out = (abi.wc_kernel_time * len(abi.KERNEL_KINDS))()
        _check(load().wc_profile_read(self._h(), out))
        return {abi.KERNEL_KINDS[k]: (int(out[k].launches), float(out[k].total_ms)) for k in range(len(abi.KERNEL_KINDS))}

    def synchronize(self) -> None:
        _check(load().wc_synchronize(self._h()))

    def stable_dt_device(self) -> float:
        out = C.c_double()
        _check(load().wc_stable_dt_device(self._h(), C.byref(out)), allow=(abi.WC_OK, abi.WC_ENAN))
        return out.value

    def diagnostics_device(self):
        d = abi.wc_diagnostics()
        _check(load().wc_diagnostics_device(self._h(), C.byref(d)))
        return d.volume, d.max_abs_momentum, d.min_depth

    def set_wait_limit(self, ns: int) -> None:
        """`wc_set_wait_limit`: the limit of the persistent kernels' bounded waits (0: 2 s)."""
        _check(load().wc_set_wait_limit(self._h(), int(ns)))

    def dispersion_system(self) -> dict:
        """The last dispersive solve's system and solution as the device holds them
        (`wc_dispersion_system`): (ny, nx) FP64 arrays c, heff, bx, by, wx, wy."""
        g = self.grid
        out = {k: np.zeros((g.ny, g.nx)) for k in ("c", "heff", "bx", "by", "wx", "wy")}
        _check(load().wc_dispersion_system(self._h(), *(abi.dptr(out[k]) for k in ("c", "heff", "bx", "by", "wx", "wy"))))
        return out

    def time_device(self) -> float:
        t = C.c_double()
        _check(load().wc_time_device(self._h(), C.byref(t)))
        return t.value

    def frame(self, tide: float = 0.0):
        """A frame of the resident state (crates/wavesim/src/lib.rs:1348-1380): eta and the
        breaking indicator, FP32 (ny, nx), and the highest surface above `tide` over wet cells.
        Raises when the surface is not finite or more than 100 m up (the driver's Unstable)."""
        n = self.grid.nx * self.grid.ny
        eta = np.zeros(n, dtype=np.float32)
        brk = np.zeros(n, dtype=np.float32)
        rise = C.c_double()
        _check(load().wc_frame(self._h(), float(tide), _fptr(eta), _fptr(brk), C.byref(rise)))
        shape = (self.grid.ny, self.grid.nx)
        return eta.reshape(shape), brk.reshape(shape), rise.value

    def set_preconditioner(self, net: "LearnedPreconditioner | None") -> None:
        """Attach a trained network (learned-preconditioned flexible CG) or detach it (None:
        Jacobi PCG, the reference's method)."""
        _check(load().wc_solver_set_lpc(self._h(), net._handle if net is not None else None))
        self._lpc = net  # keep it alive while attached

    def launch_count(self) -> int:
        return int(load().wc_launch_count(self._h()))


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_float))


class LearnedPreconditioner:
    """The network preconditioner of the dispersive solve (`wc_lpc_*`; no counterpart in the
    reference, whose solve is Jacobi-preconditioned CG, dispersion.rs:493-545).

    Its parameter layout is `lpc.UNetSpec`; it is trained on the GPU on SGN systems harvested
    from solvers (`harvest`, `train`) and attached to a solver with `Solver.set_preconditioner`.
    It must outlive the solvers it is attached to (a solver keeps a reference)."""

    def __init__(self, spec=None, seed: int = 0):
        from .lpc import UNetSpec

        self.spec = spec or UNetSpec()
        ch = (C.c_int32 * 4)(*self.spec.channels)
        out = C.c_void_p()
        _check(load().wc_lpc_create(ch, int(self.spec.gate_hidden), int(self.spec.stride), int(seed), C.byref(out)))
        self._handle = out

    def __del__(self):
        try:
            if getattr(self, "_handle", None):
                load().wc_lpc_destroy(self._handle)
            self._handle = None
        except Exception:
            pass

    @property
    def n_params(self) -> int:
        return int(load().wc_lpc_num_params(self._handle))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        _check(load().wc_lpc_get_params(self._handle, _fptr(p), p.size))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(load().wc_lpc_set_params(self._handle, _fptr(p), p.size))

    def set_rounding(self, bf16: bool) -> None:
        _check(load().wc_lpc_set_rounding(self._handle, 1 if bf16 else 0))

    def forward_backward(self, x, feat, dy):
        """(y, parameter gradient, input gradient) of one pass on [n][2][h][w] arrays."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        feat = np.ascontiguousarray(feat, dtype=np.float32)
        dy = np.ascontiguousarray(dy, dtype=np.float32)
        n, c, h, w = x.shape
        assert c == 2 and feat.shape == x.shape and dy.shape == x.shape
        y = np.zeros_like(x)
        dx = np.zeros_like(x)
        g = np.zeros(self.n_params, dtype=np.float32)
        _check(load().wc_lpc_forward_backward(self._handle, n, h, w, _fptr(x), _fptr(feat), _fptr(dy), _fptr(y),
                                              _fptr(g), _fptr(dx)))
        return y, g, dx

    def forward(self, x, feat, tensor: bool = True, fused: bool = True, small_tiles: bool = True):
        """The network's output on [n][2][h][w] arrays: BF16 tensor-core inference (as the solver
        applies it; `fused=False` runs the first level one launch per layer, `small_tiles=False`
        keeps the coarse levels' 32-channel layers on tiles of their usual height) or the FP32
        path training uses."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        feat = np.ascontiguousarray(feat, dtype=np.float32)
        n, c, h, w = x.shape
        y = np.zeros_like(x)
        mode = (1 if small_tiles else 3) if fused else 2
        mode = mode if tensor else 0
        _check(load().wc_lpc_forward(self._handle, n, h, w, _fptr(x), _fptr(feat), mode, _fptr(y)))
        return y

    def loss_grad(self, c, heff, bed, e, dx: float, dy: float):
        """The training loss of patches (c, heff, bed: [n][h][w]; error fields e: [n][2][h][w])
        and its parameter gradient."""
        c, heff, bed, e = (np.ascontiguousarray(a, dtype=np.float32) for a in (c, heff, bed, e))
        n, h, w = c.shape
        assert heff.shape == c.shape and bed.shape == c.shape and e.shape == (n, 2, h, w)
        loss = C.c_double()
        g = np.zeros(self.n_params, dtype=np.float32)
        _check(load().wc_lpc_loss_grad(self._handle, n, h, w, _fptr(c), _fptr(heff), _fptr(bed), _fptr(e), float(dx),
                                       float(dy), C.byref(loss), _fptr(g)))
        return loss.value, g

    def harvest(self, solver: "Solver") -> None:
        """Keep the solver's current SGN system (that of its last solve) for training."""
        _check(load().wc_lpc_harvest(self._handle, solver._h()))

    @property
    def n_systems(self) -> int:
        return int(load().wc_lpc_num_systems(self._handle))

    def train(self, steps: int, batch: int = 16, patch: int = 64, lr: float = 2e-3, rough: float = 1.0,
              seed: int = 0) -> np.ndarray:
        """Adam steps on random patches of the harvested systems; returns every step's loss."""
        losses = np.zeros(max(int(steps), 1), dtype=np.float64)
        _check(load().wc_lpc_train(self._handle, int(steps), int(batch), int(patch), float(lr), float(rough),
                                   int(seed), abi.dptr(losses)))
        return losses[: int(steps)]

    def save(self, path: str) -> None:
        np.save(path, self.get_params())

    @classmethod
    def load_params(cls, path: str, spec=None):
        net = cls(spec)
        net.set_params(np.load(path))
        return net


class Recorder:
    """Per-step statistics of a solver's run (`wc_recorder_*`): the reference driver's
    `Stage::record` (crates/wavesim/src/lib.rs:1276-1301) kept on the device. Every step the solver
    takes after this is created (host arrays or device-resident) is recorded."""

    def __init__(self, solver: "Solver", start_from: float, period: float):
        out = C.c_void_p()
        _check(load().wc_recorder_create(solver._h(), float(start_from), float(period), C.byref(out)))
        self._handle = out
        self._solver = solver  # the solver must outlive the recorder
        self.grid = solver.grid

    def close(self):
        if getattr(self, "_handle", None):
            load().wc_recorder_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def read(self) -> dict:
        """seconds, waves, unsettled (or None) and the per-cell (ny, nx) arrays eta_max, eta_min,
        wave_height (None before a whole wave), breaking_fraction and harmonic (complex a - ib,
        or None while the samples cannot separate it)."""
        n = self.grid.nx * self.grid.ny
        arrs = {k: np.zeros(n) for k in ("eta_max", "eta_min", "wave_height", "breaking_fraction")}
        harm = np.zeros(2 * n)
        sm = abi.wc_record_summary()
        _check(load().wc_recorder_read(self._handle, C.byref(sm), *(abi.dptr(arrs[k]) for k in
                                       ("eta_max", "eta_min", "wave_height", "breaking_fraction")), abi.dptr(harm)))
        shape = (self.grid.ny, self.grid.nx)
        out = {k: v.reshape(shape) for k, v in arrs.items()}
        if sm.waves == 0:
            out["wave_height"] = None
        out["harmonic"] = (harm[0::2] + 1j * harm[1::2]).reshape(shape) if sm.has_harmonic else None
        out["seconds"] = sm.seconds
        out["waves"] = int(sm.waves)
        out["unsettled"] = sm.unsettled if sm.has_unsettled else None
        return out


class Nest:
    """One-way nesting (`wc_nest_*`): the fine solver's relaxation zones pulled towards a coarser
    run of the same sea, as the reference's driver does (crates/wavesim/src/lib.rs:1846-1896).
    Both solvers keep their states on the device; `run` is the driver's loop."""

    def __init__(self, fine: "Solver", coarse: "Solver", zones, x_offset_m: float = 0.0, y_offset_m: float = 0.0):
        arr = (abi.wc_sponge * max(1, len(zones)))(*[z.to_c() for z in zones])
        out = C.c_void_p()
        _check(load().wc_nest_create(fine._h(), coarse._h(), arr, len(zones), float(x_offset_m), float(y_offset_m),
                                     C.byref(out)))
        self._handle = out
        self.fine, self.coarse = fine, coarse

    def close(self):
        if getattr(self, "_handle", None):
            load().wc_nest_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def cells(self) -> int:
        return int(load().wc_nest_cells(self._handle))

    def sample(self, slot: int) -> None:
        _check(load().wc_nest_sample(self._handle, int(slot)))

    def step(self, dt: float) -> None:
        _check(load().wc_nest_step(self._handle, float(dt)))

    def run(self, fine_dts, coarse_dt) -> None:
        """lib.rs:1846-1896: for each fine step, step the coarse run (by `coarse_dt(t)`, a function
        of its time) until it brackets the step's end, sample the states around that end, then
        take the fine step and relax its zones. Uses the device clocks of both solvers."""
        t_fine = self.fine.time_device()
        stepped = False
        for dt in fine_dts:
            end = t_fine + dt
            while self.coarse.time_device() < end - 1e-9:
                self.sample(0)
                self.coarse.step_device(coarse_dt(self.coarse.time_device()))
                stepped = True
            if stepped:
                self.sample(1)
                stepped = False
            self.step(dt)
            t_fine = end


class Ensemble:
    """Independent runs advanced together, one persistent launch per step (`wc_ensemble_*`).

    `members` are configured solvers (`Solver(grid, bed).with_...`); their configuration is
    copied, each member gets its own device state. No counterpart in the reference, which runs one
    `Solver` per grid in turn.
    """

    VARIANTS = ("tile 32x8, 1 CTA/SM", "tile 32x8, 2 CTAs/SM", "tile 32x16, 1 CTA/SM", "tile 32x16, 2 CTAs/SM",
                "members' own step graphs on their own streams")

    def __init__(self, members):
        L = load()
        n = len(members)
        grids = (abi.wc_grid * n)(*[m.grid.to_c() for m in members])
        cfgs, keep = [], []
        for m in members:
            cfg, k = m._c_config()
            cfgs.append(cfg)
            keep.append(k)
        carr = (abi.wc_config * n)(*cfgs)
        beds = (abi.DPTR * n)(*[abi.dptr(m.bed.b) for m in members])
        out = C.c_void_p()
        _check(L.wc_ensemble_create(n, grids, beds, carr, C.byref(out)))
        self._h = out
        self.members = members
        self.n = n

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                load().wc_ensemble_destroy(self._h)
        except Exception:
            pass

    def upload(self, m: int, s: State) -> None:
        _check(load().wc_ensemble_upload(self._h, m, abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), float(s.time)))

    def download(self, m: int, s: State) -> None:
        t = C.c_double()
        _check(load().wc_ensemble_download(self._h, m, abi.dptr(s.h), abi.dptr(s.hu), abi.dptr(s.hv), C.byref(t)))
        s.time = t.value

    def step_n(self, n: int, t_end: float = math.inf) -> None:
        _check(load().wc_ensemble_step_n(self._h, int(n), float(t_end)))

    def set_preconditioner(self, net) -> None:
        """`wc_ensemble_set_lpc`: the learned preconditioner for every dispersive member; each member
        then steps through its own captured step on its own stream (forked and joined every step).
        The network must outlive the ensemble."""
        _check(load().wc_ensemble_set_lpc(self._h, net._handle))
        self._net = net

    def autotune(self, trial_steps: int = 2):
        choice = C.c_int32()
        ms = (C.c_double * 5)()
        _check(load().wc_ensemble_autotune(self._h, int(trial_steps), C.byref(choice), ms))
        return choice.value, list(ms)

    def synchronize(self) -> None:
        _check(load().wc_ensemble_synchronize(self._h))

    def member_stats(self, m: int):
        st = abi.wc_stats()
        t = C.c_double()
        _check(load().wc_ensemble_member_stats(self._h, m, C.byref(st), C.byref(t)))
        return DispersionStats(st.solves, st.iterations, st.unconverged), t.value

    def launch_count(self) -> int:
        return int(load().wc_ensemble_launch_count(self._h))
