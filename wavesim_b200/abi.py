"""ctypes mirror of include/wavecore_c.h (structs, enums, status codes).

Shared by the product binding (`wavesim_b200.solver`) and by the test oracle's binding, so one
configuration struct feeds both libraries.
"""
from __future__ import annotations

import ctypes as C

GHOST = 3

WC_OK = 0
WC_EINVAL = 1
WC_EPERIODIC = 2
WC_ENAN = 3
WC_EUNCONVERGED = 4
WC_ETIMEOUT = 5
WC_ECUDA = 6
WC_ENOMEM = 7
WC_EUNSUPPORTED = 8

STATUS_NAMES = {
    WC_OK: "WC_OK",
    WC_EINVAL: "WC_EINVAL",
    WC_EPERIODIC: "WC_EPERIODIC",
    WC_ENAN: "WC_ENAN",
    WC_EUNCONVERGED: "WC_EUNCONVERGED",
    WC_ETIMEOUT: "WC_ETIMEOUT",
    WC_ECUDA: "WC_ECUDA",
    WC_ENOMEM: "WC_ENOMEM",
    WC_EUNSUPPORTED: "WC_EUNSUPPORTED",
}

WC_PC_JACOBI = 0
WC_PC_LEARNED = 1


class wc_grid(C.Structure):
    _fields_ = [("nx", C.c_uint64), ("ny", C.c_uint64), ("dx", C.c_double), ("dy", C.c_double)]


class wc_sponge(C.Structure):
    _fields_ = [
        ("width", C.c_uint64),
        ("strength", C.c_double),
        ("level", C.c_double),
        ("west", C.c_int32),
        ("east", C.c_int32),
        ("south", C.c_int32),
        ("north", C.c_int32),
    ]


class wc_wavemaker(C.Structure):
    _fields_ = [
        ("x", C.c_double),
        ("amplitude", C.c_double),
        ("period", C.c_double),
        ("angle", C.c_double),
        ("sigma", C.c_double),
        ("ramp_periods", C.c_double),
    ]


class wc_eddy(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("initial", "settled", "duration", "mixing", "linger")]


class wc_breaking(C.Structure):
    _fields_ = [
        ("eta_ratio_lo", C.c_double),
        ("eta_ratio_hi", C.c_double),
        ("slope_lo", C.c_double),
        ("slope_hi", C.c_double),
        ("viscosity", C.c_int32),
        ("eddy", wc_eddy),
    ]


class wc_dispersion(C.Structure):
    _fields_ = [
        ("breaking", wc_breaking),
        ("nonlinear", C.c_int32),
        ("tolerance", C.c_double),
        ("max_iterations", C.c_uint64),
        ("preconditioner", C.c_int32),
    ]


class wc_config(C.Structure):
    _fields_ = [
        ("cfl", C.c_double),
        ("order", C.c_int32),
        ("manning", C.c_double),
        ("periodic_y", C.c_int32),
        ("sponges", C.POINTER(wc_sponge)),
        ("n_sponges", C.c_uint64),
        ("wavemaker", C.POINTER(wc_wavemaker)),
        ("dispersion", C.POINTER(wc_dispersion)),
        ("shallow_cells", C.POINTER(C.c_uint8)),
    ]


class wc_stats(C.Structure):
    _fields_ = [("solves", C.c_uint64), ("iterations", C.c_uint64), ("unconverged", C.c_uint64)]


class wc_limiting(C.Structure):
    _fields_ = [("i", C.c_uint64), ("j", C.c_uint64), ("depth", C.c_double), ("speed", C.c_double)]


class wc_diagnostics(C.Structure):
    _fields_ = [
        ("volume", C.c_double),
        ("max_abs_momentum", C.c_double),
        ("min_depth", C.c_double),
    ]


class wc_kernel_time(C.Structure):
    _fields_ = [("launches", C.c_uint64), ("total_ms", C.c_double)]


KERNEL_KINDS = ("stage", "solve", "other", "network", "eddy")

DPTR = C.POINTER(C.c_double)


def dptr(a):
    """Pointer to the data of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(DPTR)


class wc_record_summary(C.Structure):
    _fields_ = [("seconds", C.c_double), ("waves", C.c_uint64), ("has_harmonic", C.c_int32),
                ("has_unsettled", C.c_int32), ("unsettled", C.c_double)]
