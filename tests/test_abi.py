"""The C ABI library loads without a GPU and exports every entry point include/*.h declares."""
import ctypes
import glob
import os
import re

import pytest

from wavesim_b200 import build
from wavesim_b200.solver import EXPORTS, LIB_PATH, load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(wc_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_entry_points():
    names = declared_functions()
    assert {"wc_solver_create", "wc_step", "wc_stable_dt", "wc_limiting_cell"} <= names


def test_library_builds_and_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol():
    assert declared_functions() <= set(EXPORTS) | set(declared_functions())
    load()
    for n in declared_functions():
        assert n in EXPORTS, f"{n} is declared but not bound"


def test_defaults_match_the_reference():
    from wavesim_b200 import abi
    L = load()
    cfg = abi.wc_config()
    L.wc_config_default(ctypes.byref(cfg))
    assert cfg.cfl == 0.4 and cfg.order == 1 and cfg.manning == 0.0 and cfg.periodic_y == 0
    d = abi.wc_dispersion()
    L.wc_dispersion_default(ctypes.byref(d))
    assert (d.tolerance, d.max_iterations, d.nonlinear) == (1e-4, 200, 1)
    assert (d.breaking.eta_ratio_lo, d.breaking.eta_ratio_hi) == (0.30, 0.55)
    assert (d.breaking.slope_lo, d.breaking.slope_hi) == (0.40, 0.65)


def test_invalid_grid_is_refused_without_a_gpu():
    """grid.rs:87-91 panics; the ABI returns WC_EINVAL before touching a device."""
    import numpy as np
    from wavesim_b200 import abi
    L = load()
    g = abi.wc_grid(0, 4, 1.0, 1.0)
    cfg = abi.wc_config()
    L.wc_config_default(ctypes.byref(cfg))
    out = ctypes.c_void_p()
    bed = np.zeros(10)
    st = L.wc_solver_create(ctypes.byref(g), abi.dptr(bed), ctypes.byref(cfg), ctypes.byref(out))
    assert st == abi.WC_EINVAL
