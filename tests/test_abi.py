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


def test_solver_creation_from_many_threads_reports_the_setup_error_in_each_thread():
    """Solvers may be created from several host threads at once (one handle per thread). On a
    host without a usable GPU the once-per-process kernel set-up fails: every thread gets that
    status, on its first call and on later ones, each with its own error text."""
    import threading

    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the set-up failure path of a host without a usable GPU")
    from wavesim_b200 import Bathymetry, Grid, Solver, WavecoreError, abi

    grid = Grid(64, 32, 2.0, 2.0)
    bed = Bathymetry.flat(grid, 5.0)
    results = [None] * 8
    start = threading.Barrier(len(results))

    def create(k):
        start.wait()
        out = []
        for _ in range(2):
            try:
                Solver(grid, bed).check()
                out.append(("created", ""))
            except WavecoreError as e:
                out.append((e.status, str(e)))
        results[k] = out

    threads = [threading.Thread(target=create, args=(k,)) for k in range(len(results))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=60)
    for out in results:
        assert out is not None and len(out) == 2
        for status, text in out:
            assert status == abi.WC_ECUDA
            assert "shared-memory limits" in text
