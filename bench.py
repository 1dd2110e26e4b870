"""Benchmark of wavecore's time step on B200: cell-steps/s with SGN on.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload config3|config2|config4|config5|swe4096|config1]
                    [--pc learned|jacobi] [--harvest beach|reef] [--lpc-channels 8,16,32,32]
    python bench.py --impl reference ...   # the reference algorithm on the host cores

A step is one SSP-RK2 step of the whole grid (both stages, both dispersive solves); one
cell-step is one interior cell advanced one step. The default workload is config 3: a 2048x1024
grid at 2 m, fifth order + SGN to a relative residual of 1e-8, periodic in y, a seeded rough 1:30
beach behind a 20 m shelf, H = 2 m, T = 14 s (see wavesim_b200/workloads.py). The state starts as
a linear wave train over the shelf, so every timed step carries the swell. With the learned
preconditioner (the default) the run first harvests systems from seeded runs of the workload's
own family and trains the network on the GPU, then times the learned arm (`value`) and plain
Jacobi PCG on the same workload (`plain_pcg`, `learned_vs_plain`).

`value` is device-timed (CUDA events on the solver's stream, one step at a time, L2 flushed
between steps by writing a 256 MiB buffer outside the timed events). `e2e` is the same metric
through the reference-facing call (`wc_step` on pinned host FP64 arrays, the copies in and out
inside the timed region). With N > 1 (torchrun) every rank advances its own replica (the runs
share nothing) and rank 0 reports the sum of cell-steps over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from wavesim_b200 import workloads as W  # noqa: E402
from wavesim_b200.model import State  # noqa: E402

METRIC = "cell-steps/s (SGN on), learned-PC vs plain PCG on 1 B200 at equal residual"
UNIT = "cell-steps/s"
L2_FLUSH_BYTES = 256 << 20

# Algorithmic bytes per interior cell (FP32 state with a compensated depth).
STAGE_BYTES_SGN = 16 + 4 + 8 + 8 + 4 + 4 + 8   # read q, b; write hn, pred, c, heff, b-vector
SOLVE_INIT_BYTES = (8 + 4 + 4 + 8 + 8 + 8 + 8) + (8 + 8 + 4 + 4 + 8)  # r = b - A w; then q0 = A (r / diag)
# read r, q, s, diag, p, c, heff and, every second iteration, w; write p, s, r, q and, every second
# iteration, w (the iterations' steps are added to w in pairs)
SOLVE_ITER_BYTES = (8 * 5 + 4 * 2 + 8 / 2) + (8 * 4 + 8 / 2)
SOLVE_FINISH_BYTES = (44 + 60) / 2 + 16 / 2     # stage 1 / stage 2 epilogue averaged; a pending step of w in half the solves
STAGE_BYTES_SWE = (36 + 52) / 2                 # stage 1 / stage 2 (RK average + damping)

# DRAM bytes per cell measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum of one capture
# each, on the network at 2048x1024, the streaming solve at 2048x1024 over 58 iterations and the
# two streaming second-order stages at 2048x2048; scaled to a launch by cells, and by iterations
# for the solve).
NETWORK_DRAM_BYTES_PER_CELL = 334.1e6 / (2048 * 1024)    # one application of the U-net
PCG_DRAM_BYTES_PER_CELL_ITER = (5.57e9 + 3.88e9) / (2048 * 1024 * 58)  # one iteration of the solve
STAGE_DRAM_BYTES_PER_CELL_SWE = ((93.0e6 + 32.1e6) + (161.3e6 + 35.6e6)) / 2 / (2048 * 2048)  # a stage


def workload(name: str, eddy: bool = False):
    """The named workload; with `eddy`, its dispersive model follows breaking fronts with Kennedy's
    eddy viscosity (Breaking::viscosity, crates/wavecore/src/eddy.rs)."""
    w = {"config1": W.config1, "config2": W.config2, "config3": W.config3, "config5": W.config5,
         "swe4096": W.swe_large}[name]()
    if eddy:
        if w.dispersion is None:
            raise SystemExit("--eddy needs a dispersive workload: followed fronts exist only with dispersion")
        from dataclasses import replace

        from wavesim_b200 import EddyViscosity
        w.dispersion = replace(w.dispersion, breaking=replace(w.dispersion.breaking, viscosity=EddyViscosity()))
        w.meta["followed_fronts"] = "Kennedy eddy viscosity (EddyViscosity::default)"
    return w

# Algorithmic bytes per cell of the eddy kernel: follow reads the state (16), bed (4) and memory
# (8) and writes the new memory (8), nu (4) and the momentum bank (8); each viscous sub-step reads
# the depth (8), nu (4) and a bank (8) and writes a bank or the momentum (8); the finish moves
# the memory (16).
EDDY_BYTES = 48 + 16
REF_BUDGET_S = 120.0  # the reference arm's timed CPU sample
EDDY_SUBSTEP_BYTES = 28


def time_ensemble(ens, n_members, steps, warmup, flush, clocks_gpu, dist=None):
    """Warm-up steps, then `steps` timed steps of every member (host wall clock around each
    synchronised step; L2 flushed between steps): (seconds, PCG iterations per solve, launches, clocks)."""
    import torch

    ens.step_n(warmup)
    ens.synchronize()
    l0 = ens.launch_count()
    it0 = [ens.member_stats(m)[0] for m in range(n_members)]
    torch.cuda.synchronize()
    times = []
    if dist:
        dist.barrier()
    with ClockSampler(clocks_gpu) as clocks:
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ens.step_n(1)
            ens.synchronize()
            times.append(time.perf_counter() - t0)
    it1 = [ens.member_stats(m)[0] for m in range(n_members)]
    solves = sum(b.solves - a.solves for a, b in zip(it0, it1))
    iters = sum(b.iterations - a.iterations for a, b in zip(it0, it1)) / max(1, solves)
    return sum(times), iters, int(ens.launch_count() - l0), clocks.summary()


def members_alone(ws, net, steps: int, flush):
    """The same members run one at a time by standalone solvers (the network attached to the
    dispersive ones when given): the sum of their device-timed steps, per ensemble step."""
    import torch

    from wavesim_b200 import Solver

    total_ms = 0.0
    st = torch.cuda.Stream()  # a real stream handle: the solver and the events share it
    for w in ws:
        sol = w.solver(Solver)
        sol.set_stream(st.cuda_stream)
        if net is not None and w.dispersion is not None:
            sol.set_preconditioner(net)
        sol.upload(W.wave_train_state(w))
        sol.step_n(2)
        sol.synchronize()
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            sol.step_n(1)
            b.record(st)
            b.synchronize()
            total_ms += a.elapsed_time(b)
        del sol
    return total_ms / steps


def run_ensemble(args, world, rank, local):
    """The 64-member ensemble (config 4): every timed step advances every member one step. With the
    learned preconditioner (the default --pc), the network is trained first and the learned
    ensemble is the reported value, beside the same ensemble by plain PCG in one persistent launch
    per step and the learned members run one at a time."""
    import torch

    from wavesim_b200 import Ensemble, Solver

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    ws = W.config4(seed=4 + 1000 * rank)
    cells = sum(w.interior_cells() for w in ws)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    learned = args.pc == "learned"
    net, train_rec = None, None
    if learned:
        from wavesim_b200.lpc import UNetSpec
        from wavesim_b200.train_lpc import trained_network

        chans = tuple(int(c) for c in args.lpc_channels.split(","))
        net, train_rec = trained_network(dx=2.5, steps=args.train_steps, spec=UNetSpec(channels=chans))

    def arm(with_net):
        ens = Ensemble([w.solver(Solver) for w in ws])
        if with_net is not None:
            ens.set_preconditioner(with_net)
        for m, w in enumerate(ws):
            ens.upload(m, W.wave_train_state(w))
        choice, tune_ms = ens.autotune(2)
        sec, iters, launches, clocks = time_ensemble(ens, len(ws), args.steps, args.warmup, flush, local, dist)
        total = rank_max(sec, dist)  # the slowest rank's time
        return {"value": rank_sum(float(cells), dist) * args.steps / total, "ms_per_step": 1e3 * total / args.steps,
                "iterations_per_solve": iters, "launches": launches, "clocks": clocks,
                "variant": Ensemble.VARIANTS[choice],
                "autotune_ms_per_step": tune_ms}

    main = arm(net)
    plain = arm(None) if learned else None
    alone_ms = members_alone(ws, net, max(2, min(args.steps, 5)), flush) if rank == 0 else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": main["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "ensemble_64_uneven_beaches", "members": len(ws), "cells": cells,
                       "scheme": "fifth order + SGN",
                       "preconditioner": "learned (flexible CG)" if learned else "jacobi (plain PCG)", "tolerance": 1e-8,
                       "pcg_iterations_per_solve": main["iterations_per_solve"], "variant": main["variant"],
                       "autotune_ms_per_step": main["autotune_ms_per_step"],
                       "timing": "host wall clock around each synchronised ensemble step",
                       "l2": "flushed between timed steps (256 MiB write outside the timed region)"},
            "gpu_launches": main["launches"],
            "clocks": main["clocks"],
            "members_alone": {"ms_per_step": alone_ms, "value": cells / (alone_ms / 1e3),
                              "ensemble_speedup": alone_ms / main["ms_per_step"],
                              "how": "each member by a standalone solver, device-timed steps summed"},
        }
        if plain is not None:
            line["plain_pcg"] = {"value": plain["value"], "ms_per_step": plain["ms_per_step"],
                                 "iterations_per_solve": plain["iterations_per_solve"], "variant": plain["variant"],
                                 "autotune_ms_per_step": plain["autotune_ms_per_step"],
                                 "gpu_launches": plain["launches"], "clocks": plain["clocks"]}
            line["learned_vs_plain"] = main["value"] / plain["value"]
            line["training"] = train_rec
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def peak_tensor():
    """Dense BF16 tensor throughput (TFLOP/s), burst figure: the network is timed per application."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured (cuBLAS bf16, burst)"
    except Exception:
        return 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for name, v in zip(names, p[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def rank_max(value: float, dist=None, device: str = "cuda") -> float:
    """The largest of one value per rank (timings: the slowest rank's), or the value itself on
    one rank. `device` is where the collective's tensor lives (cuda for NCCL, cpu for gloo)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_sum(value: float, dist=None, device: str = "cuda") -> float:
    """The sum of one value per rank (work done by all ranks), or the value itself on one rank."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(w, steps: int):
    """The FP64 oracle (the reference's algorithm restated) on all host cores, on a bounded sample
    of the same workload: `steps` steps from the same start."""
    from oracle.oracle import OracleSolver, set_threads

    threads = set_threads(0)
    sol = w.solver(OracleSolver)
    s = W.wave_train_state(w)
    sol.step(s, sol.stable_dt(s))  # untimed warm-up of caches and thread pool
    t0 = time.perf_counter()
    for _ in range(steps):
        sol.step(s, sol.stable_dt(s))
    el = time.perf_counter() - t0
    st = sol.dispersion_stats()
    return {
        "value": w.interior_cells() * steps / el,
        "unit": UNIT,
        "cores": threads,
        "kind": "port",
        "sample": f"{steps} steps of {w.name} from the wave-train start on {threads} threads "
                  f"({el:.1f} s; {st.iterations / max(1, st.solves):.1f} PCG iterations/solve)" if st else
                  f"{steps} steps of {w.name} on {threads} threads ({el:.1f} s)",
    }


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle.oracle import OracleSolver, set_threads

    w = workload(args.workload, args.eddy)
    threads = set_threads(0)
    sol = w.solver(OracleSolver)
    s = W.wave_train_state(w)
    # A bounded sample: at most 3 warm-up steps and as many of the K timed steps as fit in
    # REF_BUDGET_S seconds (the CPU step of the large workloads takes about a second).
    for _ in range(min(args.warmup, 3)):
        sol.step(s, sol.stable_dt(s))
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sol.step(s, sol.stable_dt(s))
        times.append(time.perf_counter() - t0)
        if sum(times) > REF_BUDGET_S:
            break
    el = sum(times)
    timed = len(times)
    value = w.interior_cells() * timed / el
    st = sol.dispersion_stats()
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * el / timed,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": w.name, "nx": w.grid.nx, "ny": w.grid.ny, "dx_m": w.grid.dx,
                   "tolerance": w.dispersion.tolerance if w.dispersion else None, **{k: v for k, v in w.meta.items() if k != "bed"}},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{timed} of the {args.steps} timed steps of {w.name} (bounded at {REF_BUDGET_S:.0f} s) "
                                   f"after {min(args.warmup, 3)} warm-up steps, {threads} threads"
                                   + (f"; {st.iterations / max(1, st.solves):.1f} PCG iterations/solve" if st else "")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def measure_arm(w, args, world, stream, flush, net=None):
    """One arm (Jacobi PCG, or the learned preconditioner when `net` is given): device-timed
    steps, the per-kernel profiled pass, the end-to-end pass through `wc_step`."""
    import torch

    from wavesim_b200 import Solver

    dist = torch.distributed if world > 1 else None
    sol = w.solver(Solver)
    sol.set_stream(stream.cuda_stream)
    if net is not None:
        sol.set_preconditioner(net)
    if args.direct:
        sol.profile(True)
    s0 = W.wave_train_state(w)
    sol.upload(s0)
    sol.step_n(args.warmup)  # warm-up: adaptive steps on the device
    sol.synchronize()
    st0 = sol.dispersion_stats()
    l0 = sol.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            sol.step_n(1)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    sol.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    launches = sol.launch_count() - l0
    st1 = sol.dispersion_stats()
    # A second pass of the same steps with every launch bracketed by events on the solver's
    # stream (direct launches instead of the step graph): per-kernel device times.
    sol.profile(True)
    for k in range(args.steps):
        flush.zero_()
        sol.step_n(1)
    sol.synchronize()
    prof = sol.profile_read()
    sol.profile(False)
    st2 = sol.dispersion_stats()
    total_ms_max = rank_max(sum(step_ms), dist)
    if dist:
        dist.barrier()
    cells = w.interior_cells()

    # end to end through the reference-facing call, pinned host FP64 arrays
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    hs = State(pin(s0.h), pin(s0.hu), pin(s0.hv), pin(s0.breaking), s0.time)
    e2e_sol = w.solver(Solver)
    e2e_sol.set_stream(stream.cuda_stream)
    if net is not None:
        e2e_sol.set_preconditioner(net)
    # The reference driver's loop (crates/wavesim/src/lib.rs:1385-1426): the step size from the
    # state's stable_dt, then the step, both through the C ABI on the host arrays.
    for _ in range(2):
        e2e_sol.step(hs, e2e_sol.stable_dt(hs))
    n_e2e = max(3, min(args.steps, 50))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        e2e_sol.step(hs, e2e_sol.stable_dt(hs))
    e2e_s = time.perf_counter() - t0
    e2e_max = rank_max(e2e_s, dist)
    per_solve = lambda a, b: (b.iterations - a.iterations) / max(1, b.solves - a.solves) if b else 0.0  # noqa: E731
    return {
        "value": cells * args.steps * world / (total_ms_max / 1e3),
        "ms_per_step": total_ms_max / args.steps,
        "iterations_per_solve": per_solve(st0, st1),
        "iterations_per_solve_profiled": per_solve(st1, st2),
        "unconverged": (st2.unconverged - st0.unconverged) if st2 else 0,
        "prof": prof,
        "launches": int(launches),
        "clocks": clocks.summary(),
        "e2e": {"value": cells * n_e2e * world / e2e_max, "unit": UNIT,
                "h2d_bytes_per_step": 6 * w.grid.cells() * 8 + 24, "d2h_bytes_per_step": 3 * w.grid.cells() * 8 + 24,
                "steps": n_e2e,
                "path": "per step wc_stable_dt then wc_step on pinned host FP64 arrays (each uploads the state; "
                        "the step downloads it), as the reference's driver loop calls stable_dt and step"},
    }


def true_residuals(w, arms):
    """The true FP64 relative residual ||b - A w|| / ||b|| of each arm's last dispersive solve (the
    device stops on its recursively updated FP32 residual at the tolerance), the oracle's FP64
    Jacobi PCG on the same system from zero, and that FP64 solution rounded to FP32 (the floor any
    FP32-stored solution has)."""
    from oracle.oracle import pcg_solve, true_relative_residual

    out = {"tolerance": w.dispersion.tolerance}
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)  # noqa: E731
    for k, sol in arms.items():
        sysd = sol.dispersion_system()
        wx, wy, it, conv = pcg_solve(w.grid, w.periodic_y, sysd, w.dispersion.tolerance, 2000)
        out[k] = {"device": true_relative_residual(w.grid, w.periodic_y, sysd),
                  "oracle_fp64_same_system": true_relative_residual(w.grid, w.periodic_y, {**sysd, "wx": wx, "wy": wy}),
                  "oracle_iterations_from_zero": it,
                  "fp32_solution_floor": true_relative_residual(w.grid, w.periodic_y, {**sysd, "wx": f32(wx), "wy": f32(wy)})}
    return out


def eta_errors(w, net, steps: int):
    """Max |eta - eta_oracle| over wet cells after `steps` steps from the wave-train start (the
    oracle's dt sequence), for Jacobi PCG and the learned preconditioner."""
    from oracle.oracle import OracleSolver, set_threads

    from wavesim_b200 import Solver

    set_threads(0)
    orc = w.solver(OracleSolver)
    arms = {"plain_pcg": w.solver(Solver), "learned": w.solver(Solver)}
    arms["learned"].set_preconditioner(net)
    s0 = W.wave_train_state(w)
    so = s0.clone()
    ss = {k: s0.clone() for k in arms}
    for _ in range(steps):
        dt = orc.stable_dt(so)
        orc.step(so, dt)
        for k, sol in arms.items():
            sol.step(ss[k], dt)
    g = w.grid
    ho = g.inner(so.h)
    out = {"true_rel_residual": true_residuals(w, arms)}
    for k, s in ss.items():
        hg = g.inner(s.h)
        wet = (hg > 1e-3) & (ho > 1e-3)
        d = np.abs(hg - ho)[wet]
        st = arms[k].dispersion_stats()
        out[k] = {"max": float(d.max()), "rms": float(np.sqrt(np.mean(d * d))), "cells_over_1mm": int((d > 1e-3).sum()),
                  "nan_cells": int(np.isnan(hg).sum()), "iterations_per_solve": st.iterations / max(1, st.solves),
                  "unconverged": st.unconverged}
    out["steps"] = steps
    return out


def run_b200(args, world, rank, local):
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    w = workload(args.workload, args.eddy)
    stream = torch.cuda.Stream()  # a real stream handle: the solvers and the events share it
    torch.cuda.set_stream(stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    learned = args.pc == "learned" and w.dispersion is not None

    net, train_rec = None, None
    if learned:
        from wavesim_b200.train_lpc import trained_network

        torch.cuda.synchronize()
        from wavesim_b200.lpc import UNetSpec

        spec = UNetSpec(channels=tuple(int(c) for c in args.lpc_channels.split(",")), stride=args.lpc_stride)
        if args.train_steps > 0:
            family = args.harvest or ("reef" if args.workload == "config5" else "beach")
            net, train_rec = trained_network(dx=w.grid.dx, steps=args.train_steps, seed=0, spec=spec, family=family)
        else:  # an untrained network (profiling runs: same kernels, no harvest or training launches)
            from wavesim_b200 import LearnedPreconditioner

            net, train_rec = LearnedPreconditioner(spec, seed=0), {"untrained": True}
        torch.cuda.synchronize()
    arm = measure_arm(w, args, world, stream, flush, net)
    plain = measure_arm(w, args, world, stream, flush, None) if learned else None

    line = None
    if rank == 0:
        cells = w.interior_cells()
        prof = arm["prof"]
        solve_n, solve_ms = prof["solve"]
        stage_n, stage_ms = prof["stage"]
        net_n, net_ms = prof.get("network", (0, 0.0))
        peak, peak_kind = measured_peaks()
        iters_prof = arm["iterations_per_solve_profiled"]
        if learned and net_ms >= max(solve_ms, stage_ms):
            # One network application: 18 kFLOP and 229 B per cell of its finest level, 79 FLOP/B,
            # below the B200's ridge point (about 220 FLOP/B), so its roof is HBM bandwidth.
            spec = net.spec
            ncell = w.grid.nx * w.grid.ny / spec.stride**2
            avg_ms = net_ms / net_n
            tflops = spec.flops_per_cell() * ncell / (avg_ms / 1e3) / 1e12
            gbs = spec.bytes_per_cell() * ncell / (avg_ms / 1e3) / 1e9
            bf16 = peak_tensor()
            roof = {"bound": "hbm", "kernel": "network convolution chain (one application: conv_enc0 / conv_p8 / "
                                              "conv_h / conv_up / conv_dec0 kernels, channels-innermost BF16 mma.sync "
                                              "implicit GEMM, FP32 accumulation)",
                    "achieved": gbs, "unit": "GB/s", "peak": peak, "frac": gbs / peak, "peak_source": peak_kind,
                    "algorithmic_bytes_per_cell": spec.bytes_per_cell(), "flops_per_cell": spec.flops_per_cell(),
                    "avg_ms": avg_ms, "tensor_tflops": tflops, "tensor_frac": tflops / bf16[0],
                    "tensor_peak_source": bf16[1],
                    "traffic": NETWORK_DRAM_BYTES_PER_CELL * ncell,
                    "traffic_source": "ncu DRAM bytes of one application at 2048x1024, scaled by cells"}
        else:
            if solve_n and solve_ms >= stage_ms:
                per_cell = SOLVE_INIT_BYTES + SOLVE_ITER_BYTES * iters_prof + SOLVE_FINISH_BYTES
                dom = {"kernel": "pcg_stream_kernel (persistent dispersive solve, streaming sweeps)", "launches": solve_n,
                       "avg_ms": solve_ms / solve_n, "bytes_per_cell": per_cell}
            else:
                per_cell = STAGE_BYTES_SGN if w.dispersion else STAGE_BYTES_SWE
                dom = {"kernel": ("swe_stream_kernel (fused RK stage, streaming rows)" if not w.dispersion else "stage_kernel (fused RK stage)"), "launches": stage_n,
                       "avg_ms": stage_ms / max(1, stage_n), "bytes_per_cell": per_cell}
            achieved = per_cell * cells / (dom["avg_ms"] / 1e3) / 1e9
            traffic = None
            if dom["kernel"].startswith("pcg_stream_kernel"):
                traffic = PCG_DRAM_BYTES_PER_CELL_ITER * iters_prof * cells
            elif not w.dispersion and w.order.value == 1:
                traffic = STAGE_DRAM_BYTES_PER_CELL_SWE * cells
            roof = {"bound": "hbm", "kernel": dom["kernel"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind, "algorithmic_bytes_per_cell": dom["bytes_per_cell"],
                    "avg_ms": dom["avg_ms"], "traffic": traffic,
                    "traffic_source": ("ncu DRAM bytes per cell and iteration of one solve at 2048x1024, scaled by "
                                       "cells and iterations" if dom["kernel"].startswith("pcg_stream_kernel") else
                                       "ncu DRAM bytes of the two second-order stages at 2048x2048, averaged and scaled by cells")
                    if traffic else None}
        line = {
            "metric": METRIC,
            "value": arm["value"],
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": arm["ms_per_step"],
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": w.name, "nx": w.grid.nx, "ny": w.grid.ny, "dx_m": w.grid.dx,
                "scheme": "fifth order + SGN" if w.dispersion else "second order SWE",
                "preconditioner": ("learned (gated linear U-net in a two-level cycle, flexible CG)" if learned
                                   else "jacobi (plain PCG)") if w.dispersion else None,
                "tolerance": w.dispersion.tolerance if w.dispersion else None,
                "pcg_iterations_per_solve": arm["iterations_per_solve"],
                "unconverged_solves": arm["unconverged"],
                "l2": "flushed between timed steps (256 MiB write outside the timed events)",
                "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                **{k: v for k, v in w.meta.items() if k != "bed"},
            },
            "roofline": roof,
            "kernel_ms_per_step": {"stage": stage_ms / args.steps, "solve": solve_ms / args.steps,
                                   "network": net_ms / args.steps, "other": prof["other"][1] / args.steps,
                                   "eddy": prof.get("eddy", (0, 0.0))[1] / args.steps,
                                   "source": "profiled pass of the same number of steps after the timed pass "
                                             "(direct launches; the learned solve syncs with the host every 4 iterations there)"},
            "e2e": arm["e2e"],
            "gpu_launches": arm["launches"],
            "clocks": arm["clocks"],
        }
        if args.eddy and prof.get("eddy", (0, 0.0))[0]:
            en, ems = prof["eddy"]
            total = sum(v[1] for v in prof.values())
            per = EDDY_BYTES + EDDY_SUBSTEP_BYTES  # at least one viscous sub-step when a front breaks
            line["eddy_kernel"] = {"kernel": "eddy_kernel (fronts, viscosity sub-steps, finish; cooperative)",
                                   "launches": en, "avg_ms": ems / en, "share_of_kernel_time": ems / total,
                                   "bytes_per_cell_one_substep": per,
                                   "achieved_gbs_one_substep": per * cells / (ems / en / 1e3) / 1e9, "peak": peak}
        if learned:
            line["plain_pcg"] = {
                "value": plain["value"], "ms_per_step": plain["ms_per_step"],
                "iterations_per_solve": plain["iterations_per_solve"], "unconverged_solves": plain["unconverged"],
                "e2e": plain["e2e"]["value"], "gpu_launches": plain["launches"], "clocks": plain["clocks"],
                "kernel_ms_per_step": {k: v[1] / args.steps for k, v in plain["prof"].items()},
            }
            line["learned_vs_plain"] = arm["value"] / plain["value"]
            line["training"] = train_rec
            if args.eta_steps > 0:
                line["eta_max_abs_err_vs_fp64_oracle_m"] = eta_errors(w, net, args.eta_steps)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(w, args.cpu_steps)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="config3", choices=["config1", "config2", "config3", "config4", "config5", "swe4096"])
    ap.add_argument("--pc", default="learned", choices=["learned", "jacobi"],
                    help="learned: time the learned preconditioner and plain PCG side by side (SGN workloads)")
    ap.add_argument("--train-steps", type=int, default=20000)
    ap.add_argument("--lpc-stride", type=int, default=1, choices=[1, 2, 4])
    ap.add_argument("--lpc-channels", default="8,16,32,32")
    ap.add_argument("--harvest", default=None, choices=["beach", "reef"],
                    help="workload family the training systems are harvested from (default: the workload's own)")
    ap.add_argument("--eta-steps", type=int, default=10)
    ap.add_argument("--cpu-steps", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--eddy", action="store_true",
                    help="follow breaking fronts with Kennedy's eddy viscosity (dispersive workloads)")
    ap.add_argument("--direct", action="store_true",
                    help="launch every kernel directly, no step graph (for profilers: a graph with a "
                         "conditional node hides its kernels from ncu)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "config4":
        run_ensemble(args, world, rank, local)
        return
    run_b200(args, world, rank, local)


if __name__ == "__main__":
    main()
