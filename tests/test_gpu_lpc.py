"""The learned preconditioner on the device: network gradients against the FP64 oracle, the
flexible-CG solve against the Jacobi solve and the FP64 oracle, training, and what the trained
network gains over the method without it.

Tolerances (stated per test): FP32 device arithmetic against FP64 numpy, relative to the largest
magnitude of each compared block.
"""
import math

import numpy as np
import pytest

from oracle import unet_oracle as U
from oracle.oracle import OracleSolver
from wavesim_b200 import LearnedPreconditioner, Solver
from wavesim_b200 import workloads as W
from wavesim_b200.lpc import UNetSpec, bf16_round, init_params

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def random_params(spec, seed):
    """Initial weights plus non-zero output layer and biases, so every gradient is exercised."""
    rng = np.random.default_rng(seed)
    p = init_params(spec, seed).astype(np.float64)
    for name, (w, b, co, ci, k) in spec.offsets().items():
        if name == "out":
            p[w : w + co * ci * k * k] = rng.normal(0.0, 0.3, co * ci * k * k)
        if b >= 0:
            p[b : b + co] = rng.normal(0.0, 0.2, co)
    return p.astype(np.float32)


def batch(seed, n=2, h=16, w=24):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 2, h, w)).astype(np.float32)
    feat = np.stack([rng.uniform(0.0, 1.0, (n, h, w)), rng.uniform(-1.0, 0.2, (n, h, w))], axis=1).astype(np.float32)
    dy = rng.normal(size=(n, 2, h, w)).astype(np.float32)
    return x, feat, dy


def test_network_forward_and_gradients_match_the_fp64_oracle():
    spec = UNetSpec()
    net = LearnedPreconditioner(spec)
    net.set_rounding(False)
    p = random_params(spec, 3)
    net.set_params(p)
    x, feat, dy = batch(4)
    y, g, dx = net.forward_backward(x, feat, dy)
    yo, cache = U.forward(spec, p.astype(np.float64), x.astype(np.float64), feat.astype(np.float64))
    go, dxo = U.backward(spec, p.astype(np.float64), cache, dy.astype(np.float64))
    assert rel(y, yo) < 2e-5
    assert rel(dx, dxo) < 2e-5
    for name, (w, b, co, ci, k) in spec.offsets().items():  # per layer, FP32 sums of ~1e3 terms
        n = co * ci * k * k
        assert rel(g[w : w + n], go[w : w + n]) < 1e-4, name
        if b >= 0:
            assert rel(g[b : b + co], go[b : b + co]) < 1e-4, name + " bias"


def test_forward_uses_bf16_rounded_weights():
    spec = UNetSpec()
    net = LearnedPreconditioner(spec)
    p = random_params(spec, 5)
    net.set_params(p)  # rounding on by default
    x, feat, dy = batch(6, n=1, h=32, w=32)
    y, _, _ = net.forward_backward(x, feat, dy)
    yr, _ = U.forward(spec, bf16_round(p).astype(np.float64), x.astype(np.float64), feat.astype(np.float64))
    yf, _ = U.forward(spec, p.astype(np.float64), x.astype(np.float64), feat.astype(np.float64))
    assert rel(y, yr) < 2e-5
    assert rel(yr, yf) > 1e-4  # the rounding is visible: the test can tell the two apart
    assert np.array_equal(net.get_params(), p)  # the master weights stay FP32


@pytest.mark.parametrize("channels", [(8, 16, 32, 32), (32, 32, 32, 32)])
def test_tensor_core_inference_matches_the_oracle_to_bf16(channels):
    # The solver's network: BF16 activations on the tensor cores, FP32 accumulation. Against the
    # FP64 oracle with the same (BF16-rounded) weights: a few BF16 roundings per layer. Both the
    # default widths and 32 channels at every level (the kernels of a wider first level: 2 -> 32
    # and 32 -> 32 layers, a 64-channel decoder input at full resolution, a separate output layer).
    spec = UNetSpec(channels=channels)
    net = LearnedPreconditioner(spec)
    p = random_params(spec, 11)
    net.set_params(p)
    x, feat, _ = batch(12, n=2, h=32, w=48)
    yt = net.forward(x, feat, tensor=True)
    yf = net.forward(x, feat, tensor=False)
    yo, _ = U.forward(spec, bf16_round(p).astype(np.float64), x.astype(np.float64), feat.astype(np.float64))
    assert rel(yf, yo) < 2e-5
    assert rel(yt, yo) < 3e-2
    assert rel(yt, yo) > 1e-5  # the tensor path does round to BF16


def test_fused_first_level_launches_give_the_bits_of_the_per_layer_launches():
    # conv_enc0_kernel and conv_dec0_kernel keep the first level's 8-channel maps in shared memory
    # (rounded to BF16 there, as the per-layer launches round them in HBM); on a map whose sides
    # are not whole 32x16 tiles (40 x 56), so partial tiles and the zero-filled halos of their
    # boxes are exercised, the output must be the same bits either way.
    spec = UNetSpec()
    net = LearnedPreconditioner(spec)
    net.set_params(random_params(spec, 17))
    x, feat, _ = batch(18, n=2, h=40, w=56)
    fused = net.forward(x, feat, tensor=True, fused=True)
    per_layer = net.forward(x, feat, tensor=True, fused=False)
    assert np.abs(fused).max() > 0
    assert np.array_equal(fused, per_layer)


@pytest.mark.parametrize("h,w", [(40, 56), (136, 264)])
def test_coarse_layers_on_16x8_tiles_give_the_bits_of_the_usual_tiles(h, w):
    # The 32-channel layers of maps too small to give every SM two blocks of 16 x 16 pixels (the
    # coarse levels) run on 16 x 8 tiles; each pixel's accumulation is the same sequence of MMAs,
    # so the output must be the same bits as with the usual tiles. Sides that are not whole tiles
    # at any level exercise the partial tiles and their zero-filled halos.
    spec = UNetSpec()
    net = LearnedPreconditioner(spec)
    net.set_params(random_params(spec, 19))
    x, feat, _ = batch(20, n=1, h=h, w=w)
    small = net.forward(x, feat, tensor=True)
    usual = net.forward(x, feat, tensor=True, small_tiles=False)
    assert np.abs(small).max() > 0
    assert np.array_equal(small, usual)


def test_training_loss_and_gradient_match_the_fp64_oracle():
    # The whole training objective (the cycle on patches, the energy-norm loss) and its gradient
    # through the cycle and the network, against the FP64 oracle (FP32 weights on both sides).
    from wavesim_b200.lpc import OMEGA

    spec = UNetSpec()
    net = LearnedPreconditioner(spec)
    net.set_rounding(False)
    p = random_params(spec, 7)
    net.set_params(p)
    rng = np.random.default_rng(8)
    n, h, w = 3, 32, 40
    depth = rng.uniform(-0.3, 8.0, (n, h, w)).astype(np.float32)
    depth[2] = -1.0  # an all-dry patch contributes nothing
    heff = np.maximum(depth, 1e-8).astype(np.float32)
    c = np.where(depth < 0.05, 0.0, depth**3 / 3.0).astype(np.float32)
    bed = (-depth).astype(np.float32)
    e = (rng.normal(size=(n, 2, h, w)) * (heff >= 0.05)[:, None]).astype(np.float32)
    loss, g = net.loss_grad(c, heff, bed, e, 2.0, 2.0)
    lo, go = U.cycle_loss_grad(spec, p.astype(np.float64), c, heff, bed, e, 2.0, 2.0, OMEGA)
    assert abs(loss - lo) < 1e-5 * abs(lo)
    for name, (wo, b, co, ci, k) in spec.offsets().items():
        m = co * ci * k * k
        assert rel(g[wo : wo + m], go[wo : wo + m]) < 2e-4, name
        if b >= 0:
            assert rel(g[b : b + co], go[b : b + co]) < 2e-4, name + " bias"


def test_strided_training_loss_and_gradient_match_the_fp64_oracle():
    # The network on a grid twice coarser: block-mean input and features, output repeated.
    from dataclasses import replace

    from wavesim_b200.lpc import OMEGA

    spec = replace(UNetSpec(), stride=2)
    net = LearnedPreconditioner(spec)
    net.set_rounding(False)
    p = random_params(spec, 9)
    net.set_params(p)
    rng = np.random.default_rng(10)
    n, h, w = 2, 32, 48
    depth = rng.uniform(-0.3, 8.0, (n, h, w)).astype(np.float32)
    heff = np.maximum(depth, 1e-8).astype(np.float32)
    c = np.where(depth < 0.05, 0.0, depth**3 / 3.0).astype(np.float32)
    bed = (-depth).astype(np.float32)
    e = (rng.normal(size=(n, 2, h, w)) * (heff >= 0.05)[:, None]).astype(np.float32)
    loss, g = net.loss_grad(c, heff, bed, e, 2.0, 2.0)
    lo, go = U.cycle_loss_grad(spec, p.astype(np.float64), c, heff, bed, e, 2.0, 2.0, OMEGA)
    assert abs(loss - lo) < 1e-5 * abs(lo)
    for name, (wo, b, co, ci, k) in spec.offsets().items():
        m = co * ci * k * k
        assert rel(g[wo : wo + m], go[wo : wo + m]) < 2e-4, name


def small_run(seed=11, nx=192, ny=96, tol=1e-8):
    w = W.sgn_beach(nx, ny, 2.0, seed=seed, tolerance=tol, name=f"lpc_{nx}x{ny}")
    return w, W.wave_train_state(w)


def test_untrained_network_solve_matches_the_oracle():
    # An untrained network (zero output layer) leaves flexible CG preconditioned by two Jacobi
    # sweeps; the solution is the same system's, so the state matches the oracle as closely as
    # the Jacobi build does (same tolerances as the SGN parity case).
    w, s0 = small_run()
    net = LearnedPreconditioner(UNetSpec(), seed=1)
    gpu = w.solver(Solver)
    gpu.set_preconditioner(net)
    orc = w.solver(OracleSolver)
    sg, so = s0.clone(), s0.clone()
    g = w.grid
    for _ in range(60):
        dt = orc.stable_dt(so)
        orc.step(so, dt)
        gpu.step(sg, dt)
    hg, ho = g.inner(sg.h), g.inner(so.h)
    wet = (hg > 1e-3) & (ho > 1e-3)
    d = np.abs(hg - ho)[wet]
    assert d.max() < 3e-5
    assert abs(sg.volume(g) - so.volume(g)) < 1e-5 * so.volume(g)
    st = gpu.dispersion_stats()
    assert st.solves == 120 and st.unconverged == 0


def test_streaming_and_tiled_flexible_cg_passes_agree(monkeypatch):
    # The learned solve's pre, post and dir passes run with register-streaming sweeps by default;
    # the tiled passes (WAVECORE_B200_FCG=tiled) do the same per-cell arithmetic but partition the
    # dot products differently, so the two agree to the solve's tolerance and their iteration
    # counts within one per solve. Walls and periodic; sides that are not whole strips.
    net = LearnedPreconditioner(UNetSpec(), seed=1)
    for w in (W.sgn_beach(200, 90, 2.0, seed=5, name="periodic"),
              W.sgn_beach(150, 70, 2.0, seed=6, name="walls", periodic=False)):
        s0 = W.wave_train_state(w)
        monkeypatch.setenv("WAVECORE_B200_FCG", "tiled")
        tiled = w.solver(Solver)
        monkeypatch.delenv("WAVECORE_B200_FCG")
        stream = w.solver(Solver)
        outs = []
        for sol in (tiled, stream):
            sol.set_preconditioner(net)
            sol.upload(s0)
            sol.step_n(30)
            sol.synchronize()
            s = s0.clone()
            sol.download(s)
            outs.append((s, sol.dispersion_stats()))
        (a, sa), (b, sb) = outs
        g = w.grid
        assert abs(a.time - b.time) < 1e-9 * a.time
        assert np.max(np.abs(g.inner(a.h) - g.inner(b.h))) < 2e-6, w.name
        assert np.max(np.abs(g.inner(a.hu) - g.inner(b.hu))) < 2e-5, w.name
        assert sa.solves == sb.solves and sb.unconverged == 0
        assert abs(sa.iterations - sb.iterations) <= sa.solves, (sa, sb)


def harvest(net, seeds=(21, 22, 23), steps=40, every=10, nx=256, ny=128):
    for k, seed in enumerate(seeds):
        w = W.sgn_beach(nx, ny, 2.0, seed=seed, height=1.0 + k, period=10.0 + 3 * k, angle_deg=-15.0 + 15 * k)
        sol = w.solver(Solver)
        s = W.wave_train_state(w)
        sol.upload(s)
        for _ in range(steps // every):
            sol.step_n(every)
            sol.synchronize()
            net.harvest(sol)


def test_training_lowers_the_loss():
    net = LearnedPreconditioner(UNetSpec(), seed=2)
    harvest(net)
    assert net.n_systems == 12
    before = net.train(0)
    losses = net.train(300, batch=8, patch=64, lr=2e-3, seed=1)
    assert before.size == 0 and np.all(np.isfinite(losses))
    first, last = losses[:20].mean(), losses[-20:].mean()
    assert last < 0.5 * first, (first, last)


def test_trained_network_needs_fewer_iterations_than_jacobi():
    net = LearnedPreconditioner(UNetSpec(), seed=2)
    harvest(net)
    net.train(600, batch=8, patch=64, lr=2e-3, seed=2)
    w, s0 = small_run(seed=31, nx=256, ny=128)
    plain = w.solver(Solver)
    learned = w.solver(Solver)
    learned.set_preconditioner(net)
    sa, sb = s0.clone(), s0.clone()
    for _ in range(20):
        dt = plain.stable_dt(sa)
        plain.step(sa, dt)
        learned.step(sb, dt)
    a, b = plain.dispersion_stats(), learned.dispersion_stats()
    it_plain = a.iterations / a.solves
    it_learned = b.iterations / b.solves
    print(f"iterations per solve: Jacobi PCG {it_plain:.1f}, learned {it_learned:.1f}")
    assert b.unconverged == 0
    assert it_learned < 0.8 * it_plain
    g = w.grid
    assert np.max(np.abs(g.inner(sa.h) - g.inner(sb.h))) < 1e-5  # both solve to 1e-8


def test_learned_solve_counts_its_iteration_kernels():
    w, s0 = small_run(nx=128, ny=64)
    net = LearnedPreconditioner(UNetSpec(), seed=1)
    sol = w.solver(Solver)
    sol.set_preconditioner(net)
    sol.upload(s0)
    n0 = sol.launch_count()
    sol.step_n(3)
    sol.synchronize()
    st = sol.dispersion_stats()
    n1 = sol.launch_count()
    assert st.iterations > 0
    # every iteration is 19 kernels of the device library: four passes over the cells, three
    # scalar kernels and the network's twelve convolution launches (the first level's two
    # encoder layers in one, its two decoder layers and the 1x1 output layer in another)
    assert n1 - n0 >= 19 * st.iterations
    assert math.isfinite(sol.time_device())


def test_solvers_sharing_a_network_agree_bit_for_bit():
    # Regression: set-up copies and memsets used to run on the legacy stream and could land after
    # the first kernels on the solver's non-blocking stream (a solver then stepped on a partly
    # uploaded bed). Every solver built from the same inputs must now step identically.
    w, s0 = small_run(seed=41, nx=256, ny=128)
    net = LearnedPreconditioner(UNetSpec(), seed=3)
    outs = []
    keep = []
    for k in range(4):
        sol = w.solver(Solver)
        sol.set_preconditioner(net)
        s = s0.clone()
        for _ in range(5):
            sol.step(s, 0.05)
        outs.append(s.h.copy())
        if k % 2 == 0:
            keep.append(sol)
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
