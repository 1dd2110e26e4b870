"""The FP64 oracle of the learned preconditioner's network and training objective, checked
against finite differences (CPU only)."""
import numpy as np

from oracle import unet_oracle as U
from wavesim_b200.lpc import OMEGA, UNetSpec, init_params

SPEC = UNetSpec(channels=(4, 4, 8, 8), gate_hidden=4)


def params(seed):
    rng = np.random.default_rng(seed)
    p = init_params(SPEC, seed).astype(np.float64)
    for name, (w, b, co, ci, k) in SPEC.offsets().items():
        if name == "out":
            p[w : w + co * ci * k * k] = rng.normal(0.0, 0.3, co * ci * k * k)
        if b >= 0:
            p[b : b + co] = rng.normal(0.0, 0.2, co)
    return p


def patches(seed, n=2, h=16, w=16):
    rng = np.random.default_rng(seed)
    depth = rng.uniform(-0.2, 6.0, (n, h, w))
    heff = np.maximum(depth, 1e-8)
    c = np.where(depth < 0.05, 0.0, depth**3 / 3.0)
    bed = -depth
    e = rng.normal(size=(n, 2, h, w)) * (heff >= 0.05)[:, None]
    return c, heff, bed, e


def test_network_gradient_matches_finite_differences():
    p = params(1)
    rng = np.random.default_rng(2)
    x = rng.normal(size=(1, 2, 16, 16))
    feat = rng.uniform(-1, 1, size=(1, 2, 16, 16))
    dy = rng.normal(size=(1, 2, 16, 16))
    y, cache = U.forward(SPEC, p, x, feat)
    g, dx = U.backward(SPEC, p, cache, dy)
    f = lambda q: float(np.sum(U.forward(SPEC, q, x, feat)[0] * dy))  # noqa: E731
    for idx in rng.choice(p.size, 12, replace=False):
        q1, q2 = p.copy(), p.copy()
        q1[idx] += 1e-6
        q2[idx] -= 1e-6
        assert abs((f(q1) - f(q2)) / 2e-6 - g[idx]) < 1e-5 * max(1.0, abs(g[idx]))


def test_cycle_loss_gradient_matches_finite_differences():
    p = params(3)
    c, heff, bed, e = patches(4)
    loss, g = U.cycle_loss_grad(SPEC, p, c, heff, bed, e, 2.0, 2.0, OMEGA)
    assert 0.0 < loss < 10.0
    rng = np.random.default_rng(5)
    for idx in rng.choice(p.size, 12, replace=False):
        q1, q2 = p.copy(), p.copy()
        q1[idx] += 1e-6
        q2[idx] -= 1e-6
        l1 = U.cycle_loss_grad(SPEC, q1, c, heff, bed, e, 2.0, 2.0, OMEGA)[0]
        l2 = U.cycle_loss_grad(SPEC, q2, c, heff, bed, e, 2.0, 2.0, OMEGA)[0]
        assert abs((l1 - l2) / 2e-6 - g[idx]) < 1e-6 + 1e-5 * abs(g[idx]), idx


def test_zero_network_cycle_reduces_the_error_energy():
    # The untrained network (zero output layer) leaves two damped Jacobi sweeps; with the
    # damping 0.5 the cycle contracts the error in the energy norm.
    p = init_params(SPEC, 0).astype(np.float64)
    c, heff, bed, e = patches(6, n=4, h=32, w=32)
    loss, _ = U.cycle_loss_grad(SPEC, p, c, heff, bed, e, 2.0, 2.0, OMEGA)
    assert 0.0 < loss < 1.0


def test_an_all_dry_patch_contributes_nothing():
    p = params(7)
    c, heff, bed, e = patches(8, n=2)
    l2, g2 = U.cycle_loss_grad(SPEC, p, c[:1], heff[:1], bed[:1], e[:1], 2.0, 2.0, OMEGA)
    c[1], heff[1], bed[1], e[1] = 0.0, 1e-8, 1.0, 0.0
    l, g = U.cycle_loss_grad(SPEC, p, c, heff, bed, e, 2.0, 2.0, OMEGA)
    assert np.isfinite(l) and np.all(np.isfinite(g))
    assert abs(l - l2 / 2) < 1e-12 and np.allclose(g, g2 / 2, rtol=1e-9, atol=1e-15)


def test_strided_cycle_loss_gradient_matches_finite_differences():
    from dataclasses import replace

    spec = replace(SPEC, stride=2)
    p = params(9)
    c, heff, bed, e = patches(10, n=2, h=32, w=32)
    loss, g = U.cycle_loss_grad(spec, p, c, heff, bed, e, 2.0, 2.0, OMEGA)
    rng = np.random.default_rng(11)
    for idx in rng.choice(p.size, 10, replace=False):
        q1, q2 = p.copy(), p.copy()
        q1[idx] += 1e-6
        q2[idx] -= 1e-6
        l1 = U.cycle_loss_grad(spec, q1, c, heff, bed, e, 2.0, 2.0, OMEGA)[0]
        l2 = U.cycle_loss_grad(spec, q2, c, heff, bed, e, 2.0, 2.0, OMEGA)[0]
        assert abs((l1 - l2) / 2e-6 - g[idx]) < 1e-6 + 1e-5 * abs(g[idx]), idx
