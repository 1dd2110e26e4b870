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


def _map_inventory(spec):
    """Bytes per finest-level cell of one network application, counted map by map: every map
    that reaches HBM is written once and read once per reader; maps the device keeps on chip
    (the first level's A, DA and D when `fused_maps` says so) cost nothing."""
    c, L, b = spec.channels, spec.levels, 2.0
    on_a, on_da, on_d = spec.fused_maps()
    scale = [1.0 / 4.0**l for l in range(L)]
    total = b * spec.in_ch  # the input, read by enc_a[0]
    for l in range(L):
        m = b * c[l] * scale[l]
        total += m * (2 if l < L - 1 else 1)  # the gate: read by enc_b, and by dec_b below the top
        total += 0.0 if (l == 0 and on_a) else 2 * m  # A
        total += m * (3 if l < L - 1 else 2)  # E: written; read pooled by enc_a[l + 1] and by dec_a[l] / as up(E)
    for l in range(L - 1):
        m = b * c[l] * scale[l]
        total += 0.0 if (l == 0 and on_da) else 2 * m  # DA
        if l > 0:
            total += 2 * m  # D: written, read upsampled by dec_a[l - 1]
        elif not on_d:
            total += 2 * m  # D_0: written, read by the output layer
    return total + 4.0 * spec.out_ch  # the FP32 output


def test_the_bytes_model_counts_each_map_that_reaches_hbm_once():
    from dataclasses import replace

    spec = UNetSpec()  # the device's network: 8, 16, 32, 32 channels
    assert spec.fused_maps() == (True, True, True)
    assert spec.bytes_per_cell() == 229.0 == _map_inventory(spec)
    wide = replace(spec, channels=(8, 32, 32, 32))  # the decoder's first level runs as two launches
    assert wide.fused_maps() == (True, False, True)
    assert wide.bytes_per_cell() == _map_inventory(wide)
    plain = replace(spec, channels=(16, 16, 32, 32))  # nothing of the first level on chip
    assert plain.fused_maps() == (False, False, False)
    assert plain.bytes_per_cell() == 501.0 == _map_inventory(plain)
