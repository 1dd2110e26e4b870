"""FP64 CPU forward and backward of the learned preconditioner's network (TEST INFRASTRUCTURE ONLY).

The learned preconditioner has no counterpart in the reference; its oracle is this restatement
of the network of wavesim_b200/lpc.py in numpy FP64 (NCHW, zero padding), used to check the
device training kernels' outputs and gradients. Only tests/ import it.
"""
from __future__ import annotations

import numpy as np

from wavesim_b200.lpc import UNetSpec


def conv(x, w, b, k):
    """x: (N, Ci, H, W); w: (Co, Ci, k, k); zero padding (k // 2); b may be None."""
    n, ci, h, wd = x.shape
    co = w.shape[0]
    pad = k // 2
    xp = np.zeros((n, ci, h + 2 * pad, wd + 2 * pad))
    xp[:, :, pad : pad + h, pad : pad + wd] = x
    y = np.zeros((n, co, h, wd))
    for ty in range(k):
        for tx in range(k):
            y += np.einsum("nchw,oc->nohw", xp[:, :, ty : ty + h, tx : tx + wd], w[:, :, ty, tx])
    if b is not None:
        y += b[None, :, None, None]
    return y


def conv_bwd(x, w, dy, k):
    """Gradients of conv: (dx, dw, db)."""
    n, ci, h, wd = x.shape
    pad = k // 2
    xp = np.zeros((n, ci, h + 2 * pad, wd + 2 * pad))
    xp[:, :, pad : pad + h, pad : pad + wd] = x
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for ty in range(k):
        for tx in range(k):
            patch = xp[:, :, ty : ty + h, tx : tx + wd]
            dw[:, :, ty, tx] = np.einsum("nohw,nchw->oc", dy, patch)
            dxp[:, :, ty : ty + h, tx : tx + wd] += np.einsum("nohw,oc->nchw", dy, w[:, :, ty, tx])
    return dxp[:, :, pad : pad + h, pad : pad + wd], dw, dy.sum(axis=(0, 2, 3))


def pool(x):
    n, c, h, w = x.shape
    return x.reshape(n, c, h // 2, 2, w // 2, 2).mean(axis=(3, 5))


def pool_bwd(dy):
    return np.repeat(np.repeat(dy, 2, axis=2), 2, axis=3) / 4.0


def up(x):
    return np.repeat(np.repeat(x, 2, axis=2), 2, axis=3)


def up_bwd(dy):
    n, c, h, w = dy.shape
    return dy.reshape(n, c, h // 2, 2, w // 2, 2).sum(axis=(3, 5))


def unpack(spec: UNetSpec, params):
    p = np.asarray(params, dtype=np.float64)
    out = {}
    for name, (w, b, co, ci, k) in spec.offsets().items():
        out[name] = (p[w : w + co * ci * k * k].reshape(co, ci, k, k), p[b : b + co] if b >= 0 else None)
    return out


def gates(spec: UNetSpec, P, feat):
    """Gate maps per level and the cache for their backward."""
    out, cache = [], []
    f = feat
    for l in range(spec.levels):
        if l > 0:
            f = pool(f)
        wa, ba = P[f"gate{l}a"]
        pre = conv(f, wa, ba, 3)
        hid = np.maximum(pre, 0.0)
        wb, bb = P[f"gate{l}b"]
        z = conv(hid, wb, bb, 1)
        g = 2.0 / (1.0 + np.exp(-z))
        out.append(g)
        cache.append((f, hid, g))
    return out, cache


def forward(spec: UNetSpec, params, x, feat):
    """x: (N, 2, H, W) input; feat: (N, 2, H, W) = (h/H0, b/H0). Returns (y, cache)."""
    P = unpack(spec, params)
    G, gcache = gates(spec, P, feat)
    L = spec.levels
    cache = {"gcache": gcache, "G": G}
    enc = []
    cur = x
    for l in range(L):
        if l > 0:
            cur = pool(enc[-1])
        cache[f"in{l}"] = cur
        a = conv(cur, P[f"enc{l}a"][0], None, 3)
        cache[f"enc{l}a"] = a
        u = conv(a, P[f"enc{l}b"][0], None, 3)
        cache[f"enc{l}u"] = u
        e = u * G[l]
        enc.append(e)
    d = enc[-1]
    for l in range(L - 2, -1, -1):
        cat = np.concatenate([up(d), enc[l]], axis=1)
        cache[f"cat{l}"] = cat
        a = conv(cat, P[f"dec{l}a"][0], None, 3)
        cache[f"dec{l}a"] = a
        u = conv(a, P[f"dec{l}b"][0], None, 3)
        cache[f"dec{l}u"] = u
        d = u * G[l]
    cache["dec0"] = d
    y = conv(d, P["out"][0], None, 1)
    return y, cache


def backward(spec: UNetSpec, params, cache, dy):
    """Gradient of sum(dy * output) w.r.t. the flat parameters and the input x."""
    P = unpack(spec, params)
    L = spec.levels
    G = cache["G"]
    grads = {}
    dG = [np.zeros_like(g) for g in G]
    dd, dwo, _ = conv_bwd(cache["dec0"], P["out"][0], dy, 1)
    grads["out"] = (dwo, None)
    denc = [None] * L
    for l in range(0, L - 1):
        du = dd * G[l]
        dG[l] += dd * cache[f"dec{l}u"]
        da, dwb, _ = conv_bwd(cache[f"dec{l}a"], P[f"dec{l}b"][0], du, 3)
        grads[f"dec{l}b"] = (dwb, None)
        dcat, dwa, _ = conv_bwd(cache[f"cat{l}"], P[f"dec{l}a"][0], da, 3)
        grads[f"dec{l}a"] = (dwa, None)
        cu = spec.channels[l + 1]
        denc[l] = dcat[:, cu:]
        dd = up_bwd(dcat[:, :cu])
    de = dd  # gradient into the bottleneck output enc[L-1]
    dx = None
    for l in range(L - 1, -1, -1):
        if l < L - 1:
            de = denc[l] + de_from_below
        du = de * G[l]
        dG[l] += de * cache[f"enc{l}u"]
        da, dwb, _ = conv_bwd(cache[f"enc{l}a"], P[f"enc{l}b"][0], du, 3)
        grads[f"enc{l}b"] = (dwb, None)
        din, dwa, _ = conv_bwd(cache[f"in{l}"], P[f"enc{l}a"][0], da, 3)
        grads[f"enc{l}a"] = (dwa, None)
        if l > 0:
            de_from_below = pool_bwd(din)
        else:
            dx = din
    # gate networks
    for l in range(L):
        f, hid, g = cache["gcache"][l]
        dz = dG[l] * g * (1.0 - g / 2.0)
        dhid, dwb, dbb = conv_bwd(hid, P[f"gate{l}b"][0], dz, 1)
        grads[f"gate{l}b"] = (dwb, dbb)
        dpre = dhid * (hid > 0)
        _, dwa, dba = conv_bwd(f, P[f"gate{l}a"][0], dpre, 3)
        grads[f"gate{l}a"] = (dwa, dba)
    flat = np.zeros(spec.n_params())
    for name, (w, b, co, ci, k) in spec.offsets().items():
        gw, gb = grads[name]
        flat[w : w + co * ci * k * k] = gw.ravel()
        if b >= 0:
            flat[b : b + co] = gb
    return flat, dx


# ---- the training objective: the two-level cycle on patches ------------------------------------

H_DISP_MIN = 0.05


def _shift(a, dy, dx):
    """out[..., y, x] = a[..., y + dy, x + dx], zero outside."""
    out = np.zeros_like(a)
    h, w = a.shape[-2:]
    ys, yd = (slice(dy, h), slice(0, h - dy)) if dy >= 0 else (slice(0, h + dy), slice(-dy, h))
    xs, xd = (slice(dx, w), slice(0, w - dx)) if dx >= 0 else (slice(0, w + dx), slice(-dx, w))
    out[..., yd, xd] = a[..., ys, xs]
    return out


def patch_matvec(c, heff, mask, p, dx, dy):
    """A p of crates/wavecore/src/dispersion.rs:269-317 on patches (N, H, W), zero outside."""
    ix, iy = 0.5 / dx, 0.5 / dy
    px, py = p[:, 0], p[:, 1]
    f = c * ((_shift(px, 0, 1) - _shift(px, 0, -1)) * ix + (_shift(py, 1, 0) - _shift(py, -1, 0)) * iy)
    ax = mask * (heff * px - (_shift(f, 0, 1) - _shift(f, 0, -1)) * ix)
    ay = mask * (heff * py - (_shift(f, 1, 0) - _shift(f, -1, 0)) * iy)
    return np.stack([ax, ay], axis=1)


def patch_diag(c, heff, mask, dx, dy):
    """The Jacobi diagonal (dispersion.rs:441-457) on patches; 1 where the mask is off."""
    dxv = np.where(mask > 0, heff + (_shift(c, 0, 1) + _shift(c, 0, -1)) * 0.25 / (dx * dx), 1.0)
    dyv = np.where(mask > 0, heff + (_shift(c, 1, 0) + _shift(c, -1, 0)) * 0.25 / (dy * dy), 1.0)
    return np.stack([dxv, dyv], axis=1)


def cycle_loss_grad(spec: UNetSpec, params, c, heff, bed, e, dx, dy, omega):
    """Loss mean_n <d, A d>_n / <e, A e>_n of the cycle z = M A e (d = e - z) and its gradient
    with respect to the flat parameters. c, heff, bed: (N, H, W); e: (N, 2, H, W). A patch
    without a wet cell (<e, A e> = 0) contributes nothing. With spec.stride S > 1 the network
    sees S x S block means of its input and features and its output is repeated over the block."""
    c, heff, bed, e = (np.asarray(a, dtype=np.float64) for a in (c, heff, bed, e))
    mask = (heff >= H_DISP_MIN).astype(np.float64)
    feat = np.stack([heff / 20.0, bed / 20.0], axis=1)
    A = lambda v: patch_matvec(c, heff, mask, v, dx, dy)  # noqa: E731
    D = patch_diag(c, heff, mask, dx, dy)
    m2 = mask[:, None]
    r = A(e)
    z1 = omega * r / D
    x = (r - A(z1)) / D
    S = spec.stride
    pool_s = lambda a: a.reshape(a.shape[0], a.shape[1], a.shape[2] // S, S, a.shape[3] // S, S).mean(axis=(3, 5))  # noqa: E731
    up_s = lambda a: np.repeat(np.repeat(a, S, axis=2), S, axis=3)  # noqa: E731
    y, cache = forward(spec, params, pool_s(x), pool_s(feat))
    z2 = z1 + m2 * up_s(y)
    z = z2 + omega * (r - A(z2)) / D
    d = e - z
    ad = A(d)
    n = e.shape[0]
    num = np.einsum("nchw,nchw->n", d, ad)
    den = np.einsum("nchw,nchw->n", e, r)
    ok = den > 0.0
    safe = np.where(ok, den, 1.0)
    loss = float(np.sum(np.where(ok, num / safe, 0.0)) / n)
    gz = np.where(ok[:, None, None, None], -2.0 * ad / (n * safe[:, None, None, None]), 0.0)
    gz2 = gz - omega * A(gz / D)
    grads, _ = backward(spec, params, cache, pool_s(m2 * gz2) * (S * S))  # adjoint of up_s: block sums
    return loss, grads
