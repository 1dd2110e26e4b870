"""FP64 CPU forward and backward of the learned preconditioner's U-net (TEST INFRASTRUCTURE ONLY).

The learned preconditioner has no counterpart in the reference; its oracle is this restatement
of the network in numpy FP64 (NCHW, zero padding, the architecture of wavesim_b200/lpc.py), used
to check the device training kernels' forward values and gradients. Only tests/ import it.
"""
from __future__ import annotations

import numpy as np

from wavesim_b200.lpc import UNetSpec


def conv(x, w, b, k):
    """x: (N, Ci, H, W); w: (Co, Ci, k, k); zero padding (k // 2)."""
    n, ci, h, wd = x.shape
    co = w.shape[0]
    pad = k // 2
    xp = np.zeros((n, ci, h + 2 * pad, wd + 2 * pad))
    xp[:, :, pad : pad + h, pad : pad + wd] = x
    y = np.zeros((n, co, h, wd))
    for ty in range(k):
        for tx in range(k):
            patch = xp[:, :, ty : ty + h, tx : tx + wd]
            y += np.einsum("nchw,oc->nohw", patch, w[:, :, ty, tx])
    return y + b[None, :, None, None]


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
    db = dy.sum(axis=(0, 2, 3))
    return dxp[:, :, pad : pad + h, pad : pad + wd], dw, db


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
        out[name] = (p[w : w + co * ci * k * k].reshape(co, ci, k, k), p[b : b + co])
    return out


def forward(spec: UNetSpec, params, x):
    """Returns (output (N, 2, H, W), cache for backward). H and W divisible by 2**(levels-1)."""
    P = unpack(spec, params)
    cache = {}
    L = spec.levels
    enc = []
    cur = x
    for l in range(L):
        if l > 0:
            cur = pool(enc[-1])
        cache[f"in{l}"] = cur
        wa, ba = P[f"enc{l}a"]
        a = np.maximum(conv(cur, wa, ba, 3), 0.0)
        cache[f"enc{l}a"] = a
        wb, bb = P[f"enc{l}b"]
        e = np.maximum(conv(a, wb, bb, 3), 0.0)
        cache[f"enc{l}b"] = e
        enc.append(e)
    d = enc[-1]
    for l in range(L - 2, -1, -1):
        u = up(d)
        cat = np.concatenate([u, enc[l]], axis=1)
        cache[f"cat{l}"] = cat
        wa, ba = P[f"dec{l}a"]
        a = np.maximum(conv(cat, wa, ba, 3), 0.0)
        cache[f"dec{l}a"] = a
        wb, bb = P[f"dec{l}b"]
        d = np.maximum(conv(a, wb, bb, 3), 0.0)
        cache[f"dec{l}b"] = d
    wo, bo = P["out"]
    y = conv(d, wo, bo, 1)
    return y, cache


def backward(spec: UNetSpec, params, cache, dy):
    """Gradient of sum(dy * output) with respect to the flat parameter vector and the input."""
    P = unpack(spec, params)
    L = spec.levels
    grads = {}
    wo, bo = P["out"]
    dd, dwo, dbo = conv_bwd(cache["dec0b"], wo, dy, 1)
    grads["out"] = (dwo, dbo)
    denc = [np.zeros_like(cache[f"enc{l}b"]) for l in range(L)]
    # the decoder, from the finest level back towards the bottleneck (reverse of the forward)
    for l in range(0, L - 1):
        wb, bb = P[f"dec{l}b"]
        dd = dd * (cache[f"dec{l}b"] > 0)
        da, dwb, dbb = conv_bwd(cache[f"dec{l}a"], wb, dd, 3)
        grads[f"dec{l}b"] = (dwb, dbb)
        wa, ba = P[f"dec{l}a"]
        da = da * (cache[f"dec{l}a"] > 0)
        dcat, dwa, dba = conv_bwd(cache[f"cat{l}"], wa, da, 3)
        grads[f"dec{l}a"] = (dwa, dba)
        cu = spec.channels[l + 1]
        denc[l] += dcat[:, cu:]
        dd = up_bwd(dcat[:, :cu])  # gradient into the next coarser decoder output
    # the bottleneck output is enc[L-1]
    denc[L - 1] += dd
    dx = None
    for l in range(L - 1, -1, -1):
        de = denc[l] * (cache[f"enc{l}b"] > 0)
        wb, bb = P[f"enc{l}b"]
        da, dwb, dbb = conv_bwd(cache[f"enc{l}a"], wb, de, 3)
        grads[f"enc{l}b"] = (dwb, dbb)
        wa, ba = P[f"enc{l}a"]
        da = da * (cache[f"enc{l}a"] > 0)
        din, dwa, dba = conv_bwd(cache[f"in{l}"], wa, da, 3)
        grads[f"enc{l}a"] = (dwa, dba)
        if l > 0:
            denc[l - 1] += pool_bwd(din)
        else:
            dx = din
    flat = np.zeros(spec.n_params())
    for name, (w, b, co, ci, k) in spec.offsets().items():
        gw, gb = grads[name]
        flat[w : w + co * ci * k * k] = gw.ravel()
        flat[b : b + co] = gb
    return flat, dx
