"""The learned preconditioner: a small 4-level convolutional U-net.

No counterpart in the reference (its dispersive solve is Jacobi-preconditioned CG,
crates/wavecore/src/dispersion.rs:493-545). The network maps the SGN residual r = (rx, ry), with
the depth and bed, to a correction of the Jacobi step:

    z = r / diag + (s / H0) * mask * N(h / H0, b / H0, rx / s, ry / s),   s = rms(r)

so an untrained network (last layer zero) is exactly the Jacobi preconditioner, and scaling r
scales z. N is a U-net: on each of 4 levels two 3x3 convolutions with ReLU, 2x2 average pooling
down, nearest-neighbour upsampling and concatenation with the skip up, two 3x3 convolutions per
decoder level, and a 1x1 convolution to 2 channels. Weights are stored in FP32 for training and
used in BF16; accumulation is FP32. It is applied inside flexible CG (Polak-Ribiere beta), which
stays correct for a preconditioner that is not a fixed symmetric matrix, with the same stopping
rule as the plain solve.

This module holds the architecture's parameter layout, shared by the device kernels, the
training loop and the FP64 CPU reference used to check gradients.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

DEPTH_SCALE = 20.0  # H0, metres


@dataclass(frozen=True)
class UNetSpec:
    channels: tuple = (8, 16, 32, 32)  # feature maps per level, finest first
    in_ch: int = 4
    out_ch: int = 2

    @property
    def levels(self) -> int:
        return len(self.channels)

    def layers(self):
        """(name, c_out, c_in, kernel) in parameter order."""
        c = self.channels
        out = []
        cin = self.in_ch
        for l in range(self.levels):
            out.append((f"enc{l}a", c[l], cin, 3))
            out.append((f"enc{l}b", c[l], c[l], 3))
            cin = c[l]
        for l in range(self.levels - 2, -1, -1):
            out.append((f"dec{l}a", c[l], c[l + 1] + c[l], 3))
            out.append((f"dec{l}b", c[l], c[l], 3))
        out.append(("out", self.out_ch, c[0], 1))
        return out

    def offsets(self):
        """{name: (w_offset, b_offset, c_out, c_in, k)} into the flat parameter vector."""
        off = 0
        table = {}
        for name, co, ci, k in self.layers():
            w = off
            off += co * ci * k * k
            b = off
            off += co
            table[name] = (w, b, co, ci, k)
        return table

    def n_params(self) -> int:
        n = 0
        for _, co, ci, k in self.layers():
            n += co * ci * k * k + co
        return n

    def flops_per_cell(self) -> float:
        """Multiply-adds x2 per finest-level cell for one application."""
        f = 0.0
        for name, co, ci, k in self.layers():
            level = int(name[3]) if name != "out" else 0
            f += 2.0 * co * ci * k * k / (4.0 ** level)
        return f


def init_params(spec: UNetSpec, seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases, and a zero output layer (the network starts as Jacobi)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(spec.n_params(), dtype=np.float32)
    for name, (w, b, co, ci, k) in spec.offsets().items():
        if name == "out":
            continue
        std = np.sqrt(2.0 / (ci * k * k))
        p[w : w + co * ci * k * k] = rng.normal(0.0, std, co * ci * k * k).astype(np.float32)
    return p


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    rounding = 0x7FFF + ((a >> 16) & 1)
    r = ((a + rounding) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)
