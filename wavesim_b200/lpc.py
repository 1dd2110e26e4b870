"""The learned preconditioner of the SGN solve: a depth-gated linear U-net in a two-level cycle.

No counterpart in the reference (its dispersive solve is Jacobi-preconditioned CG,
crates/wavecore/src/dispersion.rs:493-545). Given a residual r of the system
h w - grad(c div w) = r, the preconditioner returns

    z1 = omega r / diag                       damped Jacobi sweep
    z2 = z1 + mask * N(diag^-1 (r - A z1))    the network's correction
    z  = z2 + omega (r - A z2) / diag         damped Jacobi sweep

N is a 4-level U-net of 3x3 convolutions without biases or activations, so z depends linearly
on r (Krylov methods need that: a network that is nonlinear in r stalled flexible CG in
experiments), and scaling r scales z. What it cannot see from r — the depth-dependent
coefficients — enters through gates: at every level the feature maps are multiplied by
G_l = 2 sigmoid(conv1x1(relu(conv3x3(F_l)))) of F_0 = (h / H0, b / H0), pooled to the level.
Encoder: two convolutions then the gate; 2x2 average pooling down; decoder: nearest-neighbour
upsampling, concatenation with the skip, two convolutions, the gate; a 1x1 convolution to 2
channels. Weights are trained in FP32 and used in BF16; accumulation is FP32. The last layer
starts at zero, so an untrained network leaves the two Jacobi sweeps. It is applied inside
flexible CG (the previous direction A-orthogonalised out), with the plain solve's stopping rule.

This module holds the parameter layout shared by the device kernels, the training loop and the
FP64 CPU reference used to check gradients.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

DEPTH_SCALE = 20.0  # H0, metres
OMEGA = 0.5         # damping of the Jacobi sweeps (keeps the cycle positive definite)
GATE_HIDDEN = 8     # channels of the gate networks' hidden layer


@dataclass(frozen=True)
class UNetSpec:
    channels: tuple = (8, 16, 32, 32)  # feature maps per level, finest first
    in_ch: int = 2
    out_ch: int = 2
    feat_ch: int = 2
    gate_hidden: int = GATE_HIDDEN
    stride: int = 1  # the network's grid is this many times coarser than the solver's (1, 2, 4)

    @property
    def levels(self) -> int:
        return len(self.channels)

    def layers(self):
        """(name, c_out, c_in, kernel, has_bias) in parameter order."""
        c = self.channels
        out = []
        cin = self.in_ch
        for l in range(self.levels):
            out.append((f"enc{l}a", c[l], cin, 3, False))
            out.append((f"enc{l}b", c[l], c[l], 3, False))
            cin = c[l]
        for l in range(self.levels - 2, -1, -1):
            out.append((f"dec{l}a", c[l], c[l + 1] + c[l], 3, False))
            out.append((f"dec{l}b", c[l], c[l], 3, False))
        out.append(("out", self.out_ch, c[0], 1, False))
        for l in range(self.levels):
            out.append((f"gate{l}a", self.gate_hidden, self.feat_ch, 3, True))
            out.append((f"gate{l}b", c[l], self.gate_hidden, 1, True))
        return out

    def offsets(self):
        """{name: (w_offset, b_offset or -1, c_out, c_in, k)} into the flat parameter vector."""
        off = 0
        table = {}
        for name, co, ci, k, has_b in self.layers():
            w = off
            off += co * ci * k * k
            b = -1
            if has_b:
                b = off
                off += co
            table[name] = (w, b, co, ci, k)
        return table

    def n_params(self) -> int:
        return sum(co * ci * k * k + (co if hb else 0) for _, co, ci, k, hb in self.layers())

    def flops_per_cell(self) -> float:
        """2 x multiply-adds per cell of the network's finest level for one application (gates
        excluded: they are computed once per solve). Per solver cell: divide by stride**2."""
        f = 0.0
        for name, co, ci, k, _ in self.layers():
            if name.startswith("gate"):
                continue
            level = 0 if name == "out" else int(name[3])
            f += 2.0 * co * ci * k * k / (4.0 ** level)
        return f

    def fused_maps(self) -> tuple:
        """Which of the first level's maps the device keeps on chip: (A, DA, D). A: the two
        encoder layers run as one launch, their intermediate map in shared memory; D: the 1x1
        output layer runs in the last decoder layer's epilogue; DA: the two decoder layers and the
        output layer run as one launch (16 channels at the second level)."""
        a = self.channels[0] == 8 and self.in_ch == 2
        d = self.channels[0] == 8 and self.out_ch == 2
        da = d and self.levels > 2 and self.channels[1] == 16
        return a, da, d

    def bytes_per_cell(self) -> float:
        """Algorithmic DRAM bytes of one application per cell of the finest level, for the
        device's channels-innermost BF16 activations: every convolution reads each of its inputs
        and its gate once and writes its output once (a pooled input is read at the finer level,
        an upsampled one at the coarser); the input is 2 BF16 channels, the output 2 FP32. Maps
        that the device keeps on chip (`fused_maps`) are not counted."""
        c, L, b = self.channels, self.levels, 2.0
        on_chip_a, on_chip_da, on_chip_d = self.fused_maps()
        per = [0.0] * L  # bytes per pixel of level l
        for l in range(L):
            cin = self.in_ch if l == 0 else c[l - 1]
            src = b * cin * (4.0 if l > 0 else 1.0)  # enc_a reads its input (pooled: 4 finer pixels)
            a_io = 0.0 if (l == 0 and on_chip_a) else 2 * b * c[l]  # A written by enc_a, read by enc_b
            per[l] += src + a_io + 2 * b * c[l]      # enc_b: the gate in, E out
        for l in range(L - 2, -1, -1):
            below = b * c[l + 1] / 4.0               # the upsampled map, read once at its level
            da_io = 0.0 if (l == 0 and on_chip_da) else 2 * b * c[l]  # DA written by dec_a, read by dec_b
            per[l] += below + b * c[l] + da_io       # dec_a: up(below) and E in
            per[l] += b * c[l]                       # dec_b: the gate in ...
            if l > 0:
                per[l] += b * c[l]                   # ... D out
            elif not on_chip_d:
                per[l] += 2 * b * c[l]               # ... D out, and the output layer reads it
        per[0] += 4.0 * self.out_ch                  # the FP32 output
        return sum(v / 4.0 ** l for l, v in enumerate(per))


def init_params(spec: UNetSpec, seed: int = 0) -> np.ndarray:
    """Scaled normal weights, zero biases, a zero output layer (the network starts at zero)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(spec.n_params(), dtype=np.float32)
    for name, (w, b, co, ci, k) in spec.offsets().items():
        if name == "out":
            continue
        std = np.sqrt(1.0 / (ci * k * k))
        p[w : w + co * ci * k * k] = rng.normal(0.0, std, co * ci * k * k).astype(np.float32)
    return p


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    rounding = 0x7FFF + ((a >> 16) & 1)
    r = ((a + rounding) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)
