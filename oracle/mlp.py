"""Test infrastructure: the CPU oracle of the surrogate network (wadi2d_b200/surrogate.py). The tests compare the
device's forward pass and gradients with it; it is never the implementation. The surrogate has no counterpart in the
reference (its critical-duration search and network are new pieces), so this oracle restates the network's definition
in FP64 and rounds to BF16 at the same points as the device: the weights' copies, the inputs, the activations between
layers and the gradients w.r.t. the pre-activations (round to nearest even, as __float2bfloat16_rn). The two then
differ only by the accumulation order of FP32 against FP64 sums (and the rare BF16 rounding that the difference
tips)."""

from __future__ import annotations

import numpy as np


def bf16(x) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as FP64 values."""
    a = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    bits = a.view(np.uint32).astype(np.uint64)
    r = ((bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _same(x) -> np.ndarray:
    return np.asarray(x, np.float64)


def forward(weights, x, rounded: bool = True):
    """Outputs, and the layers' inputs and FP64 pre-activations. weights: [(W (out x in), b)]. ``rounded``: round to
    BF16 where the device does (False: the plain FP64 network)."""
    r = bf16 if rounded else _same
    h = r(x)
    hs, zs = [h], []
    for i, (w, b) in enumerate(weights):
        z = h @ r(w).T + b
        zs.append(z)
        if i < len(weights) - 1:
            h = r(np.maximum(z, 0.0))
            hs.append(h)
    return zs[-1], hs, zs


def gradients(weights, x, t, rounded: bool = True):
    """Mean-square error and the gradients of the weights and biases, as the device forms them (``rounded``) or in
    plain FP64."""
    r = bf16 if rounded else _same
    y, hs, zs = forward(weights, x, rounded)
    n, nout = y.shape
    d = y - t
    loss = float((d * d).sum() / (n * nout))
    dz = r(np.float32(2.0 / (n * nout)) * d.astype(np.float32)) if rounded else 2.0 / (n * nout) * d
    gW, gb = [None] * len(weights), [None] * len(weights)
    for i in range(len(weights) - 1, -1, -1):
        w, _ = weights[i]
        gW[i] = dz.T @ hs[i]
        gb[i] = dz.sum(0)
        if i > 0:
            g = dz @ r(w)
            dz = r(np.where(zs[i - 1] > 0.0, g, 0.0))
    return loss, gW, gb
