"""TEST INFRASTRUCTURE ONLY: numpy restatement of the learned warm-start network's
arithmetic, the checker of libfemtools_b200's BF16 tensor-core convolution kernels.

The reference (FEMTools.jl) has no learned component, so there is no reference
implementation to follow; this oracle restates the operations the library's kernels
compute: a 3×3 same-padded convolution on NHWC grids (zero outside the grid), ReLU,
a mean-square loss, their backward passes, and Adam (Kingma & Ba, 2015). BF16
operands are modelled by rounding to BF16 (round to nearest even) before an FP32
(float64 here) accumulation. Parity unpinned against any external implementation:
the backward passes are pinned by finite differences of the forward pass
(tests/test_cnn_oracle.py).

Weights use the library's layout: w[co][tap·ci + c] with tap = 3·ky + kx, padded
to 9·ci + 8 columns.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    r = ((u + rounding) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(x.shape)


def kpad(ci):
    return 9 * ci + 8


def conv3x3(x, w, b=None):
    """y[n, y, x, co] = Σ_{ky,kx,c} x[n, y+ky−1, x+kx−1, c]·w[co][(3ky+kx)·ci + c] (+ b[co])."""
    B, H, W, ci = x.shape
    co = w.shape[0]
    xp = np.zeros((B, H + 2, W + 2, ci))
    xp[:, 1:-1, 1:-1, :] = x
    y = np.zeros((B, H, W, co))
    for ky in range(3):
        for kx in range(3):
            tap = 3 * ky + kx
            wk = w[:, tap * ci:(tap + 1) * ci].astype(np.float64)     # co × ci
            y += np.einsum("nyxc,oc->nyxo", xp[:, ky:ky + H, kx:kx + W, :], wk)
    if b is not None:
        y += b
    return y


def conv3x3_backward(x, w, dy):
    """(dx, dw, db) of y = conv3x3(x, w, b) for the output gradient dy."""
    B, H, W, ci = x.shape
    co = w.shape[0]
    xp = np.zeros((B, H + 2, W + 2, ci))
    xp[:, 1:-1, 1:-1, :] = x
    dxp = np.zeros_like(xp)
    dw = np.zeros(w.shape)
    for ky in range(3):
        for kx in range(3):
            tap = 3 * ky + kx
            wk = w[:, tap * ci:(tap + 1) * ci].astype(np.float64)
            dxp[:, ky:ky + H, kx:kx + W, :] += np.einsum("nyxo,oc->nyxc", dy, wk)
            dw[:, tap * ci:(tap + 1) * ci] += np.einsum("nyxo,nyxc->oc", dy, xp[:, ky:ky + H, kx:kx + W, :])
    db = dy.sum(axis=(0, 1, 2))
    return dxp[:, 1:-1, 1:-1, :], dw, db


def forward(x, layers):
    """layers: list of (w, b, relu). Returns the activations [x, a1, ..., out]."""
    acts = [x]
    for w, b, relu in layers:
        y = conv3x3(acts[-1], w, b)
        acts.append(np.maximum(y, 0.0) if relu else y)
    return acts


def mse(out, target, nt, scale=1.0):
    """scale·Σ (out[..., :nt] − target)² and its gradient in out."""
    d = out[..., :nt] - target
    g = np.zeros_like(out)
    g[..., :nt] = 2.0 * scale * d
    return scale * float(np.sum(d * d)), g


def backward(acts, layers, dout):
    """Parameter gradients [(dw, db)] of the network for the output gradient dout."""
    grads = [None] * len(layers)
    dy = dout
    for li in range(len(layers) - 1, -1, -1):
        w, b, relu = layers[li]
        if relu:
            dy = dy * (acts[li + 1] > 0)
        dx, dw, db = conv3x3_backward(acts[li], w, dy)
        grads[li] = (dw, db)
        dy = dx
    return grads


def adam(w, m, v, g, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w, m, v
