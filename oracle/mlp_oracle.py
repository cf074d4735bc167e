"""Numpy restatement of the learned-guess network (the checker of the
tcgen05 kernels in distributed-cfd-solver_b200/csrc/mlp.cu).  Test
infrastructure only.

Network: 48 -> 64 -> 64 -> 16, ReLU, weights rounded to bf16, hidden
activations rounded to bf16 after bias + ReLU (they are tensor-core
operands), FP32 accumulation.  Loss: mean over rows x nvars of (y - t)^2.
With `rounding=True` the backward pass rounds dY, dZ2 and dZ1 to bf16 where
the kernels stage them as tensor-core operands; with `rounding=False` it is
the exact FP64 gradient of the unrounded network (checked against central
differences in tests/test_mlp_cpu.py).
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 48, 64, 16
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * IN
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUT * HID
N_PARAMS = OFF_B3 + OUT


def bf16(x):
    """Round to bf16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def from_bits(b):
    return (np.ascontiguousarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    W1 = p[OFF_W1:OFF_B1].reshape(HID, IN)
    b1 = p[OFF_B1:OFF_W2]
    W2 = p[OFF_W2:OFF_B2].reshape(HID, HID)
    b2 = p[OFF_B2:OFF_W3]
    W3 = p[OFF_W3:OFF_B3].reshape(OUT, HID)
    b3 = p[OFF_B3:]
    return W1, b1, W2, b2, W3, b3


def _f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def forward(p, X, rounding=True):
    """X: features (float rows x 48, already bf16 values when rounding)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    r = bf16 if rounding else (lambda a: a)
    f = _f32 if rounding else (lambda a: a)
    W1r, W2r, W3r = r(W1), r(W2), r(W3)
    z1 = f(f(X @ W1r.T) + f(b1))
    h1 = r(np.maximum(z1, 0.0))
    z2 = f(f(h1 @ W2r.T) + f(b2))
    h2 = r(np.maximum(z2, 0.0))
    y = f(f(h2 @ W3r.T) + f(b3))
    return y, (X, z1, h1, z2, h2, W1r, W2r, W3r)


def loss_and_grad(p, X, T, nvars, rounding=True):
    y, (X, z1, h1, z2, h2, W1r, W2r, W3r) = forward(p, X, rounding)
    r = bf16 if rounding else (lambda a: a)
    n = X.shape[0]
    mask = np.zeros(OUT)
    mask[:nvars] = 1.0
    d = (y - T) * mask
    loss = float((d * d).sum() / (n * nvars))
    scale = 2.0 / (n * nvars)
    dy = r(d)
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = (dy.T @ h2).ravel() * scale
    g[OFF_B3:] = dy.sum(axis=0) * scale
    dz2 = r((dy @ W3r) * (z2 > 0))
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).ravel() * scale
    g[OFF_B2:OFF_W3] = dz2.sum(axis=0) * scale
    dz1 = r((dz2 @ W2r) * (z1 > 0))
    g[OFF_W1:OFF_B1] = (dz1.T @ X).ravel() * scale
    g[OFF_B1:OFF_W2] = dz1.sum(axis=0) * scale
    return loss, g
