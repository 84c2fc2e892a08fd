"""Test infrastructure only: CPU (numpy, FP64) forward pass and hand-written
backpropagation of the surrogate ensemble, same parameter layout, features,
target standardisation and loss as the GPU kernels
(chaos_oneapi_b200/csrc/mlp.cu).  Pinned by finite differences in
tests/test_mlp_oracle.py; the GPU gradients are checked against it."""
from __future__ import annotations

import numpy as np

FEAT, OUTPAD = 16, 16


def bf16_round(a):
    """Round float values to bfloat16 (nearest, ties to even), back as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layout(width):
    W = width
    sizes = [(FEAT, W), (W,), (W, W), (W,), (W, W), (W,), (W, OUTPAD), (OUTPAD,)]
    offs, o = [], 0
    for s in sizes:
        offs.append((o, s))
        o += int(np.prod(s))
    return offs, o


def unpack(p, width):
    offs, _ = layout(width)
    return [p[o:o + int(np.prod(s))].reshape(s).astype(np.float64) for o, s in offs]


DEFAULT_FREQS = np.array([[0.5 * (j + 1), 0.0] if f % 2 == 0 else [0.0, 0.5 * (j + 1)]
                          for j in range(4) for f in range(2)])


def features(xy, domain, freqs=DEFAULT_FREQS):
    u0, u1, v0, v1 = domain
    u = (xy[:, 0] - u0) / (u1 - u0)
    v = (xy[:, 1] - v0) / (v1 - v0)
    cols = []
    for w in np.asarray(freqs, dtype=np.float64):
        ph = 2 * np.pi * (w[0] * u + w[1] * v)
        cols += [np.sin(ph), np.cos(ph)]
    return np.stack(cols, axis=1)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def loss_and_grad(p, width, xy, T, tmean, tstd, domain, outs=3, round_weights=True,
                  freqs=DEFAULT_FREQS):
    """Loss (mean squared error of standardised targets) and its gradient
    with respect to the flat parameter vector p of one network."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, width)
    if round_weights:  # the GPU multiplies BF16 copies of the weights
        W1, W2, W3, W4 = (bf16_round(w) for w in (W1, W2, W3, W4))
    X = features(xy, domain, freqs)
    z1 = X @ W1 + b1
    a1 = silu(z1)
    z2 = a1 @ W2 + b2
    a2 = silu(z2)
    z3 = a2 @ W3 + b3
    a3 = silu(z3)
    y = a3 @ W4 + b4
    t = (T - tmean[:outs]) / tstd[:outs]
    d = y[:, :outs] - t
    n = d.size
    loss = float((d * d).sum() / n)
    dy = np.zeros_like(y)
    dy[:, :outs] = 2.0 * d / n
    gW4 = a3.T @ dy
    gb4 = dy.sum(0)
    dz3 = (dy @ W4.T) * dsilu(z3)
    gW3 = a2.T @ dz3
    gb3 = dz3.sum(0)
    dz2 = (dz3 @ W3.T) * dsilu(z2)
    gW2 = a1.T @ dz2
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2.T) * dsilu(z1)
    gW1 = X.T @ dz1
    gb1 = dz1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4)])
    return loss, g
