"""Oracle (test infrastructure only): the surrogate network in numpy, FP64.

The learned part of the four-phonon screening has no counterpart in the
reference; this restates, for the gradient checks of the device kernels, the
network they train: 5 inputs -> 128 -> 128 -> 128 -> 1, SiLU after every
hidden layer, mean-squared-error loss.  Parameters are one flat vector in the
device order W1 (128x5, row-major), b1, W2 (128x128), b2, W3, b3, W4 (1x128), b4.

Only ``tests/`` may import this module.
"""
from __future__ import annotations

import numpy as np

SIZES = (5, 128, 128, 128, 1)


def n_params(sizes=SIZES):
    return sum(sizes[i + 1] * sizes[i] + sizes[i + 1] for i in range(len(sizes) - 1))


def unpack(p, sizes=SIZES):
    out, k = [], 0
    for i in range(len(sizes) - 1):
        o, n = sizes[i + 1], sizes[i]
        W = p[k:k + o * n].reshape(o, n)
        k += o * n
        b = p[k:k + o]
        k += o
        out.append((W, b))
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X, sizes=SIZES):
    """Outputs (n,) and the per-layer (input, pre-activation) cache."""
    layers = unpack(np.asarray(p, np.float64), sizes)
    a = np.asarray(X, np.float64)
    cache = []
    for i, (W, b) in enumerate(layers):
        z = a @ W.T + b
        cache.append((a, z))
        a = silu(z) if i < len(layers) - 1 else z
    return a[:, 0], cache


def loss_and_grad(p, X, y, sizes=SIZES):
    """Mean squared error and its gradient with respect to the flat parameters."""
    out, cache = forward(p, X, sizes)
    y = np.asarray(y, np.float64)
    n = len(y)
    r = out - y
    loss = float(np.mean(r * r))
    layers = unpack(np.asarray(p, np.float64), sizes)
    grads = []
    d = (2.0 / n) * r[:, None]                      # d loss / d z of the output layer
    for i in range(len(layers) - 1, -1, -1):
        a, z = cache[i]
        if i < len(layers) - 1:
            d = d * dsilu(z)
        W, _ = layers[i]
        grads.append((d.T @ a, d.sum(axis=0)))
        d = d @ W
    grads.reverse()
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
