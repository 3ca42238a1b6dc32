"""FP64 numpy restatement of the estimator MLP (test infrastructure only).

48 -> 64 -> 64 -> 64 -> 2 with ReLU on the hidden layers, parameters packed as
[W1 (64x48), b1, W2 (64x64), b2, W3 (64x64), b3, W4 (2x64), b4] (row-major,
W[j][k] multiplies input k for output j) - the layout the CUDA kernels use.
Loss = sum over samples and outputs of (y_hat - y)^2.  Used to check the GPU
forward pass and gradients.
"""
from __future__ import annotations

import numpy as np

SHAPES = [(64, 48), (64, 64), (64, 64), (2, 64)]


def unpack(p: np.ndarray):
    out, off = [], 0
    for o, i in SHAPES:
        W = p[off:off + o * i].reshape(o, i)
        off += o * i
        b = p[off:off + o]
        off += o
        out.append((W, b))
    assert off == p.size == 11586
    return out


def forward(p: np.ndarray, X: np.ndarray):
    layers = unpack(np.asarray(p, np.float64))
    a = np.asarray(X, np.float64)
    acts, pres = [a], []
    for li, (W, b) in enumerate(layers):
        z = a @ W.T + b
        pres.append(z)
        a = np.maximum(z, 0.0) if li < 3 else z
        acts.append(a)
    return a, acts, pres


def loss_and_grad(p: np.ndarray, X: np.ndarray, Y: np.ndarray):
    yhat, acts, pres = forward(p, X)
    d = 2.0 * (yhat - np.asarray(Y, np.float64))
    loss = float(np.sum((yhat - Y) ** 2))
    layers = unpack(np.asarray(p, np.float64))
    grads = []
    for li in range(3, -1, -1):
        W, _ = layers[li]
        gW = d.T @ acts[li]
        gb = d.sum(axis=0)
        grads.append((gW, gb))
        if li > 0:
            d = (d @ W) * (pres[li - 1] > 0)
    flat = []
    for gW, gb in reversed(grads):
        flat += [gW.ravel(), gb]
    return loss, np.concatenate(flat)
