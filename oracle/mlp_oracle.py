"""FP64 oracle of the surrogate network's forward pass, loss and gradient.  TEST
INFRASTRUCTURE ONLY (see oracle.py).

Network: x (8) -> [W_l x + b_l, GELU] x 4 (width 256) -> w_5 . h + b_5; loss = sum of
squared errors.  Parameters are one flat vector, layer l stored as W_l [out x in]
row-major followed by b_l, the layout the library's opb_mlp_* kernels use.  GELU is the
exact form 0.5 z (1 + erf(z / sqrt 2)).  The gradient is checked against central finite
differences in tests/test_oracle.py, and the library's gradient against this one.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf

SIZES = [(8, 256), (256, 256), (256, 256), (256, 256), (256, 1)]


def layout():
    off, out = 0, []
    for i, o in SIZES:
        w = (off, off + i * o)
        off += i * o
        b = (off, off + o)
        off += o
        out.append((i, o, w, b))
    return out, off


def unpack(theta):
    L, _ = layout()
    return [(theta[w[0]:w[1]].reshape(o, i), theta[b[0]:b[1]]) for i, o, w, b in L]


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(theta, X):
    layers = unpack(np.asarray(theta, dtype=np.float64))
    h = np.asarray(X, dtype=np.float64)
    cache = []
    for W, b in layers[:-1]:
        z = h @ W.T + b
        cache.append((h, z))
        h = gelu(z)
    W, b = layers[-1]
    return (h @ W.T + b)[:, 0], cache, h


def bf16_round(a):
    """Round to the nearest BF16 value (ties to even), returned as FP64."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (u & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)


def forward_inference(theta, X):
    """The numerics of the library's tensor-core inference (opb_mlp_infer), in FP64: every
    parameter and the input rounded to BF16 (the packed weights), products summed exactly,
    the exact-erf GELU, each hidden layer's activations rounded to BF16 (they are stored as
    BF16 between layers), then y = w5 . h4 + b5.  Returns y [n]."""
    layers = [(bf16_round(W), bf16_round(b)) for W, b in unpack(np.asarray(theta, dtype=np.float64))]
    h = bf16_round(X)
    for W, b in layers[:-1]:
        h = bf16_round(gelu(h @ W.T + b))
    W, b = layers[-1]
    return (h @ W.T + b)[:, 0]


def loss_grad(theta, X, t):
    """Sum of squared errors and its gradient; the library's kernels use the gradient of
    the mean (the 1/B factor), so compare with grad / B."""
    theta = np.asarray(theta, dtype=np.float64)
    y, cache, h4 = forward(theta, X)
    e = y - np.asarray(t, dtype=np.float64)
    loss = float(np.sum(e * e))
    L, n = layout()
    g = np.zeros(n)
    layers = unpack(theta)
    dy = 2.0 * e
    i, o, w, b = L[-1]
    g[w[0]:w[1]] = (dy[:, None] * h4).sum(axis=0)
    g[b[0]:b[1]] = dy.sum()
    dh = dy[:, None] * layers[-1][0][0][None, :]
    for l in range(3, -1, -1):
        hin, z = cache[l]
        dz = dh * gelu_grad(z)
        i, o, w, b = L[l]
        g[w[0]:w[1]] = (dz.T @ hin).ravel()
        g[b[0]:b[1]] = dz.sum(axis=0)
        dh = dz @ layers[l][0]
    return loss, g
