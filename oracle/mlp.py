"""CPU restatement of the surrogate network (include/orkan_mlp.h) -- TEST INFRASTRUCTURE ONLY.

The network has no counterpart in the reference; this numpy (float64) version is the
checker for the FP32 CUDA kernels in orkan_b200/csrc/cuda/mlp.cu:

    z1 = x W1 + b1,  a1 = gelu(z1),  z2 = a1 W2 + b2,  a2 = gelu(z2),  y = a2 . w3 + b3
    gelu(z) = z Phi(z) = z (1 + erf(z / sqrt 2)) / 2
    L = mean_b (y_b - t_b)^2
    Adam: m = 0.9 m + 0.1 g, v = 0.999 v + 0.001 g^2, p -= lr mhat / (sqrt(vhat) + 1e-8)

Parameter vector layout: W1 [n_in][h], b1 [h], W2 [h][h], b2 [h], w3 [h], b3 [1].
Its own gradients are pinned by central finite differences in tests/test_mlp_oracle.py.
"""
from __future__ import annotations

import math

import numpy as np

_erf = np.vectorize(math.erf, otypes=[np.float64])


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(p, n_in, h):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + n_in * h].reshape(n_in, h); o += n_in * h
    b1 = p[o:o + h]; o += h
    W2 = p[o:o + h * h].reshape(h, h); o += h * h
    b2 = p[o:o + h]; o += h
    w3 = p[o:o + h]; o += h
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def pack(W1, b1, W2, b2, w3, b3):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, w3, np.atleast_1d(b3)])


def forward(p, x, n_in, h):
    W1, b1, W2, b2, w3, b3 = unpack(p, n_in, h)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W1 + b1
    a1 = gelu(z1)
    z2 = a1 @ W2 + b2
    a2 = gelu(z2)
    y = a2 @ w3 + b3
    return y, (x, z1, a1, z2, a2)


def gradients(p, x, t, n_in, h):
    """(loss, dL/dp, dL/dx) of the mean squared error."""
    W1, b1, W2, b2, w3, b3 = unpack(p, n_in, h)
    y, (x, z1, a1, z2, a2) = forward(p, x, n_in, h)
    t = np.asarray(t, dtype=np.float64)
    B = len(y)
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d / B
    gw3 = a2.T @ dy
    gb3 = dy.sum()
    dz2 = np.outer(dy, w3) * gelu_grad(z2)
    gW2 = a1.T @ dz2
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ W2.T) * gelu_grad(z1)
    gW1 = x.T @ dz1
    gb1 = dz1.sum(axis=0)
    gx = dz1 @ W1.T
    return loss, pack(gW1, gb1, gW2, gb2, gw3, gb3), gx


def input_gradient(p, x, n_in, h):
    """d f / d x for every row (the ascent direction of the proposals)."""
    W1, b1, W2, b2, w3, b3 = unpack(p, n_in, h)
    y, (x, z1, a1, z2, a2) = forward(p, x, n_in, h)
    dz2 = np.outer(np.ones(len(y)), w3) * gelu_grad(z2)
    dz1 = (dz2 @ W2.T) * gelu_grad(z1)
    return dz1 @ W1.T


def adam_step(p, g, m, v, t, lr):
    b1, b2, eps = 0.9, 0.999, 1e-8
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def init_params(n_in, h, seed):
    """The library's deterministic initialisation (splitmix64 stream, uniform +-sqrt(6/fan_in))."""
    M64 = (1 << 64) - 1

    def mix(z):
        z = (z + 0x9E3779B97F4A7C15) & M64
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    st = seed & M64

    def uni(bound):
        nonlocal st
        st = (st + 0x9E3779B97F4A7C15) & M64
        z = mix(st)
        return np.float32(((z >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0) * bound

    b1 = np.sqrt(np.float32(6.0) / np.float32(n_in))
    b2 = np.sqrt(np.float32(6.0) / np.float32(h))
    W1 = np.array([uni(b1) for _ in range(n_in * h)], dtype=np.float32)
    W2 = np.array([uni(b2) for _ in range(h * h)], dtype=np.float32)
    w3 = np.array([uni(b2) for _ in range(h)], dtype=np.float32)
    z = np.zeros(h, dtype=np.float32)
    return np.concatenate([W1, z, W2, z, w3, np.zeros(1, np.float32)])
