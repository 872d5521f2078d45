"""Test infrastructure only: an FP64 numpy restatement of the learned correction's perceptron
(softx-d-16-00083_b200/csrc/mlp.cu), the checker of its hand-written GPU forward and backward kernels.

    y = W3 gelu(W2 gelu(W1 x + b1) + b2) + b3,   gelu(z) = z Phi(z)
    loss = mean over all entries of w_col (y - t)^2

The GPU multiplies with BF16 copies of the weights (FP32 accumulation); the oracle rounds the weights
to BF16 the same way (round to nearest even) and computes everything else in FP64.  Parameters are one
flat FP32 vector in the order W1 (hidden x in, row-major), b1, W2, b2, W3, b3.
"""
import math

import numpy as np


def bf16(a):
    """Round FP32 values to BF16 (nearest, ties to even) and return them as FP64."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def split(params, dims):
    i, h1, h2, o = dims
    sizes = [h1 * i, h1, h2 * h1, h2, o * h2, o]
    out, k = [], 0
    for s in sizes:
        out.append(np.asarray(params[k:k + s], dtype=np.float64))
        k += s
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(h1, i), b1, W2.reshape(h2, h1), b2, W3.reshape(o, h2), b3


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(params, dims, x):
    W1, b1, W2, b2, W3, b3 = split(params, dims)
    W1, W2, W3 = bf16(W1), bf16(W2), bf16(W3)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    y = h2 @ W3.T + b3
    return y, (x, z1, h1, z2, h2)


def gradients(params, dims, x, t, w=None):
    """Loss and its gradient with respect to the flat parameter vector."""
    W1, b1, W2, b2, W3, b3 = split(params, dims)
    W1q, W2q, W3q = bf16(W1), bf16(W2), bf16(W3)
    y, (x, z1, h1, z2, h2) = forward(params, dims, x)
    t = np.asarray(t, dtype=np.float64)
    wcol = np.ones(y.shape[1]) if w is None else np.asarray(w, dtype=np.float64)
    n = y.size
    d = y - t
    loss = float((wcol[None] * d * d).sum() / n)
    dy = 2.0 * wcol[None] * d / n
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    dz2 = (dy @ W3q) * gelu_grad(z2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2q) * gelu_grad(z1)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
