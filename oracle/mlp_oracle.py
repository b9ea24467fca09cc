"""CPU oracle (test infrastructure only) of the learned-guess network: the
forward pass, backward pass, masked squared error and Adam step that the
CUDA kernels in veloxchem_b200/csrc/vlx_mlp.cu implement, in float64 numpy.
Only tests import this module.  There is no reference counterpart (the
reference has no learned guess), so the oracle is pinned by finite
differences of its own loss (tests/test_mlp_oracle.py), not by reference
golden vectors."""

import numpy as np


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(x, layers):
    """layers: list of (W[N, K], b[N], act); returns output and the per-layer
    (input, pre-activation) cache."""
    cache = []
    h = np.asarray(x, dtype=np.float64)
    for w, b, act in layers:
        z = h @ w.T + b
        cache.append((h, z))
        h = silu(z) if act else z
    return h, cache


def mse(y, t, mask):
    r = y - t
    count = float(mask.sum())
    return float((mask * r * r).sum()) / count, 2.0 * mask * r / count


def backward(dy, layers, cache):
    """Gradients [(dW, db), ...] of the loss whose output gradient is dy."""
    grads = [None] * len(layers)
    g = dy
    for i in range(len(layers) - 1, -1, -1):
        w, b, act = layers[i]
        h, z = cache[i]
        if act:
            g = g * silu_grad(z)
        grads[i] = (g.T @ h, g.sum(axis=0))
        g = g @ w
    return grads


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def bf16_round(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)
