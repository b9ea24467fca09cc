"""The learned-guess network's CPU oracle against finite differences of its
own loss (the oracle has no reference counterpart to be pinned against)."""

import numpy as np

from oracle import mlp_oracle as mo


def _layers(rng, dims):
    return [(rng.standard_normal((dims[i + 1], dims[i])) / np.sqrt(dims[i]), 0.1 * rng.standard_normal(dims[i + 1]),
             i < len(dims) - 2) for i in range(len(dims) - 1)]


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    layers = _layers(rng, [7, 9, 8, 5])
    x = rng.standard_normal((11, 7))
    t = rng.standard_normal((11, 5))
    mask = (rng.uniform(size=(11, 5)) > 0.3).astype(np.float64)
    y, cache = mo.forward(x, layers)
    loss, dy = mo.mse(y, t, mask)
    grads = mo.backward(dy, layers, cache)
    h = 1e-6
    for li, (w, b, act) in enumerate(layers):
        for arr, g in ((w, grads[li][0]), (b, grads[li][1])):
            for idx in [tuple(rng.integers(0, s) for s in arr.shape) for _ in range(5)]:
                old = arr[idx]
                arr[idx] = old + h
                lp = mo.mse(mo.forward(x, layers)[0], t, mask)[0]
                arr[idx] = old - h
                lm = mo.mse(mo.forward(x, layers)[0], t, mask)[0]
                arr[idx] = old
                assert abs((lp - lm) / (2 * h) - g[idx]) < 1e-6 * max(1.0, abs(g[idx]))


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e-3], dtype=np.float32)
    r = mo.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625 and r[3] == -2.5
    assert abs(r[4] - 3.0e-3) / 3.0e-3 < 2 ** -8
