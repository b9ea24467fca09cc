"""The learned-guess network's CUDA kernels (forward, backward, masked error,
Adam, BF16 inference) against the float64 numpy oracle.  Tolerances: FP32
kernels 2e-5 relative to the largest magnitude of each tensor; the BF16
forward against the oracle evaluated on BF16-rounded inputs and weights,
1e-3 relative (only the FP32 accumulation order differs)."""

import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _net(dims, seed):
    import torch
    from veloxchem_b200.guess_net import GuessMLP
    net = GuessMLP(dims[0], dims[-1], width=dims[1], depth=len(dims) - 1, seed=seed)
    rng = np.random.default_rng(seed + 1)
    for i in range(len(net.b)):
        net.b[i] = torch.tensor(0.1 * rng.standard_normal(net.b[i].shape[0]), dtype=torch.float32,
                                device=net.dev)
    layers = [(net.W[i].double().cpu().numpy(), net.b[i].double().cpu().numpy(), i < len(net.W) - 1)
              for i in range(len(net.W))]
    return net, layers


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


@pytest.mark.parametrize('m', [1, 37, 1000])
def test_forward_backward_against_oracle(m):
    import torch
    dims = [36, 128, 128, 196]
    net, layers = _net(dims, 5)
    rng = np.random.default_rng(m)
    x = rng.standard_normal((m, dims[0])).astype(np.float32)
    t = rng.standard_normal((m, dims[-1])).astype(np.float32)
    mask = (rng.uniform(size=(m, dims[-1])) > 0.4).astype(np.float32)
    xd = torch.tensor(x, device=net.dev)
    y, cache = net.forward(xd, keep=True)
    loss, dy = net.mse(y, torch.tensor(t, device=net.dev), torch.tensor(mask, device=net.dev))
    grads = net.backward(dy, cache)
    torch.cuda.synchronize()
    yo, co = mo.forward(x.astype(np.float64), layers)
    lo, dyo = mo.mse(yo, t.astype(np.float64), mask.astype(np.float64))
    go = mo.backward(dyo, layers, co)
    assert _rel(y.double().cpu().numpy(), yo) < 2e-5
    assert abs(float(loss.item()) - lo) < 2e-5 * lo
    for (dw, db), (dwo, dbo) in zip(grads, go):
        assert _rel(dw.double().cpu().numpy(), dwo) < 2e-5
        assert _rel(db.double().cpu().numpy(), dbo) < 2e-5


def test_adam_step_against_oracle():
    import torch
    dims = [12, 16, 16, 8]
    net, layers = _net(dims, 9)
    rng = np.random.default_rng(0)
    x = torch.tensor(rng.standard_normal((20, 12)).astype(np.float32), device=net.dev)
    t = torch.tensor(rng.standard_normal((20, 8)).astype(np.float32), device=net.dev)
    mask = torch.ones_like(t)
    ms = [(np.zeros_like(w), np.zeros_like(b)) for w, b, _ in layers]
    vs = [(np.zeros_like(w), np.zeros_like(b)) for w, b, _ in layers]
    for step in (1, 2, 3):
        y, cache = net.forward(x, keep=True)
        _, dy = net.mse(y, t, mask)
        grads = net.backward(dy, cache)
        host = [(dw.double().cpu().numpy(), db.double().cpu().numpy()) for dw, db in grads]
        net.adam_step(grads, lr=1e-2)
        for i, (w, b, act) in enumerate(layers):
            w2, mw, vw = mo.adam(w, host[i][0], ms[i][0], vs[i][0], step, 1e-2)
            b2, mb, vb = mo.adam(b, host[i][1], ms[i][1], vs[i][1], step, 1e-2)
            layers[i] = (w2, b2, act)
            ms[i], vs[i] = (mw, mb), (vw, vb)
            assert _rel(net.W[i].double().cpu().numpy(), w2) < 1e-5
            assert _rel(net.b[i].double().cpu().numpy(), b2) < 1e-5


def test_bf16_inference_against_rounded_oracle():
    import torch
    dims = [36, 128, 128, 70]
    net, layers = _net(dims, 21)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((300, 36)).astype(np.float32)
    y = net.predict_bf16(torch.tensor(x, device=net.dev)).double().cpu().numpy()
    h = x.astype(np.float64)
    for w, b, act in layers:
        z = mo.bf16_round(h.astype(np.float32)) @ mo.bf16_round(w.astype(np.float32)).T + b
        h = mo.silu(z) if act else z
    assert _rel(y, h) < 1e-3
    full = mo.forward(x.astype(np.float64), layers)[0]
    assert 1e-5 < _rel(y, full) < 5e-2
