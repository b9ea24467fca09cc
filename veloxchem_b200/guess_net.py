"""The density-block network of the learned initial guess, driven through the
library's own CUDA kernels (vlx_b200_mlp_*, vlx_b200_adam_step,
vlx_b200_to_bf16).  torch only holds the device buffers and streams.

Architecture: in -> 128 -> 128 -> out, SiLU after the two hidden layers
(three linear layers), FP32 weights for training, BF16 weights for inference.
"""

import ctypes

import numpy as np

from . import _native as nat


def _torch():
    import torch
    return torch


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class GuessMLP:
    def __init__(self, n_in, n_out, width=128, depth=3, seed=0, device=0):
        torch = _torch()
        self.dev = torch.device('cuda', device)
        self.dims = [n_in] + [width] * (depth - 1) + [n_out]
        rng = np.random.default_rng(seed)
        self.W, self.b = [], []
        for i in range(depth):
            k, n = self.dims[i], self.dims[i + 1]
            w = rng.standard_normal((n, k)) * np.sqrt(2.0 / k) * (0.5 if i == depth - 1 else 1.0)
            self.W.append(torch.tensor(w, dtype=torch.float32, device=self.dev))
            self.b.append(torch.zeros(n, dtype=torch.float32, device=self.dev))
        self._adam = None
        self.step = 0
        self._bf16 = None

    # ---- parameters
    def params(self):
        out = []
        for w, b in zip(self.W, self.b):
            out += [w, b]
        return out

    def state_dict(self):
        d = {}
        for i, (w, b) in enumerate(zip(self.W, self.b)):
            d['W%d' % i] = w.cpu().numpy()
            d['b%d' % i] = b.cpu().numpy()
        return d

    def load_state_dict(self, d):
        torch = _torch()
        for i in range(len(self.W)):
            self.W[i] = torch.tensor(np.asarray(d['W%d' % i]), dtype=torch.float32, device=self.dev)
            self.b[i] = torch.tensor(np.asarray(d['b%d' % i]), dtype=torch.float32, device=self.dev)
        self._bf16 = None

    def _stream(self):
        return ctypes.c_void_p(_torch().cuda.current_stream(self.dev).cuda_stream)

    # ---- training
    def forward(self, x, keep=False):
        """x: [M, n_in] float32 device tensor; keep=True stores what backward needs."""
        torch = _torch()
        h = x.contiguous()
        cache = []
        st = self._stream()
        for i, (w, b) in enumerate(zip(self.W, self.b)):
            act = 1 if i < len(self.W) - 1 else 0
            m, k, n = h.shape[0], w.shape[1], w.shape[0]
            y = torch.empty((m, n), dtype=torch.float32, device=self.dev)
            z = torch.empty_like(y) if (keep and act) else None
            nat.check(nat.lib().vlx_b200_mlp_linear(_p(h), _p(w), _p(b), _p(z), _p(y), m, k, n, act, st),
                      'mlp_linear')
            cache.append((h, z))
            h = y
        return (h, cache) if keep else h

    def backward(self, dy, cache):
        """Gradients [(dW, db)] per layer for the output gradient dy."""
        torch = _torch()
        grads = [None] * len(self.W)
        g = dy.contiguous()
        st = self._stream()
        for i in range(len(self.W) - 1, -1, -1):
            w = self.W[i]
            h, z = cache[i]
            act = 1 if i < len(self.W) - 1 else 0
            m, k, n = h.shape[0], w.shape[1], w.shape[0]
            dw = torch.empty_like(w)
            db = torch.empty_like(self.b[i])
            dz = torch.empty_like(g) if act else None
            dx = torch.empty_like(h) if i > 0 else None
            nat.check(nat.lib().vlx_b200_mlp_linear_backward(_p(h), _p(w), _p(z), _p(g), _p(dz), _p(dx), _p(dw),
                                                              _p(db), m, k, n, act, st), 'mlp_linear_backward')
            grads[i] = (dw, db)
            g = dx
        return grads

    def mse(self, y, t, mask):
        """Masked mean squared error (device FP64 scalar) and dL/dy."""
        torch = _torch()
        dy = torch.empty_like(y)
        loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        count = float(mask.sum().item())
        nat.check(nat.lib().vlx_b200_mlp_mse(_p(y), _p(t), _p(mask), _p(dy), _p(loss), y.numel(), max(count, 1.0),
                                             self._stream()), 'mlp_mse')
        return loss / max(count, 1.0), dy

    def adam_step(self, grads, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        torch = _torch()
        if self._adam is None:
            self._adam = [(torch.zeros_like(p), torch.zeros_like(p)) for p in self.params()]
        self.step += 1
        flat = []
        for dw, db in grads:
            flat += [dw, db]
        st = self._stream()
        for p, g, (m, v) in zip(self.params(), flat, self._adam):
            nat.check(nat.lib().vlx_b200_adam_step(_p(p), _p(g), _p(m), _p(v), p.numel(), lr, beta1, beta2, eps,
                                                   self.step, st), 'adam_step')
        self._bf16 = None

    # ---- inference
    def _bf16_weights(self):
        torch = _torch()
        if self._bf16 is None:
            self._bf16 = []
            for w in self.W:
                wb = torch.empty(w.shape, dtype=torch.bfloat16, device=self.dev)
                nat.check(nat.lib().vlx_b200_to_bf16(_p(w), _p(wb), w.numel(), self._stream()), 'to_bf16')
                self._bf16.append(wb)
        return self._bf16

    def predict_bf16(self, x):
        """Inference with BF16 weights and BF16-rounded inputs, FP32 accumulation."""
        torch = _torch()
        h = x.contiguous()
        st = self._stream()
        for i, (wb, b) in enumerate(zip(self._bf16_weights(), self.b)):
            act = 1 if i < len(self.W) - 1 else 0
            m, k, n = h.shape[0], wb.shape[1], wb.shape[0]
            y = torch.empty((m, n), dtype=torch.float32, device=self.dev)
            nat.check(nat.lib().vlx_b200_mlp_linear_bf16(_p(h), _p(wb), _p(b), _p(y), m, k, n, act, st),
                      'mlp_linear_bf16')
            h = y
        return h
