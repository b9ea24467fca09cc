"""Batched Fock builds of many independent molecules on one GPU.

``FockBatch(screeners)`` wraps ``vlx_b200_batch_*``: all quartet classes of
all molecules run as one persistent launch per class, replayed from a CUDA
graph.  Each molecule's result is the same Fock matrix that
``FockDriver.compute`` (reference CFockDriver::compute,
src/t4c_func/FockDriver.cpp:120-172) returns for it alone; the reference has
no batched entry point.
"""

import ctypes

import numpy as np

from . import _native as nat


def _torch():
    import torch
    return torch


class FockBatch:
    """Independent molecules (their partitioned T4CScreener objects) built together."""

    def __init__(self, screeners, device=0):
        self.screeners = list(screeners)
        self.device = int(device)
        arr = (ctypes.c_void_p * len(self.screeners))(*[s.handle.value for s in self.screeners])
        h = ctypes.c_void_p()
        nat.check(nat.lib().vlx_b200_batch_create(ctypes.byref(h), arr, len(self.screeners)), 'batch_create')
        self._h = h
        off = (ctypes.c_longlong * (len(self.screeners) + 1))()
        nat.check(nat.lib().vlx_b200_batch_offsets(self._h, off), 'batch_offsets')
        self.offsets = np.array(off[:], dtype=np.int64)
        self.naos = [s.nao for s in self.screeners]
        self.last_stats = None

    def __del__(self):
        try:
            if getattr(self, '_h', None) is not None:
                nat.lib().vlx_b200_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def pack(self, matrices, out=None):
        """Packed FP64 host array of the molecules' nao x nao matrices."""
        buf = np.empty(int(self.offsets[-1])) if out is None else out
        for k, m in enumerate(matrices):
            buf[self.offsets[k]:self.offsets[k + 1]] = np.ascontiguousarray(m, dtype=np.float64).ravel()
        return buf

    def unpack(self, packed):
        return [np.asarray(packed[self.offsets[k]:self.offsets[k + 1]]).reshape(n, n)
                for k, n in enumerate(self.naos)]

    def build_device(self, d_densities, d_focks, label='2jk', exchange_factor=1.0, omega=0.0, ithreshold=12,
                     symmetric=True, stream=None, use_graph=True):
        """Enqueue one batched build on ``stream`` (a torch stream or raw handle);
        d_densities / d_focks are packed device tensors (float64)."""
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        sp = stream.cuda_stream if hasattr(stream, 'cuda_stream') else int(stream)
        if sp == 0:
            # torch's default stream is the legacy stream (handle 0); a NULL
            # stream would select the batch's own stream, which does not
            # order with it
            sp = 1  # cudaStreamLegacy
        stats = nat.Stats()
        nat.check(nat.lib().vlx_b200_batch_fock_build(self._h, ctypes.c_void_p(d_densities.data_ptr()),
                                                       int(symmetric), label.encode(), float(exchange_factor),
                                                       float(omega), int(ithreshold),
                                                       ctypes.c_void_p(d_focks.data_ptr()), ctypes.c_void_p(sp),
                                                       int(use_graph), ctypes.byref(stats)), 'batch_fock_build')
        self.last_stats = stats.as_dict()
        return d_focks

    def compute(self, densities, label='2jk', exchange_factor=1.0, omega=0.0, ithreshold=12, symmetric=True,
                use_graph=True):
        """Host densities in, host Fock matrices out (one per molecule)."""
        torch = _torch()
        dev = torch.device('cuda', self.device)
        d = torch.from_numpy(self.pack(densities)).to(dev)
        f = torch.empty_like(d)
        self.build_device(d, f, label, exchange_factor, omega, ithreshold, symmetric, use_graph=use_graph)
        return self.unpack(f.cpu().numpy())
