"""FockDriver: the reference's Fock-build API on the B200 kernels.

Mirrors src/pymodule/fockdriver.py and the pybind class ``_FockDriver``
(src/python/ExportT4CIntegrals.cpp:48-124):

* ``FockDriver(comm).compute(screener, *args)`` ->
  ``_compute_local_fock(screener, rank, nodes, *args)`` (fockdriver.py:69-72);
* ``_compute_fock_omp(screener, density, label, exchange_factor, omega,
  ithreshold) -> Matrix`` and the ``(Matrices, [labels])`` overload
  (FockDriver.cpp:120-230);
* ``_compute_local_fock(screener, rank, nodes, ...)`` (FockDriver.cpp:234-352);
* ``compute_eri(molecule, basis, eri_thresh)`` (fockdriver.py:93-114,
  FockDriver.cpp:76-117);
* ``_set_block_size_factor(factor)`` (fockdriver.py:120-135).

The density is copied to the GPU, the Fock matrix copied back into a new
``Matrix`` with the density's layout (reference: CMatrix(density), zeroed,
FockDriver.cpp:131-133).  Every call goes through the native library; there is
no CPU path.
"""

import ctypes
import math

import numpy as np

from . import _native as nat
from .matrix import Matrices, Matrix, mat_t
from .screener import T4CScreener


def _comm_rank_size(comm):
    if comm is None:
        return 0, 1
    if isinstance(comm, tuple):
        return int(comm[0]), int(comm[1])
    if hasattr(comm, 'Get_rank'):
        return comm.Get_rank(), comm.Get_size()
    import torch.distributed as dist
    return dist.get_rank(comm), dist.get_world_size(comm)


class _FockDriver:
    """Native Fock driver (reference pybind class ``_FockDriver``)."""

    def __init__(self):
        self._bsf = None
        self.last_stats = None
        self._stage = None  # page-locked host staging buffers (density in, Fock out)

    def _staging(self, n):
        """Page-locked nao x nao host buffers for the copies to and from the
        GPU (allocated once per size through torch; plain host memory where
        torch cannot pin it)."""
        if self._stage is None or self._stage[0].shape != (n, n):
            try:
                import torch
                ti = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
                to = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
                self._stage = (ti.numpy(), to.numpy(), ti, to)
            except (RuntimeError, ImportError):
                self._stage = (np.empty((n, n)), np.empty((n, n)), None, None)
        return self._stage[0], self._stage[1]

    def _set_block_size_factor(self, factor):
        self._bsf = int(factor)

    def _prepare(self, screener):
        if self._bsf is not None:
            screener.set_block_size_factor(self._bsf)

    def _one(self, screener, rank, nodes, density, label, exchange_factor, omega, ithreshold):
        self._prepare(screener)
        dense = nat.f64(density.full_matrix().to_numpy())
        if dense.shape != (screener.nao, screener.nao):
            raise ValueError('FockDriver: density is %s, basis has %d functions' % (dense.shape, screener.nao))
        symmetric = int(density.get_type() == mat_t.symmetric)
        din, out = self._staging(dense.shape[0])
        din[:, :] = dense
        st = nat.Stats()
        nat.check(nat.lib().vlx_b200_fock_build_local(screener.handle, int(rank), int(nodes), nat.dptr(din),
                                                       symmetric, label.encode(), float(exchange_factor),
                                                       float(omega), int(ithreshold), nat.dptr(out),
                                                       ctypes.byref(st)), 'fock_build')
        self.last_stats = st.as_dict()
        fock = density.copy()
        fock.zero()
        fock.set_values(out)
        return fock

    def _many(self, screener, rank, nodes, densities, labels, exchange_factor, omega, ithreshold):
        self._prepare(screener)
        keys = densities.keys()
        if len(keys) != len(labels):
            raise ValueError('FockDriver: number of densities and labels differ')
        dens = [nat.f64(densities.matrix(k).full_matrix().to_numpy()) for k in keys]
        symmetric = int(all(densities.matrix(k).get_type() == mat_t.symmetric for k in keys))
        outs = [np.zeros_like(d) for d in dens]
        dp = (ctypes.POINTER(ctypes.c_double) * len(dens))(*[nat.dptr(d) for d in dens])
        op = (ctypes.POINTER(ctypes.c_double) * len(outs))(*[nat.dptr(o) for o in outs])
        lp = (ctypes.c_char_p * len(labels))(*[l.encode() for l in labels])
        st = nat.Stats()
        nat.check(nat.lib().vlx_b200_fock_build_multi(screener.handle, int(rank), int(nodes), len(dens), dp,
                                                       symmetric, lp, float(exchange_factor), float(omega),
                                                       int(ithreshold), op, ctypes.byref(st)), 'fock_build_multi')
        self.last_stats = st.as_dict()
        result = Matrices()
        for k, o in zip(keys, outs):
            m = densities.matrix(k).copy()
            m.zero()
            m.set_values(o)
            result.add(m, k)
        return result

    def _compute_fock_omp(self, screener, density, label, exchange_factor, omega, ithreshold=None):
        return self._compute_local_fock(screener, 0, 1, density, label, exchange_factor, omega, ithreshold)

    def _compute_local_fock(self, screener, rank, nodes, density, label, exchange_factor, omega, ithreshold=None):
        if ithreshold is None:
            raise NotImplementedError('FockDriver: the (basis, molecule, ...) overload is served by '
                                      'T4CScreener.partition + ithreshold')
        if isinstance(density, Matrices):
            return self._many(screener, rank, nodes, density, label, exchange_factor, omega, ithreshold)
        return self._one(screener, rank, nodes, density, label, exchange_factor, omega, ithreshold)

    def compute_eri(self, screener, nao, ithreshold):
        out = np.zeros((nao, nao, nao, nao))
        nat.check(nat.lib().vlx_b200_compute_eri(screener.handle, int(ithreshold), nat.dptr(out)), 'compute_eri')
        return out


class FockDriver:
    """Fock driver over a communicator (reference src/pymodule/fockdriver.py).

    ``comm`` may be None (single rank), an ``(rank, nodes)`` tuple, an object
    with ``Get_rank()``/``Get_size()`` or a torch.distributed process group.
    """

    def __init__(self, comm=None, ostream=None):
        self.comm = comm
        self.rank, self.nodes = _comm_rank_size(comm)
        self.ostream = ostream
        self._fock_drv = _FockDriver()

    def compute(self, screener, *args):
        return self._fock_drv._compute_local_fock(screener, self.rank, self.nodes, *args)

    def compute_on_subcomm(self, subcomm, screener, *args):
        rank, nodes = _comm_rank_size(subcomm)
        return self._fock_drv._compute_local_fock(screener, rank, nodes, *args)

    def compute_eri(self, molecule, basis, eri_thresh=1.0e-12):
        screener = T4CScreener()
        screener.partition(basis, molecule, 'eri')
        nao = basis.get_dimensions_of_basis()
        return self._fock_drv.compute_eri(screener, nao, int(-math.log10(eri_thresh)))

    def _compute_fock_omp(self, *args):
        return self._fock_drv._compute_fock_omp(*args)

    def _set_block_size_factor(self, factor):
        if factor not in (1, 2, 4, 8, 16, 32, 64, 128):
            raise ValueError('FockDriver._set_block_size_factor: Invalid factor')
        self._fock_drv._set_block_size_factor(factor)

    @property
    def last_stats(self):
        return self._fock_drv.last_stats
