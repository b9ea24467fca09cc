"""TEST INFRASTRUCTURE ONLY: ctypes access to the two CPU oracles.

* ``RefOracle``  — the reference's own Fock build compiled from source
  (oracle/_ref/libvlxref.so, built by oracle/Makefile from the reference tree).
* ``PortOracle`` — the plain-C restatement in oracle/eri_oracle.c
  (oracle/_ref/liberioracle.so).

Both take a ``Molecule`` and ``MolecularBasis`` of the product package (only to
read coordinates and the raw shell table) and return dense NumPy matrices in
the reference AO order.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / reference arm may import this module.
"""

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_REF_LIB = _HERE / '_ref' / 'libvlxref.so'
_PORT_LIB = _HERE / '_ref' / 'liberioracle.so'

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _system_arrays(molecule, basis):
    z = np.ascontiguousarray(molecule.get_element_ids(), dtype=np.int32)
    xyz = np.ascontiguousarray(molecule.get_coordinates_in_bohr(), dtype=np.float64)
    atom, lval, nprim, exps, coefs = basis.shell_table()
    return (z, xyz, np.ascontiguousarray(atom), np.ascontiguousarray(lval), np.ascontiguousarray(nprim),
            np.ascontiguousarray(exps), np.ascontiguousarray(coefs))


def ref_available():
    return _REF_LIB.exists()


def port_available():
    return _PORT_LIB.exists()


class RefOracle:
    """The reference FockDriver (CFockDriver::compute et al.) on the host CPU."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not _REF_LIB.exists():
                raise RuntimeError('reference oracle not built: ' + str(_REF_LIB))
            lib = ctypes.CDLL(str(_REF_LIB))
            lib.vlxref_create.restype = ctypes.c_void_p
            lib.vlxref_create.argtypes = [ctypes.c_int, _ip, _dp, ctypes.c_int, _ip, _ip, _ip, _dp, _dp]
            lib.vlxref_destroy.argtypes = [ctypes.c_void_p]
            lib.vlxref_nao.argtypes = [ctypes.c_void_p]
            lib.vlxref_partition.argtypes = [ctypes.c_void_p]
            lib.vlxref_set_threads.argtypes = [ctypes.c_int]
            lib.vlxref_set_block_size_factor.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.vlxref_screened_pairs.argtypes = [ctypes.c_void_p, _ip]
            lib.vlxref_pair_bins.argtypes = [ctypes.c_void_p, _ip]
            lib.vlxref_fock.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_char_p, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
            lib.vlxref_fock_multi.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_char_p), ctypes.c_double, ctypes.c_double,
                                              ctypes.c_int, _dp]
            lib.vlxref_eri.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
            lib.vlxref_one_electron.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
            lib.vlxref_overlap_mixed.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _dp]
            cls._lib = lib
        return cls._lib

    def __init__(self, molecule, basis, partition=True):
        lib = self.lib()
        arrs = _system_arrays(molecule, basis)
        self._arrs = arrs
        z, xyz, atom, lval, nprim, exps, coefs = arrs
        self._h = lib.vlxref_create(len(z), _i(z), _d(xyz), len(atom), _i(atom), _i(lval), _i(nprim), _d(exps),
                                    _d(coefs))
        self.nao = lib.vlxref_nao(self._h)
        if partition:
            self.partition()

    def __del__(self):
        if getattr(self, '_h', None):
            self.lib().vlxref_destroy(self._h)
            self._h = None

    @staticmethod
    def set_threads(n):
        RefOracle.lib().vlxref_set_threads(int(n))

    def set_block_size_factor(self, f):
        self.lib().vlxref_set_block_size_factor(self._h, int(f))

    def partition(self):
        self.lib().vlxref_partition(self._h)

    def pair_bins(self):
        n = ctypes.c_int(0)
        self.lib().vlxref_screened_pairs(self._h, ctypes.byref(n))
        out = np.zeros((n.value, 6), dtype=np.int32)
        self.lib().vlxref_pair_bins(self._h, _i(out))
        return out

    def fock(self, density, label='2jk', exchange_factor=1.0, omega=0.0, ithreshold=15, symmetric=True,
             rank=0, nodes=1):
        d = np.ascontiguousarray(density, dtype=np.float64)
        out = np.zeros((self.nao, self.nao))
        self.lib().vlxref_fock(self._h, _d(d), int(symmetric), label.encode(), float(exchange_factor),
                               float(omega), int(ithreshold), int(rank), int(nodes), _d(out))
        return out

    def fock_multi(self, densities, labels, exchange_factor=0.0, omega=0.0, ithreshold=15, symmetric=True):
        d = np.ascontiguousarray(np.stack(densities), dtype=np.float64)
        out = np.zeros_like(d)
        labs = (ctypes.c_char_p * len(labels))(*[l.encode() for l in labels])
        self.lib().vlxref_fock_multi(self._h, len(labels), _d(d), int(symmetric), labs, float(exchange_factor),
                                     float(omega), int(ithreshold), _d(out))
        return [out[i] for i in range(len(labels))]

    def eri(self, ithreshold=12):
        out = np.zeros((self.nao,) * 4)
        self.lib().vlxref_eri(self._h, int(ithreshold), _d(out))
        return out

    def one_electron(self, which):
        """0 = overlap S, 1 = kinetic T, 2 = nuclear attraction V (negative)."""
        out = np.zeros((self.nao, self.nao))
        self.lib().vlxref_one_electron(self._h, int(which), _d(out))
        return out

    def overlap_mixed(self, other):
        """Overlap between this system's basis (rows) and other's basis (columns)."""
        out = np.zeros((self.nao, other.nao))
        self.lib().vlxref_overlap_mixed(self._h, other._h, _d(out))
        return out


class PortOracle:
    """The C restatement of the reference algorithm (oracle/eri_oracle.c)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not _PORT_LIB.exists():
                raise RuntimeError('restatement oracle not built: ' + str(_PORT_LIB))
            lib = ctypes.CDLL(str(_PORT_LIB))
            lib.eo_create.restype = ctypes.c_void_p
            lib.eo_create.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, _ip, _dp, _dp]
            lib.eo_destroy.argtypes = [ctypes.c_void_p]
            lib.eo_nao.argtypes = [ctypes.c_void_p]
            lib.eo_npairs.argtypes = [ctypes.c_void_p]
            lib.eo_pair_info.argtypes = [ctypes.c_void_p, _ip, _dp]
            lib.eo_normalized_norms.argtypes = [ctypes.c_void_p, _dp]
            lib.eo_shell_quartet.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, _dp]
            lib.eo_fock.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_char_p, ctypes.c_double,
                                    ctypes.c_int, _dp]
            lib.eo_eri.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
            lib.eo_boys.restype = ctypes.c_double
            lib.eo_boys.argtypes = [ctypes.c_int, ctypes.c_double]
            lib.eo_sph_factor.restype = ctypes.c_double
            lib.eo_sph_factor.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
            lib.eo_normalize.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
            cls._lib = lib
        return cls._lib

    def __init__(self, molecule, basis):
        lib = self.lib()
        arrs = _system_arrays(molecule, basis)
        self._arrs = arrs
        z, xyz, atom, lval, nprim, exps, coefs = arrs
        self._nprim = nprim
        self._h = lib.eo_create(len(z), _d(xyz), len(atom), _i(atom), _i(lval), _i(nprim), _d(exps), _d(coefs))
        self.nao = lib.eo_nao(self._h)

    def __del__(self):
        if getattr(self, '_h', None):
            self.lib().eo_destroy(self._h)
            self._h = None

    def pair_info(self):
        n = self.lib().eo_npairs(self._h)
        info = np.zeros((n, 6), dtype=np.int32)
        maxv = np.zeros(n)
        self.lib().eo_pair_info(self._h, _i(info), _d(maxv))
        return info, maxv

    def normalized_norms(self):
        out = np.zeros(int(self._nprim.sum()))
        self.lib().eo_normalized_norms(self._h, _d(out))
        return out

    def shell_quartet(self, p, q, r, s, dims):
        out = np.zeros(int(np.prod(dims)))
        self.lib().eo_shell_quartet(self._h, p, q, r, s, _d(out))
        return out.reshape(dims)

    def fock(self, density, label='2jk', exchange_factor=1.0, ithreshold=15, symmetric=True):
        d = np.ascontiguousarray(density, dtype=np.float64)
        out = np.zeros((self.nao, self.nao))
        self.lib().eo_fock(self._h, _d(d), int(symmetric), label.encode(), float(exchange_factor),
                           int(ithreshold), _d(out))
        return out

    def eri(self, ithreshold=12):
        out = np.zeros((self.nao,) * 4)
        self.lib().eo_eri(self._h, int(ithreshold), _d(out))
        return out

    @staticmethod
    def boys(m, t):
        return PortOracle.lib().eo_boys(int(m), float(t))

    @staticmethod
    def sph_factor(l, m, cart):
        return PortOracle.lib().eo_sph_factor(int(l), int(m), int(cart))

    @staticmethod
    def set_threads(n):
        os.environ['OMP_NUM_THREADS'] = str(int(n))
