"""T4CScreener: shell-pair data and Schwarz screening on the GPU.

Mirrors the reference ``T4CScreener`` (src/t4c_func/T4CScreener.cpp,
exported in src/python/ExportT4CIntegrals.cpp:127-140): ``partition(basis,
molecule, 'eri')`` evaluates max (ab|ab) per shell pair and bins the pairs
into 16 decades; ``gto_pair_blocks()`` exposes the result; the object
pickles (by its inputs, the device state is rebuilt on unpickling) and
compares by value.
"""

import ctypes

import numpy as np

from . import _native as nat


class PairBlockInfo:
    """Screening result of one pair block: angular momenta and per-pair bins."""

    def __init__(self, index, la, lb, bins, maxv, bra_ao, ket_ao):
        self.index = index
        self.angular_momentums = (la, lb)
        self.bins = bins
        self.max_values = maxv
        self.bra_orbital_indices = bra_ao
        self.ket_orbital_indices = ket_ao

    def number_of_contracted_pairs(self):
        return len(self.bins)

    def is_empty_gto_pair_block(self, b):
        return not np.any(self.bins == b)

    def __eq__(self, other):
        return (self.angular_momentums == other.angular_momentums and np.array_equal(self.bins, other.bins)
                and np.array_equal(self.bra_orbital_indices, other.bra_orbital_indices)
                and np.array_equal(self.ket_orbital_indices, other.ket_orbital_indices))


class T4CScreener:
    """GPU Schwarz screener; owns the device shell-pair data of one molecule."""

    def __init__(self, device=0):
        self._h = None
        self._device = int(device)
        self._inputs = None
        self._blocks = None
        self.nao = 0

    # -- reference API --------------------------------------------------------
    def partition(self, basis, molecule, label='eri'):
        if label != 'eri':
            raise ValueError('T4CScreener.partition: only the "eri" label is supported')
        xyz = nat.f64(molecule.get_coordinates_in_bohr())
        atom, lval, nprim, exps, coefs = basis.shell_table()
        self._inputs = (xyz, nat.i32(atom), nat.i32(lval), nat.i32(nprim), nat.f64(exps), nat.f64(coefs))
        self._create()

    def gto_pair_blocks(self):
        if self._blocks is None:
            info, maxv = self.pair_info()
            blocks = []
            for b in np.unique(info[:, 0]):
                sel = info[:, 0] == b
                blocks.append(PairBlockInfo(int(b), int(info[sel][0, 2]), int(info[sel][0, 3]), info[sel, 1].copy(),
                                            maxv[sel].copy(), info[sel, 4].copy(), info[sel, 5].copy()))
            self._blocks = blocks
        return self._blocks

    # -- helpers --------------------------------------------------------------
    def _create(self):
        self._release()
        xyz, atom, lval, nprim, exps, coefs = self._inputs
        h = ctypes.c_void_p()
        nat.check(nat.lib().vlx_b200_screener_create(ctypes.byref(h), self._device, len(xyz), nat.dptr(xyz),
                                                      len(atom), nat.iptr(atom), nat.iptr(lval), nat.iptr(nprim),
                                                      nat.dptr(exps), nat.dptr(coefs)), 'screener_create')
        self._h = h
        n = ctypes.c_int(0)
        nat.check(nat.lib().vlx_b200_screener_nao(self._h, ctypes.byref(n)), 'screener_nao')
        self.nao = n.value
        self._blocks = None

    def _release(self):
        if self._h is not None:
            nat.lib().vlx_b200_screener_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError('T4CScreener: partition() has not been called')
        return self._h

    def pair_info(self):
        n = ctypes.c_int(0)
        nat.check(nat.lib().vlx_b200_screener_npairs(self.handle, ctypes.byref(n)), 'screener_npairs')
        info = np.zeros((n.value, 6), dtype=np.int32)
        maxv = np.zeros(n.value)
        nat.check(nat.lib().vlx_b200_screener_pair_info(self.handle, nat.iptr(info), nat.dptr(maxv)), 'pair_info')
        return info, maxv

    def set_fp32_threshold(self, cutoff, max_abs_density):
        """Mixed precision: quartets with Schwarz bound x max|D| below cutoff in
        FP32 for the following builds (cutoff <= 0: FP64 only)."""
        nat.check(nat.lib().vlx_b200_set_fp32_threshold(self.handle, float(cutoff), float(max_abs_density)),
                  'set_fp32_threshold')

    def set_density_screening(self, fp32_cutoff=0.0, skip_cutoff=0.0):
        """Per-quartet screening of the following builds on the bound
        sqrt((PQ|PQ)(RS|RS)) x (local shell-block maxima of |D|): quartets
        below skip_cutoff are skipped, those below fp32_cutoff evaluated in
        FP32 (0 switches a part off; both 0: the reference's screening)."""
        nat.check(nat.lib().vlx_b200_set_density_screening(self.handle, float(fp32_cutoff), float(skip_cutoff)),
                  'set_density_screening')

    def set_fp32_digestion(self, on):
        """FP32 digestion of the FP32 quartets of density-screened builds
        (for builds whose result is replaced later: see the C header)."""
        nat.check(nat.lib().vlx_b200_set_fp32_digestion(self.handle, int(bool(on))), 'set_fp32_digestion')

    def set_work_threshold(self, ithreshold_base):
        """Build work lists for max(ithreshold, ithreshold_base) and filter at
        run time, so builds at several thresholds share one list."""
        nat.check(nat.lib().vlx_b200_set_work_threshold(self.handle, int(ithreshold_base)), 'set_work_threshold')

    def set_partition(self, partition):
        """Work-item partition of the rank/nodes builds: 'round_robin' (the
        reference's deal) or 'balanced' (greedy by estimated cost)."""
        from .distributed import PARTITIONS
        if partition not in PARTITIONS:
            raise ValueError('T4CScreener.set_partition: unknown partition %r' % (partition,))
        nat.check(nat.lib().vlx_b200_set_partition(self.handle, PARTITIONS[partition]), 'set_partition')

    def set_block_size_factor(self, factor):
        nat.check(nat.lib().vlx_b200_set_block_size_factor(self.handle, int(factor)), 'set_block_size_factor')

    def __getstate__(self):
        return {'device': self._device, 'inputs': self._inputs}

    def __setstate__(self, state):
        self._h = None
        self._blocks = None
        self._device = state['device']
        self._inputs = state['inputs']
        self.nao = 0
        if self._inputs is not None:
            self._create()

    def __eq__(self, other):
        a, b = self.gto_pair_blocks(), other.gto_pair_blocks()
        return len(a) == len(b) and all(x == y for x, y in zip(a, b))

    def __ne__(self, other):
        return not self.__eq__(other)
