"""Molecular basis: contracted shells per atom, in the reference's order.

Mirrors ``MolecularBasis.read`` (src/pymodule/molecularbasis.py:112-169): one
atom basis per atom taken from the named basis set, shells kept in file order.
The AO order the Fock build uses is the reference's
(``CMolecularBasis::index_map``, src/orbdata/MolecularBasis.cpp:468-490):
all functions of angular momentum l come after those of l-1; inside l the
index is ``offset_l + m * N_l + s`` with s the running index of l-shells over
atoms in order and m = 0..2l (real solid harmonics m = -l..l).

Contraction coefficients are kept raw here; the native library normalises
them exactly as ``CBasisFunction::normalize`` does.
"""

import json
from pathlib import Path

import numpy as np

_DATA = Path(__file__).parent / 'basis_data'
_ALIASES = {'DEF2-SVP': 'def2-svp', 'DEF2-SVPD': 'def2-svpd', 'DEF2-TZVP': 'def2-tzvp',
            'STO-3G': 'sto-3g', 'AO-START-GUESS': 'ao-start-guess'}
_LABELS = ['BQ', 'H', 'HE', 'LI', 'BE', 'B', 'C', 'N', 'O', 'F', 'NE']


class Shell:
    __slots__ = ('atom', 'l', 'exps', 'coefs')

    def __init__(self, atom, l, exps, coefs):
        self.atom = atom
        self.l = l
        self.exps = np.asarray(exps, dtype=np.float64)
        self.coefs = np.asarray(coefs, dtype=np.float64)

    @property
    def nprim(self):
        return len(self.exps)


class MolecularBasis:
    """Contracted shells of a molecule (spherical functions only)."""

    def __init__(self, shells, name='', natoms=0):
        self.shells = list(shells)
        self.name = name
        self._natoms = natoms

    @staticmethod
    def read(molecule, basis_name, ostream=None):
        key = basis_name.upper()
        if key not in _ALIASES:
            raise ValueError('MolecularBasis.read: basis set not shipped: ' + basis_name)
        data = json.loads((_DATA / (_ALIASES[key] + '.json')).read_text())
        shells = []
        for a, z in enumerate(molecule.get_element_ids()):
            lab = _LABELS[z]
            if lab not in data:
                raise ValueError('MolecularBasis.read: no %s data for %s' % (basis_name, lab))
            for lval, exps, coefs in data[lab]:
                shells.append(Shell(a, lval, exps, coefs))
        return MolecularBasis(shells, key, molecule.number_of_atoms())

    def get_label(self):
        return self.name

    def max_angular_momentum(self):
        return max(s.l for s in self.shells) if self.shells else -1

    def number_of_basis_functions(self, l):
        return sum(1 for s in self.shells if s.l == l)

    def get_dimensions_of_basis(self, upto=None):
        lmax = self.max_angular_momentum() if upto is None else upto - 1
        return sum(self.number_of_basis_functions(l) * (2 * l + 1) for l in range(lmax + 1))

    def dimensions_of_basis(self, upto=None):
        return self.get_dimensions_of_basis(upto)

    def angular_offsets(self):
        """AO offset of the first function of each angular momentum."""
        offs, off = [], 0
        for l in range(self.max_angular_momentum() + 1):
            offs.append(off)
            off += self.number_of_basis_functions(l) * (2 * l + 1)
        return offs

    def shell_table(self):
        """Flat arrays handed to the native library (reference shell order)."""
        atom = np.array([s.atom for s in self.shells], dtype=np.int32)
        lval = np.array([s.l for s in self.shells], dtype=np.int32)
        nprim = np.array([s.nprim for s in self.shells], dtype=np.int32)
        exps = np.concatenate([s.exps for s in self.shells]).astype(np.float64)
        coefs = np.concatenate([s.coefs for s in self.shells]).astype(np.float64)
        return atom, lval, nprim, exps, coefs

    def ao_indices(self):
        """AO index of component m of every shell: list of int arrays."""
        offs = self.angular_offsets()
        counters = [0] * (self.max_angular_momentum() + 1)
        out = []
        for s in self.shells:
            n_l = self.number_of_basis_functions(s.l)
            base = offs[s.l] + counters[s.l]
            counters[s.l] += 1
            out.append(np.array([base + m * n_l for m in range(2 * s.l + 1)], dtype=np.int64))
        return out
