"""Molecule: element identifiers and Cartesian coordinates (bohr internally).

Mirrors the parts of the reference ``Molecule`` the Fock build uses:
``Molecule.read_str`` (src/pymodule/molecule.py), ``CMolecule`` storing
coordinates in bohr after an angstrom -> bohr conversion with the CODATA-2018
Bohr radius (src/moldata/Molecule.cpp:60-73, src/general/Codata.cpp:33-37).
"""

import numpy as np

BOHR_IN_ANGSTROM = 0.529177210903

_ELEMENTS = ['BQ', 'H', 'HE', 'LI', 'BE', 'B', 'C', 'N', 'O', 'F', 'NE']


def element_id(label):
    return _ELEMENTS.index(label.upper())


def element_label(z):
    lab = _ELEMENTS[z]
    return lab[0] + lab[1:].lower()


class Molecule:
    """A set of atoms (nuclear charge + position in bohr)."""

    def __init__(self, elem_ids, coords, units='angstrom'):
        self._ids = np.asarray(elem_ids, dtype=np.int32).copy()
        xyz = np.asarray(coords, dtype=np.float64).reshape(-1, 3).copy()
        if units.lower() in ('angstrom', 'angs', 'a'):
            xyz /= BOHR_IN_ANGSTROM
        elif units.lower() not in ('bohr', 'au', 'a.u.'):
            raise ValueError('Molecule: unknown unit ' + units)
        self._xyz = xyz
        self._charge = 0.0

    @staticmethod
    def read_str(text, units='angstrom'):
        ids, xyz = [], []
        for line in text.strip().splitlines():
            parts = line.split()
            if not parts:
                continue
            ids.append(element_id(parts[0]))
            xyz.append([float(v) for v in parts[1:4]])
        return Molecule(ids, xyz, units)

    def number_of_atoms(self):
        return len(self._ids)

    def get_element_ids(self):
        return self._ids.copy()

    def get_labels(self):
        return [element_label(z) for z in self._ids]

    def get_coordinates_in_bohr(self):
        return self._xyz.copy()

    def get_charge(self):
        return self._charge

    def set_charge(self, charge):
        self._charge = float(charge)

    def number_of_electrons(self):
        return int(round(float(self._ids.sum()) - self._charge))

    def nuclear_repulsion_energy(self):
        z = self._ids.astype(np.float64)
        e = 0.0
        for i in range(len(z)):
            d = np.linalg.norm(self._xyz[i + 1:] - self._xyz[i], axis=1)
            e += float(np.sum(z[i] * z[i + 1:] / d))
        return e
