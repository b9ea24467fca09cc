"""veloxchem_b200: B200-native four-centre Fock build with the reference's API.

Public names follow the reference (VeloxChem): ``Molecule``,
``MolecularBasis``, ``Matrix`` / ``SubMatrix`` / ``Matrices`` /
``make_matrix`` / ``mat_t``, ``T4CScreener``, ``FockDriver``.
"""

from .fockdriver import FockDriver, _FockDriver
from .matrix import Matrices, Matrix, SubMatrix, make_matrix, mat_t
from .molecularbasis import MolecularBasis
from .molecule import Molecule
from .screener import T4CScreener

__all__ = ['FockDriver', '_FockDriver', 'Matrices', 'Matrix', 'SubMatrix', 'make_matrix', 'mat_t',
           'MolecularBasis', 'Molecule', 'T4CScreener']
