import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / 'tests' / 'golden'


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200); runs through the native library')


def load_golden(name):
    """Golden fixture -> (npz, Molecule, MolecularBasis)."""
    from veloxchem_b200 import MolecularBasis, Molecule
    g = np.load(GOLDEN / name)
    if 'xyz_angstrom' in g:
        mol = Molecule(g['z'], g['xyz_angstrom'], 'angstrom')
    else:
        mol = Molecule(g['z'], g['xyz_bohr'], 'bohr')
    bas = MolecularBasis.read(mol, str(g['basis']))
    return g, mol, bas


@pytest.fixture(scope='session')
def has_gpu():
    from veloxchem_b200 import _native
    return _native.device_count() > 0
