"""CPU-side checks of the product: the C-ABI library loads and exports every
symbol include/vlx_b200.h declares, host-side logic (normalisation, AO layout,
Matrix semantics, input generators) matches the reference conventions.  No
device compute is called here."""

import re

import numpy as np
import pytest

from conftest import ROOT, load_golden


def declared_symbols():
    text = (ROOT / 'include' / 'vlx_b200.h').read_text()
    return sorted(set(re.findall(r'\b(vlx_b200_[a-z0-9_]+)\s*\(', text)))


def test_library_exports_every_declared_symbol():
    from veloxchem_b200 import _native
    lib = _native.lib()
    names = declared_symbols()
    assert len(names) >= 16
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_native.SIGNATURES)
    assert lib.vlx_b200_version().startswith(b'vlx_b200')


def test_errors_are_codes_not_aborts():
    import ctypes
    from veloxchem_b200 import _native
    lib = _native.lib()
    assert lib.vlx_b200_normalize_shell(9, 1, None, None) == 1
    assert b'invalid' in lib.vlx_b200_last_error()
    h = ctypes.c_void_p()
    assert lib.vlx_b200_screener_create(ctypes.byref(h), 0, 0, None, 0, None, None, None, None, None) == 1


def test_normalization_matches_oracle():
    from oracle.oracle import PortOracle, port_available
    if not port_available():
        pytest.skip('oracle not built')
    from veloxchem_b200 import _native
    g, mol, bas = load_golden('h2o_dimer_tzvp.npz')
    ours = np.concatenate([_native.normalize_shell(s.l, s.exps, s.coefs) for s in bas.shells])
    ref = PortOracle(mol, bas).normalized_norms()
    assert np.allclose(ours, ref, rtol=1e-14, atol=0)


@pytest.mark.parametrize('basis,nao', [('sto-3g', 7), ('def2-svp', 24), ('def2-svpd', 39), ('def2-tzvp', 43)])
def test_water_basis_dimensions(basis, nao):
    from veloxchem_b200 import MolecularBasis, Molecule
    mol = Molecule.read_str('O 0 0 0\nH 0 0.76 0.59\nH 0 -0.76 0.59')
    assert MolecularBasis.read(mol, basis).get_dimensions_of_basis() == nao


def test_ao_order_follows_reference_index_map():
    from veloxchem_b200 import MolecularBasis, Molecule
    mol = Molecule.read_str('O 0 0 0\nH 0 0.76 0.59\nH 0 -0.76 0.59')
    bas = MolecularBasis.read(mol, 'def2-svp')
    idx = bas.ao_indices()
    # s block 7 shells, p block 4 shells x 3 (m-major), d block 1 shell x 5
    assert [list(i) for i in idx[:3]] == [[0], [1], [2]]
    p = [i for s, i in zip(bas.shells, idx) if s.l == 1]
    assert list(p[0]) == [7, 11, 15] and list(p[1]) == [8, 12, 16]
    d = [i for s, i in zip(bas.shells, idx) if s.l == 2]
    assert list(d[0]) == [19, 20, 21, 22, 23]
    assert sorted(np.concatenate(idx).tolist()) == list(range(24))


def test_matrix_symmetric_semantics():
    from veloxchem_b200 import MolecularBasis, Molecule, SubMatrix, make_matrix, mat_t
    mol = Molecule.read_str('O 0 0 0\nH 0 0.76 0.59\nH 0 -0.76 0.59')
    bas = MolecularBasis.read(mol, 'def2-svp')
    rng = np.random.default_rng(3)
    a = rng.standard_normal((24, 24))
    a = a + a.T
    m = make_matrix(bas, mat_t.symmetric)
    assert m.angular_pairs() == [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    m.set_values(a)
    assert np.array_equal(m.full_matrix().to_numpy(), a)
    assert m.submatrix((0, 1)) == SubMatrix([0, 7, 7, 12], a[0:7, 7:19])
    g = make_matrix(bas, mat_t.general)
    assert len(g.angular_pairs()) == 9


def test_water_cluster_generator_is_seeded():
    from veloxchem_b200.geometry import random_density, water_cluster
    a = water_cluster((4, 4, 2), 1).get_coordinates_in_bohr()
    b = water_cluster((4, 4, 2), 1).get_coordinates_in_bohr()
    assert a.shape == (96, 3) and np.array_equal(a, b)
    # rigid waters: O-H 0.9572 A
    oh = np.linalg.norm(a[1] - a[0]) * 0.529177210903
    assert abs(oh - 0.9572) < 1e-12
    d = random_density(30, 5, 7)
    assert np.allclose(d, d.T) and abs(np.trace(d) - 5) < 1e-12 and np.allclose(d @ d, d)
