"""Host logic of the learned guess: the AO rotation of the reference's real
solid harmonics (checked on the compiled reference's overlap matrix of a
rotated molecule), invariance of the pair descriptors and local-frame
blocks under rigid motions, and the block cut / assemble round trip."""

import numpy as np
import pytest

from oracle.oracle import RefOracle, ref_available


def _cluster(n=3, seed=4):
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200.geometry import water_cluster
    mol = water_cluster((3, 3, 2), seed, n)
    return mol, MolecularBasis.read(mol, 'def2-svp')


def _moved(mol, Q, t):
    from veloxchem_b200 import Molecule
    from veloxchem_b200.guess import BOHR_IN_ANGSTROM
    xyz = mol.get_coordinates_in_bohr() * BOHR_IN_ANGSTROM
    return Molecule(mol.get_element_ids(), xyz @ Q.T + t, 'angstrom')


def _full_rotation(lay, Q):
    from veloxchem_b200.guess import atom_rotation
    R = np.zeros((lay.nao, lay.nao))
    for a in range(len(lay.z)):
        R[np.ix_(lay.atom_aos[a], lay.atom_aos[a])] = atom_rotation(lay.atom_ls[a], Q)
    return R


Q0 = np.linalg.qr(np.random.default_rng(8).standard_normal((3, 3)))[0]
Q0 = Q0 * np.sign(np.linalg.det(Q0))


def test_sh_rotation_is_orthogonal_representation():
    from veloxchem_b200.guess import sh_rotation
    Q1 = np.linalg.qr(np.random.default_rng(1).standard_normal((3, 3)))[0]
    Q1 *= np.sign(np.linalg.det(Q1))
    for l in (0, 1, 2):
        D = sh_rotation(l, Q0)
        assert np.allclose(D @ D.T, np.eye(2 * l + 1), atol=1e-12)
        assert np.allclose(sh_rotation(l, Q0 @ Q1), sh_rotation(l, Q0) @ sh_rotation(l, Q1), atol=1e-12)


@pytest.mark.skipif(not ref_available(), reason='reference oracle not built')
def test_overlap_of_rotated_molecule_transforms_by_ao_rotation():
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200.guess import ClusterLayout
    mol, bas = _cluster(2)
    mol2 = _moved(mol, Q0, np.array([0.3, -1.2, 2.0]))
    bas2 = MolecularBasis.read(mol2, 'def2-svp')
    S = RefOracle(mol, bas, partition=False).one_electron(0)
    S2 = RefOracle(mol2, bas2, partition=False).one_electron(0)
    R = _full_rotation(ClusterLayout(mol, bas), Q0)
    assert np.max(np.abs(S2 - R @ S @ R.T)) < 1e-12


def test_descriptors_and_blocks_invariant_under_rigid_motion():
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200.guess import ClusterLayout
    mol, bas = _cluster(4)
    mol2 = _moved(mol, Q0, np.array([1.0, 2.0, -0.5]))
    bas2 = MolecularBasis.read(mol2, 'def2-svp')
    a, b = ClusterLayout(mol, bas), ClusterLayout(mol2, bas2)
    assert np.array_equal(a.pairs, b.pairs)
    assert np.max(np.abs(a.descriptors() - b.descriptors())) < 1e-5
    rng = np.random.default_rng(2)
    c = rng.standard_normal((a.nao, 20))
    D = c @ c.T
    D2 = _full_rotation(a, Q0) @ D @ _full_rotation(a, Q0).T
    Ta, Ma = a.local_blocks(D)
    Tb, Mb = b.local_blocks(D2)
    assert np.array_equal(Ma, Mb)
    assert np.max(np.abs(Ta - Tb)) < 1e-5 * np.max(np.abs(Ta))


def test_blocks_round_trip():
    from veloxchem_b200.guess import ClusterLayout
    mol, bas = _cluster(2)
    lay = ClusterLayout(mol, bas)
    assert np.all(lay.dist[lay.pairs[:, 0], lay.pairs[:, 1]] <= 5.0)
    rng = np.random.default_rng(5)
    c = rng.standard_normal((lay.nao, 10))
    D = c @ c.T
    T, M = lay.local_blocks(D)
    back = lay.assemble(T.astype(np.float64))
    covered = np.zeros_like(D, dtype=bool)
    for i, j in lay.pairs:
        covered[np.ix_(lay.atom_aos[i], lay.atom_aos[j])] = True
        covered[np.ix_(lay.atom_aos[j], lay.atom_aos[i])] = True
    assert np.max(np.abs((back - D)[covered])) < 1e-5 * np.max(np.abs(D))
    assert np.all(back[~covered] == 0.0)


def _loop_descriptors(lay):
    """Per-pair loop form of the descriptors (the form the shipped network was
    trained with), to pin the vectorised implementation."""
    import math
    from veloxchem_b200.guess import ENV_CUTOFF, MOM_CENTERS, MOM_WIDTH, NFEAT, NTYPES, RBF_CENTERS, RBF_WIDTH

    def env(i):
        d = lay.dist[i]
        mask = (d > 1e-8) & (d < ENV_CUTOFF)
        out = []
        for el in (8, 1):
            sel = mask & (lay.z == el)
            out.append(np.exp(-((d[sel][:, None] - RBF_CENTERS[None, :]) / RBF_WIDTH) ** 2).sum(axis=0))
        v = (lay.xyz[mask] - lay.xyz[i]) / d[mask][:, None]
        v = v @ lay.frames[lay.water[i]]
        g = np.exp(-((d[mask][:, None] - MOM_CENTERS[None, :]) / MOM_WIDTH) ** 2)
        out.append((g[:, :, None] * v[:, None, :]).sum(axis=0).ravel())
        q = (g[:, :, None, None] * v[:, None, :, None] * v[:, None, None, :]).sum(axis=0)
        out.append(np.stack([q[:, 0, 0], q[:, 1, 1], q[:, 2, 2], q[:, 0, 1], q[:, 0, 2], q[:, 1, 2]], axis=1).ravel())
        return np.concatenate(out)

    e = [env(i) for i in range(len(lay.z))]
    X = np.zeros((len(lay.pairs), NFEAT))
    for p, (i, j) in enumerate(lay.pairs):
        zi, zj = lay.z[i], lay.z[j]
        t = (0 if zi == 8 else 1) if i == j else (2 if (zi == 8 and zj == 8) else (3 if zi == 8 else 4))
        wa, wb = lay.water[i], lay.water[j]
        Fa, Fb = lay.frames[wa], lay.frames[wb]
        dv = lay.xyz[j] - lay.xyz[i]
        d = lay.dist[i, j]
        f = [np.eye(NTYPES)[t], [1.0 if wa == wb else 0.0], [d, math.exp(-d), 1.0 / (1.0 + d)], dv @ Fa, dv @ Fb,
             (Fa.T @ Fb).ravel(), (lay.xyz[i] - lay.origin[wa]) @ Fa, (lay.xyz[j] - lay.origin[wb]) @ Fb, e[i], e[j]]
        X[p] = np.concatenate([np.asarray(v, dtype=np.float64).ravel() for v in f])
    return X


def test_vectorised_layout_matches_pair_loop():
    from veloxchem_b200.guess import ClusterLayout, atom_rotation
    mol, bas = _cluster(6, seed=9)
    lay = ClusterLayout(mol, bas)
    assert np.max(np.abs(lay.descriptors() - _loop_descriptors(lay))) < 1e-5
    for a in range(len(lay.z)):
        assert np.allclose(lay.rot[a], atom_rotation(lay.atom_ls[a], lay.frames[lay.water[a]].T), atol=1e-12)
    rng = np.random.default_rng(1)
    c = rng.standard_normal((lay.nao, 12))
    D = c @ c.T
    T, M = lay.local_blocks(D)
    for p, (i, j) in enumerate(lay.pairs):
        blk = lay.rot[i] @ D[np.ix_(lay.atom_aos[i], lay.atom_aos[j])] @ lay.rot[j].T
        assert np.allclose(T[p, :blk.size], blk.ravel(), atol=1e-5 * np.max(np.abs(D)))
        assert M[p, :blk.size].all() and not M[p, blk.size:].any()


def test_sad_atom_ao_indices_follow_the_reference_order():
    """Per-atom AO indices of the SAD guess: the reference order (angular
    momentum, component, atom, shell), checked against a direct enumeration."""
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200.geometry import water_cluster
    from veloxchem_b200.scf import SadGuessDriver
    mol = water_cluster((2, 1, 1), 5)
    for name in ('def2-tzvp', 'ao-start-guess'):
        bas = MolecularBasis.read(mol, name)
        expect = [[] for _ in range(mol.number_of_atoms())]
        ao = 0
        for l in range(bas.max_angular_momentum() + 1):
            for _m in range(2 * l + 1):
                for a in range(mol.number_of_atoms()):
                    for s in bas.shells:
                        if s.atom == a and s.l == l:
                            expect[a].append(ao)
                            ao += 1
        assert SadGuessDriver.ao_indices_of_atoms(mol, bas) == expect
        assert ao == bas.get_dimensions_of_basis()

