"""One-electron integrals and the restricted HF SCF.

Pins: the reference's own overlap / kinetic / nuclear-attraction drivers
(compiled into oracle/_ref) and the reference's SCF energy known answer for the
water dimer / def2-SVP, -151.9220860932 Eh to 1e-8 (tests/test_scf_rest.py of
the reference, geometry from the same test)."""

import numpy as np
import pytest

from oracle.oracle import ref_available

REF_ENERGY = -151.9220860932

DIMER_XYZ = """
O   -0.1858140  -1.1749469   0.7662596
H   -0.1285513  -0.8984365   1.6808606
H   -0.0582782  -0.3702550   0.2638279
O    0.1747051  11.1050002  -0.7244430
H   -0.5650842  11.3134964  -1.2949455
H    0.9282185  11.0652990  -1.3134026
"""


def _dimer(basis='def2-svp'):
    from veloxchem_b200 import MolecularBasis, Molecule
    mol = Molecule.read_str(DIMER_XYZ)
    return mol, MolecularBasis.read(mol, basis)


def _oracle_scf(mol, bas, conv=1e-7, max_iter=80):
    """A plain numpy restricted HF over the compiled reference (its S, T, V
    drivers and FockDriver at ithreshold 12), Pulay DIIS, core guess; returns
    the energy once the electronic gradient 2 ||X^T (FDS - SDF) X|| < conv."""
    from oracle.oracle import RefOracle
    ref = RefOracle(mol, bas)
    S, T, V = ref.one_electron(0), ref.one_electron(1), ref.one_electron(2)
    H = T + V
    w, u = np.linalg.eigh(S)
    X = u[:, w > 1e-6] / np.sqrt(w[w > 1e-6])
    nocc = mol.number_of_electrons() // 2
    e, c = np.linalg.eigh(X.T @ H @ X)
    D = X @ c[:, :nocc] @ (X @ c[:, :nocc]).T
    focks, errs, energy = [], [], 0.0
    for _ in range(max_iter):
        F2 = ref.fock(D, '2jk', 1.0, 0.0, 12)
        energy = np.sum(D * F2) + 2 * np.sum(D * H) + mol.nuclear_repulsion_energy()
        F = F2 + H
        err = X.T @ (F @ D @ S - S @ D @ F) @ X
        if 2 * np.linalg.norm(err) < conv:
            return energy
        focks.append(F)
        errs.append(err)
        if len(focks) > 10:
            focks.pop(0)
            errs.pop(0)
        n = len(focks)
        B = -np.ones((n + 1, n + 1))
        B[n, n] = 0
        for i in range(n):
            for j in range(n):
                B[i, j] = np.sum(errs[i] * errs[j])
        rhs = np.zeros(n + 1)
        rhs[n] = -1
        coef = np.linalg.lstsq(B, rhs, rcond=None)[0]
        Fe = sum(cf * f for cf, f in zip(coef[:n], focks))
        e, c = np.linalg.eigh(X.T @ Fe @ X)
        D = X @ c[:, :nocc] @ (X @ c[:, :nocc]).T
    raise AssertionError('oracle SCF did not converge')


@pytest.mark.skipif(not ref_available(), reason='reference oracle not built')
def test_cpu_scf_restatement_reaches_reference_energy():
    """The numpy SCF over the compiled reference pins the energy expression
    and the orthogonalisation used by the driver."""
    mol, bas = _dimer()
    assert abs(_oracle_scf(mol, bas) - REF_ENERGY) < 1e-8


@pytest.mark.gpu
@pytest.mark.skipif(not ref_available(), reason='reference oracle not built')
@pytest.mark.parametrize('guess,incremental,fp32', [('sad', False, 0.0), ('learned', True, 1e-6)])
def test_scf_energy_against_oracle_driven_scf(guess, incremental, fp32):
    """The converged RHF energy of a water cluster ((H2O)_4 / def2-SVP, 96
    functions) against the SCF driven by the reference's own integrals and
    FockDriver, both to an electronic gradient of 1e-8: within 1e-9 Eh, for
    the plain driver and for learned guess + incremental + mixed builds."""
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200.geometry import water_cluster
    from veloxchem_b200.scf import ScfRestrictedDriver
    mol = water_cluster((2, 2, 1), 1)
    bas = MolecularBasis.read(mol, 'def2-svp')
    e_ref = _oracle_scf(mol, bas, conv=1e-8)
    drv = ScfRestrictedDriver()
    drv.conv_thresh = 1e-8
    drv.guess = guess
    drv.incremental = incremental
    drv.fp32_cutoff = fp32
    res = drv.compute(mol, bas)
    assert res['converged']
    assert abs(res['scf_energy'] - e_ref) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize('basis', ['def2-svpd', 'def2-tzvp'])
def test_one_electron_against_reference(basis):
    from conftest import load_golden
    from oracle.oracle import RefOracle
    from veloxchem_b200 import _native as nat
    name = 'h2o_dimer_svpd.npz' if basis == 'def2-svpd' else 'h2o_dimer_tzvp.npz'
    g, mol, bas = load_golden(name)
    ref = RefOracle(mol, bas, partition=False)
    for which in range(3):
        assert np.max(np.abs(nat.one_electron(which, mol, bas) - ref.one_electron(which))) < 1e-11, which


@pytest.mark.gpu
def test_one_electron_device_output_matches_host_output():
    """vlx_b200_one_electron_device (output in device memory, as the SCF
    driver keeps S, T, V) gives the host-output entry's matrices."""
    import torch
    from veloxchem_b200 import _native as nat
    mol, bas = _dimer()
    n = bas.get_dimensions_of_basis()
    for which in range(3):
        out = torch.full((n, n), 7.0, dtype=torch.float64, device='cuda')
        nat.one_electron_device(which, mol, bas, out)
        assert np.max(np.abs(out.cpu().numpy() - nat.one_electron(which, mol, bas))) < 1e-14, which


@pytest.mark.gpu
def test_mixed_overlap_against_reference():
    from oracle.oracle import RefOracle
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200 import _native as nat
    mol, bas = _dimer()
    mini = MolecularBasis.read(mol, 'ao-start-guess')
    ref = RefOracle(mol, mini, partition=False).overlap_mixed(RefOracle(mol, bas, partition=False))
    assert np.max(np.abs(nat.one_electron(0, mol, mini, bas) - ref)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize('guess', ['sad', 'core'])
def test_scf_energy_known_answer(guess):
    from veloxchem_b200.scf import ScfRestrictedDriver
    mol, bas = _dimer()
    drv = ScfRestrictedDriver()
    drv.guess = guess
    res = drv.compute(mol, bas)
    assert res['converged']
    assert abs(res['scf_energy'] - REF_ENERGY) < 1e-8


@pytest.mark.gpu
def test_sad_density_is_a_valid_guess():
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200 import _native as nat
    from veloxchem_b200.scf import SadGuessDriver
    mol, bas = _dimer()
    mini = MolecularBasis.read(mol, 'ao-start-guess')
    D = SadGuessDriver().compute(mol, mini, bas)
    S = nat.one_electron(0, mol, bas)
    # trace(D S) = number of alpha electrons of the neutral atoms
    assert abs(np.trace(D @ S) - mol.number_of_electrons() / 2) < 1e-10
    assert np.allclose(D, D.T)
    # the driver projects once per element; every atom projected on its own
    # gives the same density
    s12 = nat.one_electron(0, mol, mini, bas)
    ao1 = SadGuessDriver.ao_indices_of_atoms(mol, mini)
    ao2 = SadGuessDriver.ao_indices_of_atoms(mol, bas)
    c = np.zeros((S.shape[0], s12.shape[0]))
    for a, z in enumerate(mol.get_element_ids()):
        i1, i2 = ao1[a], ao2[a]
        occ = np.array(SadGuessDriver.occupation_numbers(int(z)))
        b22_inv = np.linalg.inv(S[np.ix_(i2, i2)])
        m = s12[np.ix_(i1, i2)] @ b22_inv @ s12[np.ix_(i1, i2)].T
        w, v = np.linalg.eigh(m)
        c[np.ix_(i2, i1)] = b22_inv @ s12[np.ix_(i1, i2)].T @ ((v / np.sqrt(w)) @ v.T) * np.sqrt(occ)[None, :]
    assert np.max(np.abs(D - c @ c.T)) < 1e-10


@pytest.mark.gpu
def test_incremental_fock_builds_reach_the_full_build_energy():
    """Incremental builds (G of the density change, screened against max|dD|)
    end on the energy of full builds to 1e-9 Eh; convergence is confirmed on a
    full build, and the run does use incremental iterations."""
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200.geometry import water_cluster
    from veloxchem_b200.scf import ScfRestrictedDriver
    mol = water_cluster((2, 2, 2), 3)
    bas = MolecularBasis.read(mol, 'def2-svp')
    res = {}
    for inc in (False, True):
        drv = ScfRestrictedDriver()
        drv.incremental = inc
        res[inc] = drv.compute(mol, bas)
        assert res[inc]['converged']
    assert abs(res[True]['scf_energy'] - res[False]['scf_energy']) < 1e-9
    assert any(h.get('incremental') for h in res[True]['history'])
    assert not res[True]['history'][-1].get('incremental')


@pytest.mark.gpu
def test_early_loose_iterations_reach_the_reference_energy():
    """Early iterations at ithreshold 8 with FP32 below 1e-4 (mixed precision,
    incremental builds): the converged energy is still the reference's, and
    the early iterations did use the looser threshold."""
    from veloxchem_b200.scf import ScfRestrictedDriver
    mol, bas = _dimer()
    drv = ScfRestrictedDriver()
    drv.fp32_cutoff = 1e-6
    drv.early_ithreshold = 8
    res = drv.compute(mol, bas)
    assert res['converged']
    assert abs(res['scf_energy'] - REF_ENERGY) < 1e-8
    assert res['history'][0]['ithreshold'] == 8
    assert res['history'][-1]['ithreshold'] == 12


@pytest.mark.gpu
def test_full_builds_with_fp32_digestion_reach_the_reference_energy():
    """The fast configuration with FP32 evaluation and digestion of the
    quartets bounded below 1e-6 in the full builds after the early phase
    (full_fp32_digestion_cutoff), per-quartet density screening and
    incremental builds: it converges to the reference energy."""
    from veloxchem_b200.scf import ScfRestrictedDriver
    mol, bas = _dimer()
    drv = ScfRestrictedDriver()
    drv.fp32_cutoff = 1e-4
    drv.early_ithreshold = 8
    drv.full_skip_factor = 1e-2
    drv.early_skip_factor = 1e-1
    drv.full_fp32_digestion_cutoff = 1e-6
    res = drv.compute(mol, bas)
    assert res['converged']
    assert abs(res['scf_energy'] - REF_ENERGY) < 1e-8
    # the switch build after the early phase is a mixed full build
    assert any(not h['incremental'] and h['ithreshold'] > 8 and h['mixed'] for h in res['history'])


def test_scf_threshold_schedule():
    """The reference's dynamic ERI threshold (ScfDriver._get_dyn_threshold:
    1e-10 for gradients >= 1, one decade tighter per decade of gradient, 1e-12
    floor) and the optional looser early iterations."""
    from veloxchem_b200.scf import ScfRestrictedDriver
    drv = ScfRestrictedDriver()
    assert [drv._ithreshold(g, False) for g in (20.0, 1.0, 0.5, 0.05, 5e-3, 1e-7)] == [10, 10, 11, 12, 12, 12]
    drv.early_ithreshold = 8
    assert [drv._ithreshold(g, True) for g in (20.0, 0.5, 5e-3)] == [8, 8, 8]
    assert drv._fp32_cutoff(True) == 0.0  # mixed precision off: no FP32 at all
    drv.fp32_cutoff = 1e-6
    assert drv._fp32_cutoff(True) == 1e-4 and drv._fp32_cutoff(False) == 1e-6


def test_c2diis_weights_find_the_zero_residual_combination():
    """C2-DIIS picks the unit-sum eigenvector of the error overlap matrix with
    the smallest residual: for error vectors e and -e/3 that is the exact
    cancellation w = (1/4, 3/4), applied to the Fock matrices."""
    import torch
    from veloxchem_b200.scf import ScfRestrictedDriver
    rng = np.random.default_rng(0)
    e = torch.from_numpy(rng.standard_normal((6, 6)))
    f1, f2 = torch.ones((6, 6), dtype=torch.float64), 2.0 * torch.ones((6, 6), dtype=torch.float64)
    out = ScfRestrictedDriver._c2diis([f1, f2], [e, -e / 3.0])
    assert torch.allclose(out, 0.25 * f1 + 0.75 * f2, atol=1e-12)


@pytest.mark.gpu
def test_scf_energy_known_answer_pulay_diis():
    """The known answer with Pulay DIIS (the driver's default is the
    reference's C2-DIIS, which the other SCF tests use)."""
    from veloxchem_b200.scf import ScfRestrictedDriver
    mol, bas = _dimer()
    drv = ScfRestrictedDriver()
    drv.acc_type = 'diis'
    res = drv.compute(mol, bas)
    assert res['converged']
    assert abs(res['scf_energy'] - REF_ENERGY) < 1e-8
