"""Parity of the CUDA Fock build (through the C ABI) with the oracle and the
reference's golden matrices.  Tolerances: J, K and 2J-K to 1e-10 absolute
(max element), ERI tensors to 1e-12, Schwarz values to 1e-12 relative."""

import json
import pickle

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _fock(screener, dense, label, xfac=1.0, ith=15, symmetric=True, rank=0, nodes=1):
    from veloxchem_b200 import FockDriver, make_matrix, mat_t
    drv = FockDriver((rank, nodes))
    m = make_matrix(screener._basis, mat_t.symmetric if symmetric else mat_t.general)
    m.set_values(dense)
    return drv.compute(screener, m, label, xfac, 0.0, ith).full_matrix().to_numpy()


def _screener(mol, bas):
    from veloxchem_b200 import T4CScreener
    s = T4CScreener()
    s.partition(bas, mol, 'eri')
    s._basis = bas
    return s


def test_boys_device_against_oracle():
    from oracle.oracle import PortOracle
    from veloxchem_b200 import _native
    t = np.concatenate([np.linspace(0.0, 45.0, 901), [1e-12, 39.999999, 40.0, 60.0, 120.0, 700.0]])
    for m in range(0, 17):
        dev = _native.boys_device(m, t)
        ref = np.array([PortOracle.boys(m, x) for x in t])
        assert np.max(np.abs(dev - ref) / np.maximum(ref, 1e-300)) < 5e-14, m


def test_screener_known_answers_and_bins():
    from oracle.oracle import PortOracle
    kat = json.loads((GOLDEN / 'screener_sto3g.json').read_text())
    g, mol, bas = load_golden('h2o_sto3g.npz')
    s = _screener(mol, bas)
    info, maxv = s.pair_info()
    for blk, key in enumerate(['ss', 'sp', 'pp']):
        assert np.allclose(maxv[info[:, 0] == blk], kat[key], rtol=1e-12, atol=1e-14)
    oinfo, omax = PortOracle(mol, bas).pair_info()
    assert np.array_equal(info, oinfo)


def test_screener_pickle_roundtrip():
    g, mol, bas = load_golden('h2o_sto3g.npz')
    a = _screener(mol, bas)
    b = pickle.loads(pickle.dumps(a))
    assert a == b


def test_eri_tensor_sto3g_golden():
    from veloxchem_b200 import FockDriver
    g, mol, bas = load_golden('h2o_sto3g.npz')
    eri = FockDriver().compute_eri(mol, bas)
    assert np.max(np.abs(eri - g['eri'])) < 1e-12


@pytest.mark.parametrize('basis', ['def2-svp', 'def2-tzvp'])
def test_eri_tensor_every_class(basis):
    """All quartet classes of the basis (compiled and table-driven) against
    the oracle's ERI tensor, on one water molecule."""
    from oracle.oracle import PortOracle
    from veloxchem_b200 import FockDriver, MolecularBasis, Molecule
    mol = Molecule.read_str('O 0.1 -0.05 0.02\nH 0.0 0.76 0.59\nH -0.02 -0.74 0.61')
    bas = MolecularBasis.read(mol, basis)
    eri = FockDriver().compute_eri(mol, bas, 1e-15)
    ref = PortOracle(mol, bas).eri(15)
    assert np.max(np.abs(eri - ref)) < 1e-12


@pytest.mark.parametrize('name', ['h2o_sto3g.npz', 'h2o_dimer_svpd.npz', 'h2o_dimer_tzvp.npz'])
def test_jk_against_reference_goldens(name):
    g, mol, bas = load_golden(name)
    s = _screener(mol, bas)
    j = _fock(s, g['density'], 'j', 0.0)
    k = _fock(s, g['density'], 'k', 0.0)
    f = _fock(s, g['density'], '2jk', 0.0)
    assert np.max(np.abs(j - g['j'])) < TOL
    assert np.max(np.abs(k - g['k'])) < TOL
    assert np.max(np.abs(f - (2 * g['j'] - g['k']))) < TOL


def test_general_density_against_goldens():
    g, mol, bas = load_golden('h2o_dimer_svpd.npz')
    s = _screener(mol, bas)
    j = _fock(s, g['density_gen'], 'j', 0.0, symmetric=False)
    k = _fock(s, g['density_gen'], 'k', 0.0, symmetric=False)
    assert np.max(np.abs(j - g['j_gen'])) < TOL
    assert np.max(np.abs(k - g['k_gen'].T)) < TOL


@pytest.mark.parametrize('label,xfac', [('2jk', 1.0), ('2jkx', 0.28), ('j', 1.0), ('k', 1.0), ('kx', 0.73)])
def test_labels_against_oracle(label, xfac):
    from oracle.oracle import PortOracle
    g, mol, bas = load_golden('h2o_dimer_tzvp.npz')
    s = _screener(mol, bas)
    ref = PortOracle(mol, bas).fock(g['density'], label, xfac, 15)
    assert np.max(np.abs(_fock(s, g['density'], label, xfac) - ref)) < TOL


def test_unknown_label_gives_zero_matrix():
    g, mol, bas = load_golden('h2o_sto3g.npz')
    s = _screener(mol, bas)
    assert np.all(_fock(s, g['density'], 'nonsense', 0.0) == 0.0)


def test_cluster_fixture_ithreshold12():
    """(H2O)_4 / def2-SVP, seeded density, against the compiled reference."""
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    assert np.max(np.abs(_fock(s, g['density'], 'j', 1.0, 12) - g['j'])) < TOL
    assert np.max(np.abs(_fock(s, g['density'], 'k', 1.0, 12) - g['k'])) < TOL
    assert np.max(np.abs(_fock(s, g['density'], '2jk', 1.0, 12) - g['f2jk'])) < TOL


@pytest.mark.parametrize('ith', [4, 8, 10])
def test_loose_thresholds_match_oracle(ith):
    """The screening rule (bin sums) at thresholds that drop many quartets."""
    from oracle.oracle import PortOracle
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    ref = PortOracle(mol, bas).fock(g['density'], '2jk', 1.0, ith)
    assert np.max(np.abs(_fock(s, g['density'], '2jk', 1.0, ith) - ref)) < TOL


def test_rank_partition_sums_to_full_build():
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    full = _fock(s, g['density'], '2jk', 1.0, 12)
    parts = [_fock(s, g['density'], '2jk', 1.0, 12, rank=r, nodes=3) for r in range(3)]
    assert np.max(np.abs(sum(parts) - full)) < 1e-12
    assert all(np.max(np.abs(p)) > 0 for p in parts)


def test_multi_density_overload():
    from veloxchem_b200 import FockDriver, Matrices, make_matrix, mat_t
    g, mol, bas = load_golden('h2o_dimer_svpd.npz')
    s = _screener(mol, bas)
    dm = make_matrix(bas, mat_t.general)
    dm.set_values(g['density_gen'])
    dens = Matrices()
    dens.add(dm, '0')
    dens.add(dm, '1')
    out = FockDriver().compute(s, dens, ['j', 'k'], 0.0, 0.0, 15)
    assert np.max(np.abs(out.matrix('0').full_matrix().to_numpy() - g['j_gen'])) < TOL
    assert np.max(np.abs(out.matrix('1').full_matrix().to_numpy() - g['k_gen'].T)) < TOL


def test_multi_density_single_pass_labels_and_omega():
    """One pass over the quartets for several densities (more than one pass
    of 8 here): each result equals its own single build; with a mixed label
    list the range-separated label takes the Coulomb operator, as the
    reference's CT4CMatricesDistributor::need_omega decides; with all labels
    range-separated omega applies to all.  The single pass costs about one
    build, not one per density (device times printed)."""
    from veloxchem_b200 import FockDriver, Matrices, make_matrix, mat_t
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    rng = np.random.default_rng(3)
    dens = []
    for i in range(10):
        a = g['density'] + 0.01 * i * rng.standard_normal(g['density'].shape)
        dens.append(0.5 * (a + a.T))
    labels = ['2jk', 'j', 'k', 'kx', '2jkx', 'j', 'k', '2jk', 'k_rs', 'j']
    drv = FockDriver()
    mats = Matrices()
    for i, d in enumerate(dens):
        m = make_matrix(bas, mat_t.symmetric)
        m.set_values(d)
        mats.add(m, str(i))
    out = drv.compute(s, mats, labels, 0.3, 0.4, 12)
    multi_ms = drv.last_stats['device_ms']
    for i, (d, lab) in enumerate(zip(dens, labels)):
        single = _fock(s, d, 'k' if lab == 'k_rs' else lab, 0.3, 12)
        assert np.max(np.abs(out.matrix(str(i)).full_matrix().to_numpy() - single)) < TOL, (i, lab)
    drv.compute(s, mats.matrix('0'), '2jk', 1.0, 0.0, 12)
    one_ms = drv.last_stats['device_ms']
    # all range-separated: omega for every density
    mats2 = Matrices()
    for i in range(2):
        m = make_matrix(bas, mat_t.symmetric)
        m.set_values(dens[i])
        mats2.add(m, str(i))
    out2 = drv.compute(s, mats2, ['j_rs', 'k_rs'], 1.0, 0.4, 12)
    for i, lab in enumerate(['j_rs', 'k_rs']):
        mm = make_matrix(bas, mat_t.symmetric)
        mm.set_values(dens[i])
        ref = drv.compute(s, mm, lab, 1.0, 0.4, 12).full_matrix().to_numpy()
        assert np.max(np.abs(out2.matrix(str(i)).full_matrix().to_numpy() - ref)) < TOL
    print('multi-density: 10 densities in %.2f ms, one single build %.2f ms' % (multi_ms, one_ms))


def test_block_size_factor_does_not_change_result():
    from veloxchem_b200 import FockDriver, make_matrix, mat_t
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    drv = FockDriver()
    m = make_matrix(bas, mat_t.symmetric)
    m.set_values(g['density'])
    a = drv.compute(s, m, '2jk', 1.0, 0.0, 12).full_matrix().to_numpy()
    drv._set_block_size_factor(8)
    b = drv.compute(s, m, '2jk', 1.0, 0.0, 12).full_matrix().to_numpy()
    assert np.max(np.abs(a - b)) < 1e-12


@pytest.mark.parametrize('label,xfac', [('k_rs', 0.0), ('kx_rs', 0.21)])
def test_range_separated_exchange_against_golden(label, xfac):
    """erf-attenuated K (omega = 0.63) against the reference's golden matrix
    (its tests/test_fock_erf_driver.py: k_rs with xfac 0, kx_rs with 0.21)."""
    g, mol, bas = load_golden('h2o_dimer_tzvp.npz')
    s = _screener(mol, bas)
    from veloxchem_b200 import FockDriver, make_matrix, mat_t
    m = make_matrix(bas, mat_t.symmetric)
    m.set_values(g['density'])
    f = FockDriver()._compute_fock_omp(s, m, label, xfac, 0.63, 15).full_matrix().to_numpy()
    scale = 1.0 if label == 'k_rs' else xfac
    assert np.max(np.abs(f - scale * g['erf_k'])) < TOL


def test_range_separated_j_against_oracle_and_limits():
    """j_rs against the compiled reference; omega is ignored by plain labels,
    omega = 0 gives a zero matrix, a negative omega is an error."""
    from oracle.oracle import RefOracle
    from veloxchem_b200._native import NativeError
    g, mol, bas = load_golden('h2o_dimer_svpd.npz')
    s = _screener(mol, bas)
    from veloxchem_b200 import FockDriver, make_matrix, mat_t
    m = make_matrix(bas, mat_t.symmetric)
    m.set_values(g['density'])
    drv = FockDriver()
    j_rs = drv._compute_fock_omp(s, m, 'j_rs', 0.0, 0.4, 15).full_matrix().to_numpy()
    ref = RefOracle(mol, bas).fock(g['density'], 'j_rs', 0.0, 0.4, 15)
    assert np.max(np.abs(j_rs - ref)) < TOL
    assert np.max(np.abs(j_rs - g['j'])) > 1e-3
    j = drv._compute_fock_omp(s, m, 'j', 0.0, 0.4, 15).full_matrix().to_numpy()
    assert np.max(np.abs(j - g['j'])) < TOL
    assert np.all(drv._compute_fock_omp(s, m, 'k_rs', 0.0, 0.0, 15).full_matrix().to_numpy() == 0.0)
    with pytest.raises(NativeError):
        drv._compute_fock_omp(s, m, 'k_rs', 0.0, -0.3, 15)


def test_large_cluster_properties():
    """(H2O)_32 / def2-SVP at ithreshold 12 (the bench workload): size-independent
    checks -- F symmetric, J positive semidefinite energy, linearity in D."""
    from veloxchem_b200.geometry import CLUSTERS, random_density, water_cluster
    from veloxchem_b200 import MolecularBasis
    lattice, seed = CLUSTERS['h2o32']
    mol = water_cluster(lattice, seed)
    bas = MolecularBasis.read(mol, 'def2-svp')
    s = _screener(mol, bas)
    assert s.nao == 768
    d1 = random_density(768, 160, 1)
    d2 = random_density(768, 160, 2)
    j1 = _fock(s, d1, 'j', 1.0, 12)
    j2 = _fock(s, d2, 'j', 1.0, 12)
    j12 = _fock(s, d1 + 0.5 * d2, 'j', 1.0, 12)
    assert np.max(np.abs(j12 - (j1 + 0.5 * j2))) < 1e-9
    assert np.max(np.abs(j1 - j1.T)) < 1e-12
    assert np.sum(d1 * j1) > 0
    k1 = _fock(s, d1, 'k', 1.0, 12)
    f1 = _fock(s, d1, '2jk', 1.0, 12)
    assert np.max(np.abs(f1 - (2 * j1 - k1))) < 1e-9


def test_mixed_precision_build():
    """FP32 for quartets with bound x max|D| below the cutoff: no FP32 quartet
    at a vanishing cutoff (bitwise the FP64 path), a bounded Fock error and a
    real FP32 share at the default cutoffs; switching off restores FP64."""
    import torch
    from veloxchem_b200 import _native as nat
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    d = torch.from_numpy(g['density']).cuda()
    f64 = torch.empty_like(d)
    prof64 = nat.fock_profile(s, d.data_ptr(), f64.data_ptr(), '2jk', 1.0, 12)
    assert sum(p['fp32_quartets'] for p in prof64) == 0
    dmax = float(d.abs().max())
    errors = {}
    for cutoff in (1e-9, 1e-7, 1e-5):
        s.set_fp32_threshold(cutoff, dmax)
        fm = torch.empty_like(d)
        prof = nat.fock_profile(s, d.data_ptr(), fm.data_ptr(), '2jk', 1.0, 12)
        n32 = sum(p['fp32_quartets'] for p in prof)
        assert n32 > 0
        if cutoff >= 1e-7:
            assert any(p['fp32_quartets'] > 0 for p in prof if not p['table_driven'])
        errors[cutoff] = float((fm - f64).abs().max())
    assert errors[1e-9] < 1e-10 and errors[1e-7] < 1e-8 and errors[1e-5] < 1e-6
    s.set_fp32_threshold(0.0, 0.0)
    f2 = torch.empty_like(d)
    nat.fock_profile(s, d.data_ptr(), f2.data_ptr(), '2jk', 1.0, 12)
    assert float((f2 - f64).abs().max()) < 1e-12


def test_mixed_precision_warp_cooperative_classes():
    """The FP32 twin of the warp-cooperative kernel (the f classes that stay
    interpreted, present in the def2-TZVP water dimer): FP32 quartets are
    evaluated there and the Fock error stays below a tenth of the cutoff."""
    import torch
    from veloxchem_b200 import _native as nat
    g, mol, bas = load_golden('h2o_dimer_tzvp.npz')
    s = _screener(mol, bas)
    d = torch.from_numpy(g['density']).cuda()
    f64 = torch.empty_like(d)
    prof64 = nat.fock_profile(s, d.data_ptr(), f64.data_ptr(), '2jk', 1.0, 12)
    assert any(p['table_driven'] for p in prof64)
    s.set_fp32_threshold(1e-5, float(d.abs().max()))
    fm = torch.empty_like(d)
    prof = nat.fock_profile(s, d.data_ptr(), fm.data_ptr(), '2jk', 1.0, 12)
    s.set_fp32_threshold(0.0, 0.0)
    assert any(p['fp32_quartets'] > 0 for p in prof if p['table_driven'])
    assert float((fm - f64).abs().max()) < 1e-6


def test_density_screening_build():
    """Per-quartet density screening (bound sqrt((PQ|PQ)(RS|RS)) x weighted
    local shell-block maxima of |D|): both cutoffs 0 is the reference's
    screening; an FP32 cutoff keeps every quartet and evaluates some in FP32
    with the Fock error below a tenth of the cutoff (the decade-bin split's
    FP32 count at the same cutoff is printed beside it); a skip cutoff evaluates fewer quartets with
    the error bounded; general densities are bounded in both orientations."""
    import torch
    from veloxchem_b200 import _native as nat
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    d = torch.from_numpy(g['density']).cuda()

    def build(dens, symmetric=True):
        f = torch.empty_like(dens)
        prof = nat.fock_profile(s, dens.data_ptr(), f.data_ptr(), '2jk', 1.0, 12, symmetric)
        return f, sum(p['shell_quartets'] for p in prof), sum(p['fp32_quartets'] for p in prof)

    f64, nq, _ = build(d)
    s.set_density_screening(0.0, 0.0)
    f0, nq0, n320 = build(d)
    assert nq0 == nq and n320 == 0 and float((f0 - f64).abs().max()) < 1e-13
    dmax = float(d.abs().max())
    for cutoff in (1e-9, 1e-7, 1e-5):
        s.set_fp32_threshold(cutoff, dmax)
        _, _, n32_bins = build(d)
        s.set_density_screening(cutoff, 0.0)
        fm, nqm, n32 = build(d)
        err = float((fm - f64).abs().max())
        print('density screening fp32 cutoff %.0e: FP32 %d of %d quartets (bins: %d), error %.2e'
              % (cutoff, n32, nqm, n32_bins, err))
        assert nqm == nq and n32 > 0
        assert err < 0.1 * cutoff
    # FP32 digestion of the FP32 quartets (FP32 copy of D, FP32 accumulator)
    s.set_fp32_digestion(True)
    for cutoff in (1e-7, 1e-5):
        s.set_density_screening(cutoff, 0.0)
        fd, nqd, n32 = build(d)
        err = float((fd - f64).abs().max())
        print('density screening fp32 cutoff %.0e with FP32 digestion: error %.2e' % (cutoff, err))
        assert nqd == nq and n32 > 0 and err < 0.1 * cutoff
    s.set_fp32_digestion(False)
    for skip in (1e-12, 1e-10):
        s.set_density_screening(0.0, skip)
        fs, nqs, _ = build(d)
        err = float((fs - f64).abs().max())
        print('density screening skip %.0e: %d of %d quartets, error %.2e' % (skip, nqs, nq, err))
        assert nqs < nq
        assert err < 1e4 * skip
    # general (non-symmetric) density: the bound covers D_ab and D_ba
    rng = np.random.default_rng(5)
    dg = torch.from_numpy(g['density'] + 1e-3 * rng.standard_normal(g['density'].shape)).cuda()
    s.set_density_screening(0.0, 0.0)
    fg64, _, _ = build(dg, False)
    s.set_density_screening(1e-7, 0.0)
    fg, _, n32 = build(dg, False)
    assert n32 > 0 and float((fg - fg64).abs().max()) < 1e-8
    s.set_density_screening(0.0, 0.0)


def test_mixed_precision_scf_energy():
    """SCF with FP32 small quartets until the gradient is below 1e-4 reaches the
    FP64 energy (the final iterations are FP64)."""
    from test_scf import REF_ENERGY, _dimer
    from veloxchem_b200.scf import ScfRestrictedDriver
    mol, bas = _dimer()
    drv = ScfRestrictedDriver()
    drv.fp32_cutoff = 1e-6
    res = drv.compute(mol, bas)
    assert res['converged'] and any(h['mixed'] for h in res['history'])
    assert abs(res['scf_energy'] - REF_ENERGY) < 1e-8


def test_autotune_keeps_the_result():
    """Per-class work-item lengths chosen by timing change only the order of
    the FP64 additions: the build after tuning equals the one before (1e-12)."""
    import torch
    from veloxchem_b200 import _native as nat
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    d = torch.from_numpy(g['density']).cuda()
    before = _fock(s, g['density'], '2jk', 1.0, 12)
    res = nat.autotune(s, d.data_ptr(), 12)
    torch.cuda.synchronize()
    assert res and all(r['segment'] > 0 and r['best_ms'] <= r['default_ms'] for r in res)
    after = _fock(s, g['density'], '2jk', 1.0, 12)
    assert np.max(np.abs(after - before)) < 1e-12
    assert np.max(np.abs(after - g['f2jk'])) < TOL


def test_shared_work_list_filters_thresholds_at_run_time():
    """One work list built for ithreshold 15 serves builds at looser
    thresholds: the quartets above each build's threshold are skipped in the
    kernels, and every result equals the oracle at that threshold."""
    from oracle.oracle import PortOracle
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    s.set_work_threshold(15)
    ref = PortOracle(mol, bas)
    for ith in (4, 8, 12, 15):
        f = _fock(s, g['density'], '2jk', 1.0, ith)
        assert np.max(np.abs(f - ref.fock(g['density'], '2jk', 1.0, ith))) < TOL, ith


@pytest.mark.parametrize('xyz,basis', [('H 0.0 0.0 0.0', 'sto-3g'),
                                       ('He 0.0 0.0 0.0\nHe 0.0 0.0 50.0', 'def2-svp'),
                                       ('H 0.0 0.0 0.0\nH 0.0 0.0 0.74', 'def2-tzvp')])
def test_edge_systems_against_oracle(xyz, basis):
    """Smallest systems: one function; two atoms 50 Angstrom apart (every
    cross pair screened out); a molecule with only H shells up to p."""
    from oracle.oracle import PortOracle
    from veloxchem_b200 import MolecularBasis, Molecule
    mol = Molecule.read_str(xyz)
    bas = MolecularBasis.read(mol, basis)
    s = _screener(mol, bas)
    rng = np.random.default_rng(1)
    c = rng.standard_normal((s.nao, max(1, s.nao // 2)))
    d = c @ c.T / s.nao
    for label in ('2jk', 'j', 'k'):
        ref = PortOracle(mol, bas).fock(d, label, 1.0, 15)
        assert np.max(np.abs(_fock(s, d, label, 1.0, 15) - ref)) < TOL, label


def test_threshold_zero_keeps_only_the_largest_quartets():
    from oracle.oracle import PortOracle
    g, mol, bas = load_golden('h2o4_svp.npz')
    s = _screener(mol, bas)
    f = _fock(s, g['density'], '2jk', 1.0, 0)
    assert np.max(np.abs(f - PortOracle(mol, bas).fock(g['density'], '2jk', 1.0, 0))) < TOL
    assert np.max(np.abs(f)) > 0.0
