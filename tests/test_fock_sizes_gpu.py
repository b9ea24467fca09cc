"""Parity at the workload sizes: the plain FP64 GPU build against the
reference FockDriver (compiled from source) on

* (H2O)_32 / def2-SVP (768 functions, ithreshold 12): J, K and 2J - K
  computed by the reference here (a few seconds per label on the host
  cores) -- max abs element within 1e-10;
* (H2O)_64 / def2-TZVP (2,752 functions, f shells, ithreshold 12): the
  committed fixture tests/golden/h2o64_tzvp_jk.npz (made once by
  tests/golden/make_c3_fixture.py with the reference: 48 full rows of J
  and K, and the per-row max |J|, |K|) -- within 1e-10;
* the batched 256-cluster workload (def2-SVP, n ~ U{1..16}): a seeded sample
  of 12 molecules of the full-size batched build against the reference run
  one molecule at a time.
"""

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _ref_available():
    from oracle.oracle import ref_available
    return ref_available()


@pytest.mark.skipif(not _ref_available(), reason='reference oracle not built')
def test_h2o32_svp_against_reference():
    import os
    from oracle.oracle import RefOracle
    from veloxchem_b200 import FockDriver, MolecularBasis, T4CScreener, make_matrix, mat_t
    from veloxchem_b200.geometry import random_density, water_cluster
    mol = water_cluster((4, 4, 2), 1)
    bas = MolecularBasis.read(mol, 'def2-svp')
    dens = random_density(768, 160, 1)
    scr = T4CScreener()
    scr.partition(bas, mol, 'eri')
    dm = make_matrix(bas, mat_t.symmetric)
    dm.set_values(dens)
    RefOracle.set_threads(os.cpu_count() or 4)
    ref = RefOracle(mol, bas)
    drv = FockDriver()
    for label in ('j', 'k', '2jk'):
        f = drv.compute(scr, dm, label, 1.0, 0.0, 12).full_matrix().to_numpy()
        r = ref.fock(dens, label, 1.0, 0.0, 12)
        assert np.max(np.abs(f - r)) < TOL, label


def test_h2o64_tzvp_against_reference_fixture():
    from veloxchem_b200 import FockDriver, MolecularBasis, T4CScreener, make_matrix, mat_t
    from veloxchem_b200.geometry import random_density, water_cluster
    path = GOLDEN / 'h2o64_tzvp_jk.npz'
    g = np.load(path)
    mol = water_cluster(tuple(int(v) for v in g['lattice']), int(g['seed']))
    bas = MolecularBasis.read(mol, str(g['basis']))
    nao = int(g['nao'])
    assert bas.get_dimensions_of_basis() == nao == 2752
    dens = random_density(nao, int(g['nocc']), int(g['seed']))
    ck = np.array([dens.sum(), (dens * dens).sum(), np.abs(dens).max(), dens.trace()])
    assert np.allclose(ck, g['d_checksums'], rtol=1e-10, atol=1e-10), 'density generator drifted'
    scr = T4CScreener()
    scr.partition(bas, mol, 'eri')
    dm = make_matrix(bas, mat_t.symmetric)
    dm.set_values(dens)
    drv = FockDriver()
    rows = g['rows']
    for label in ('j', 'k'):
        f = drv.compute(scr, dm, label, 1.0, 0.0, int(g['ithreshold'])).full_matrix().to_numpy()
        assert np.max(np.abs(f[rows] - g[label + '_rows'])) < TOL, label
        assert np.max(np.abs(np.abs(f).max(axis=1) - g[label + '_rowmax'])) < TOL, label


@pytest.mark.skipif(not _ref_available(), reason='reference oracle not built')
def test_batched_256_clusters_sample_against_reference():
    import os
    import torch
    from oracle.oracle import RefOracle
    from veloxchem_b200 import MolecularBasis, T4CScreener
    from veloxchem_b200.batch import FockBatch
    from veloxchem_b200.geometry import batch_clusters, random_density
    mols, ns = batch_clusters(256, 16, 7)
    scrs, dens, bases = [], [], []
    for i, (m, n) in enumerate(zip(mols, ns)):
        b = MolecularBasis.read(m, 'def2-svp')
        s = T4CScreener()
        s.partition(b, m, 'eri')
        scrs.append(s)
        bases.append(b)
        dens.append(random_density(s.nao, 5 * n, 1000 + i))
    batch = FockBatch(scrs)
    d = torch.from_numpy(batch.pack(dens)).cuda()
    f = torch.empty_like(d)
    batch.build_device(d, f, use_graph=True)
    torch.cuda.synchronize()
    out = f.cpu().numpy()
    RefOracle.set_threads(os.cpu_count() or 4)
    sample = np.random.default_rng(11).choice(256, size=12, replace=False)
    for k in sample:
        nao = scrs[k].nao
        got = out[batch.offsets[k]:batch.offsets[k + 1]].reshape(nao, nao)
        ref = RefOracle(mols[k], bases[k]).fock(dens[k], '2jk', 1.0, 0.0, 12)
        assert np.max(np.abs(got - ref)) < TOL, (k, ns[k])
