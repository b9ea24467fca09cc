"""Batched many-molecule Fock builds (one launch per quartet class over all
molecules, replayed from a CUDA graph) against one build per molecule through
the single-molecule entry point and against the oracle.  Tolerance: 1e-10
absolute per element, as for the single builds (the batched kernels differ
only in the order of the FP64 atomic additions)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _setup(count, nmax, seed=11):
    from veloxchem_b200 import MolecularBasis, T4CScreener
    from veloxchem_b200.geometry import batch_clusters, random_density
    mols, ns = batch_clusters(count, nmax, seed)
    bases, scrs, dens = [], [], []
    for i, (m, n) in enumerate(zip(mols, ns)):
        b = MolecularBasis.read(m, 'def2-svp')
        s = T4CScreener()
        s.partition(b, m, 'eri')
        bases.append(b)
        scrs.append(s)
        dens.append(random_density(s.nao, 5 * n, 1000 + i))
    return mols, bases, scrs, dens


def _single(scr, bas, d, label='2jk', xfac=1.0, ith=12, symmetric=True):
    from veloxchem_b200 import FockDriver, make_matrix, mat_t
    m = make_matrix(bas, mat_t.symmetric if symmetric else mat_t.general)
    m.set_values(d)
    return FockDriver().compute(scr, m, label, xfac, 0.0, ith).full_matrix().to_numpy()


@pytest.mark.parametrize('use_graph', [True, False])
def test_batch_matches_single_builds(use_graph):
    from veloxchem_b200.batch import FockBatch
    mols, bases, scrs, dens = _setup(24, 6)
    batch = FockBatch(scrs)
    out = batch.compute(dens, '2jk', 1.0, 0.0, 12, use_graph=use_graph)
    for k in range(len(mols)):
        ref = _single(scrs[k], bases[k], dens[k])
        assert np.max(np.abs(out[k] - ref)) < TOL, k
    assert batch.last_stats['shell_quartets'] > 0


def test_batch_graph_replay_follows_new_densities():
    """Same device buffers, new contents: the replayed graph reads them."""
    import torch
    from veloxchem_b200.batch import FockBatch
    mols, bases, scrs, dens = _setup(12, 4, seed=5)
    batch = FockBatch(scrs)
    d = torch.from_numpy(batch.pack(dens)).cuda()
    f = torch.empty_like(d)
    batch.build_device(d, f)
    first = batch.unpack(f.cpu().numpy())
    dens2 = [0.5 * x + 0.1 * np.eye(x.shape[0]) for x in dens]
    d.copy_(torch.from_numpy(batch.pack(dens2)))
    batch.build_device(d, f)
    second = batch.unpack(f.cpu().numpy())
    for k in range(len(mols)):
        assert np.max(np.abs(first[k] - _single(scrs[k], bases[k], dens[k]))) < TOL
        assert np.max(np.abs(second[k] - _single(scrs[k], bases[k], dens2[k]))) < TOL


def test_batch_labels_general_density_and_oracle():
    from oracle.oracle import PortOracle
    from veloxchem_b200.batch import FockBatch
    mols, bases, scrs, dens = _setup(6, 3, seed=3)
    batch = FockBatch(scrs)
    rng = np.random.default_rng(0)
    gen = [d + 0.05 * rng.standard_normal(d.shape) for d in dens]
    out_k = batch.compute(gen, 'k', 1.0, 0.0, 12, symmetric=False)
    out_j = batch.compute(dens, 'j', 1.0, 0.0, 12)
    for k in range(len(mols)):
        assert np.max(np.abs(out_k[k] - _single(scrs[k], bases[k], gen[k], 'k', 1.0, 12, False))) < TOL
        ref = PortOracle(mols[k], bases[k]).fock(dens[k], 'j', 1.0, 12)
        assert np.max(np.abs(out_j[k] - ref)) < TOL
