"""Multi-rank plumbing on CPU (gloo, world size 2).

* ``reduce_fock`` over the reference's own rank shares (the compiled reference
  FockDriver stands in for the GPU on a host without one) gives the full
  matrix on both ranks;
* ``distributed_fock`` itself, with its GPU driver replaced by a stub that
  records the (rank, nodes) it receives and returns the reference's share for
  them: every rank must build its own share (not the full matrix) and the
  reduced result must equal one full build.
"""

import os

import numpy as np
import pytest

from oracle.oracle import ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason='reference oracle not built')


def _init(rank, world, port):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / 'tests'))
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    return dist


def _reduce_worker(rank, world, port, out_dir):
    dist = _init(rank, world, port)
    from conftest import load_golden
    from oracle.oracle import RefOracle
    from veloxchem_b200.distributed import reduce_fock
    g, mol, bas = load_golden('h2o4_svp.npz')
    RefOracle.set_threads(2)
    part = RefOracle(mol, bas).fock(g['density'], '2jk', 1.0, 0.0, 12, True, rank, world)
    full = reduce_fock(part)
    np.save(os.path.join(out_dir, 'full_%d.npy' % rank), full)
    np.save(os.path.join(out_dir, 'part_%d.npy' % rank), part)
    dist.barrier()
    dist.destroy_process_group()


def _distributed_worker(rank, world, port, out_dir):
    dist = _init(rank, world, port)
    from conftest import load_golden
    from oracle.oracle import RefOracle
    import veloxchem_b200.fockdriver as fd
    from veloxchem_b200 import make_matrix, mat_t
    from veloxchem_b200.distributed import distributed_fock
    g, mol, bas = load_golden('h2o4_svp.npz')
    RefOracle.set_threads(2)
    ref = RefOracle(mol, bas)
    seen = []

    class StubDriver:
        """Stands in for the GPU FockDriver: the reference's share of the
        (rank, nodes) the caller passes."""

        def __init__(self, comm=None):
            self.rank, self.nodes = fd._comm_rank_size(comm)

        def compute(self, screener, density, label, xfac, omega, ith):
            seen.append((self.rank, self.nodes))
            part = ref.fock(density.full_matrix().to_numpy(), label, xfac, omega, ith, True, self.rank, self.nodes)
            out = density.copy()
            out.zero()
            out.set_values(part)
            return out

    class StubScreener:
        def __init__(self):
            self.partitions = []

        def set_partition(self, p):
            self.partitions.append(p)

    fd.FockDriver = StubDriver
    scr = StubScreener()
    dm = make_matrix(bas, mat_t.symmetric)
    dm.set_values(g['density'])
    full = distributed_fock(scr, dm, '2jk', 1.0, 0.0, 12, partition='balanced').full_matrix().to_numpy()
    np.save(os.path.join(out_dir, 'dfull_%d.npy' % rank), full)
    np.save(os.path.join(out_dir, 'seen_%d.npy' % rank), np.array(seen))
    np.save(os.path.join(out_dir, 'parts_%d.npy' % rank), np.array([scr.partitions[0] == 'balanced',
                                                                     scr.partitions[-1] == 'round_robin']))
    dist.barrier()
    dist.destroy_process_group()


def _spawn(fn, tmp_path):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    mp.start_processes(fn, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method='spawn')


def test_two_rank_reduce_matches_full_build(tmp_path):
    from conftest import load_golden
    _spawn(_reduce_worker, tmp_path)
    g, _, _ = load_golden('h2o4_svp.npz')
    for r in range(2):
        full = np.load(tmp_path / ('full_%d.npy' % r))
        assert np.max(np.abs(full - g['f2jk'])) < 1e-12
    p0, p1 = np.load(tmp_path / 'part_0.npy'), np.load(tmp_path / 'part_1.npy')
    assert np.max(np.abs(p0)) > 0 and np.max(np.abs(p1)) > 0
    assert np.max(np.abs(p0 - g['f2jk'])) > 1e-6


def test_distributed_fock_builds_own_share_and_reduces(tmp_path):
    from conftest import load_golden
    _spawn(_distributed_worker, tmp_path)
    g, _, _ = load_golden('h2o4_svp.npz')
    for r in range(2):
        # each rank built exactly its own share of a 2-rank split
        assert np.load(tmp_path / ('seen_%d.npy' % r)).tolist() == [[r, 2]]
        # the partition was switched for the call and restored after it
        assert np.load(tmp_path / ('parts_%d.npy' % r)).all()
        full = np.load(tmp_path / ('dfull_%d.npy' % r))
        assert np.max(np.abs(full - g['f2jk'])) < 1e-12
