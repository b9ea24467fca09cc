"""Multi-rank plumbing on CPU: two gloo ranks each produce the reference's
rank/nodes share of one build (the compiled reference FockDriver stands in for
the GPU on a host without one) and reduce_fock must give the full matrix on
both ranks."""

import os

import numpy as np
import pytest

from oracle.oracle import ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason='reference oracle not built')


def _worker(rank, world, port, out_dir):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / 'tests'))
    import torch.distributed as dist
    from conftest import load_golden
    from oracle.oracle import RefOracle
    from veloxchem_b200.distributed import reduce_fock
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    g, mol, bas = load_golden('h2o4_svp.npz')
    RefOracle.set_threads(2)
    part = RefOracle(mol, bas).fock(g['density'], '2jk', 1.0, 0.0, 12, True, rank, world)
    full = reduce_fock(part)
    np.save(os.path.join(out_dir, 'full_%d.npy' % rank), full)
    np.save(os.path.join(out_dir, 'part_%d.npy' % rank), part)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduce_matches_full_build(tmp_path):
    import socket
    import torch.multiprocessing as mp
    from conftest import load_golden
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method='spawn')
    g, _, _ = load_golden('h2o4_svp.npz')
    for r in range(2):
        full = np.load(tmp_path / ('full_%d.npy' % r))
        assert np.max(np.abs(full - g['f2jk'])) < 1e-12
    p0, p1 = np.load(tmp_path / 'part_0.npy'), np.load(tmp_path / 'part_1.npy')
    assert np.max(np.abs(p0)) > 0 and np.max(np.abs(p1)) > 0
    assert np.max(np.abs(p0 - g['f2jk'])) > 1e-6
