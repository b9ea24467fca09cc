"""The product's sharded Fock build on two ranks: two processes (gloo for the
host-side sum) each build their share of the work items on the GPU through
``distributed_fock``, for both partitions, and every rank must end with the
reference's full 2J - K.  The two processes share one GPU; their kernels do
not wait on one another (the only exchange is the host all-reduce)."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _worker(rank, world, port, out_dir):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / 'tests'))
    import torch.distributed as dist
    from conftest import load_golden
    from veloxchem_b200 import FockDriver, T4CScreener, make_matrix, mat_t
    from veloxchem_b200.distributed import distributed_fock
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    g, mol, bas = load_golden('h2o4_svp.npz')
    scr = T4CScreener(device=0)
    scr.partition(bas, mol, 'eri')
    dm = make_matrix(bas, mat_t.symmetric)
    dm.set_values(g['density'])
    for part in ('round_robin', 'balanced'):
        full = distributed_fock(scr, dm, '2jk', 1.0, 0.0, 12, partition=part).full_matrix().to_numpy()
        np.save(os.path.join(out_dir, 'full_%s_%d.npy' % (part, rank)), full)
        scr.set_partition(part)
        share = FockDriver((rank, world)).compute(scr, dm, '2jk', 1.0, 0.0, 12).full_matrix().to_numpy()
        scr.set_partition('round_robin')
        np.save(os.path.join(out_dir, 'share_%s_%d.npy' % (part, rank)), share)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_distributed_fock_on_gpu(tmp_path):
    import socket
    import torch.multiprocessing as mp
    from conftest import load_golden
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method='spawn')
    g, _, _ = load_golden('h2o4_svp.npz')
    for part in ('round_robin', 'balanced'):
        for r in range(2):
            full = np.load(tmp_path / ('full_%s_%d.npy' % (part, r)))
            assert np.max(np.abs(full - g['f2jk'])) < 1e-10, part
        s0 = np.load(tmp_path / ('share_%s_0.npy' % part))
        s1 = np.load(tmp_path / ('share_%s_1.npy' % part))
        assert np.max(np.abs(s0 + s1 - g['f2jk'])) < 1e-10, part
        assert np.max(np.abs(s0 - g['f2jk'])) > 1e-6, part  # a share, not the full build
