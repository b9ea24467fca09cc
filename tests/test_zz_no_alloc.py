"""GPU test of vlx_b200_fock_build_noalloc, the build for callers that cannot
let the library allocate device memory (their own pool owns the GPU memory, or
they cannot afford the device-wide synchronisation of cudaFree).  It must
match the ordinary allocating build on two calls in a row (its static scratch
keeps the previous call's contents), reject bases above its static limit, and
refuse to run before the screener has a work list for the threshold."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _noalloc(scr, d_density, d_fock, label='2jk', symmetric=1, ith=12):
    from veloxchem_b200 import _native as nat
    return nat.lib().vlx_b200_fock_build_noalloc(scr.handle, ctypes.c_void_p(d_density.data_ptr()), symmetric,
                                                 label.encode(), 1.0, 0.0, ith, ctypes.c_void_p(d_fock.data_ptr()),
                                                 None)


def _system(lattice, nwaters, seed):
    from veloxchem_b200 import MolecularBasis, T4CScreener
    from veloxchem_b200.geometry import random_density, water_cluster
    mol = water_cluster(lattice, seed, nwaters)
    bas = MolecularBasis.read(mol, 'def2-svp')
    scr = T4CScreener()
    scr.partition(bas, mol, 'eri')
    return mol, bas, scr, random_density(scr.nao, 5 * nwaters, seed)


def test_noalloc_matches_allocating_build_twice():
    import torch
    from veloxchem_b200 import FockDriver, make_matrix, mat_t
    from veloxchem_b200 import _native as nat
    mol, bas, scr, dens = _system((2, 2, 2), 8, 3)
    dm = make_matrix(bas, mat_t.symmetric)
    dm.set_values(dens)
    for label in ('2jk', 'k'):
        # the existing entry point gives the expected matrix (and builds the work list)
        ref = FockDriver().compute(scr, dm, label, 1.0, 0.0, 12).full_matrix().to_numpy()
        d_dens = torch.from_numpy(dens).cuda()
        for _ in range(2):
            d_fock = torch.full_like(d_dens, float('nan'))
            torch.cuda.synchronize()
            nat.check(_noalloc(scr, d_dens, d_fock, label), 'fock_build_noalloc')
            torch.cuda.synchronize()
            assert np.max(np.abs(d_fock.cpu().numpy() - ref)) < TOL


def test_noalloc_rejects_basis_above_limit():
    import torch
    from veloxchem_b200 import _native as nat
    mol, bas, scr, dens = _system((6, 6, 2), 43, 5)
    assert scr.nao > 1024
    dummy = torch.zeros(1, dtype=torch.float64, device='cuda')
    assert _noalloc(scr, dummy, dummy) == 1
    assert b'1024' in nat.lib().vlx_b200_last_error()


def test_noalloc_needs_existing_work_list():
    import torch
    from veloxchem_b200 import _native as nat
    mol, bas, scr, dens = _system((2, 2, 1), 4, 9)
    d = torch.from_numpy(dens).cuda()
    f = torch.zeros_like(d)
    assert _noalloc(scr, d, f, ith=11) == 1
    assert b'work list' in nat.lib().vlx_b200_last_error()
