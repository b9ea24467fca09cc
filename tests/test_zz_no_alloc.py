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


def test_noalloc_honours_mixed_precision():
    """With the screener's FP32 split active the allocation-free build
    evaluates the same quartets in FP32 as the allocating device build."""
    import ctypes
    import torch
    from veloxchem_b200 import _native as nat
    mol, bas, scr, dens = _system((2, 2, 2), 8, 3)
    d = torch.from_numpy(dens).cuda()
    f64, fmix, fna = torch.zeros_like(d), torch.zeros_like(d), torch.zeros_like(d)

    def device_build(out):
        nat.check(nat.lib().vlx_b200_fock_build_device(scr.handle, ctypes.c_void_p(d.data_ptr()), 1, b'2jk', 1.0,
                                                        0.0, 12, ctypes.c_void_p(out.data_ptr()), None),
                  'fock_build_device')

    device_build(f64)
    scr.set_fp32_threshold(1e-3, float(d.abs().max()))
    device_build(fmix)
    nat.check(_noalloc(scr, d, fna), 'fock_build_noalloc')
    torch.cuda.synchronize()
    scr.set_fp32_threshold(0.0, 0.0)
    assert float((fmix - f64).abs().max()) > 1e-10      # the FP32 quartets changed the matrix
    assert float((fna - fmix).abs().max()) < 1e-10      # ... and the same way in both builds
