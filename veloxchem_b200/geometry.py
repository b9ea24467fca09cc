"""Seeded synthetic inputs for the Fock-build workloads.

Water clusters: rigid waters (O-H 0.9572 A, H-O-H 104.52 deg), the O atom of
each water placed on an nx x ny x nz lattice with 3.0 A spacing (x fastest),
shifted by a uniform jitter in [-0.3, 0.3] A per axis and given a uniformly
random orientation (random unit quaternion, Shoemake's method).  Per water the
generator draws 3 jitter values then 3 quaternion values from one
``numpy.random.default_rng(seed)`` stream, in lattice order.

Densities: D = C C^T with C the Q factor of a QR decomposition of an
N(0, 1) nao x nocc matrix (nocc = 5 per water), i.e. a random closed-shell
(idempotent in an orthonormal basis) occupied projector, in FP64.
"""

import numpy as np

from .molecule import Molecule

OH_ANGSTROM = 0.9572
HOH_DEGREES = 104.52
SPACING = 3.0
JITTER = 0.3


def _water_local():
    half = np.radians(HOH_DEGREES) / 2.0
    return np.array([[0.0, 0.0, 0.0],
                     [OH_ANGSTROM * np.sin(half), 0.0, OH_ANGSTROM * np.cos(half)],
                     [-OH_ANGSTROM * np.sin(half), 0.0, OH_ANGSTROM * np.cos(half)]])


def _rotation(u):
    u1, u2, u3 = u
    q = np.array([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(lattice, seed, nwaters=None):
    """(H2O)_n on the first ``nwaters`` sites of an nx*ny*nz lattice (x fastest)."""
    nx, ny, nz = lattice
    n = nx * ny * nz if nwaters is None else int(nwaters)
    if n > nx * ny * nz:
        raise ValueError('water_cluster: more waters than lattice sites')
    rng = np.random.default_rng(seed)
    local = _water_local()
    ids, xyz = [], []
    for k in range(n):
        ix, iy, iz = k % nx, (k // nx) % ny, k // (nx * ny)
        site = SPACING * np.array([ix, iy, iz], dtype=np.float64)
        jit = rng.uniform(-JITTER, JITTER, size=3)
        rot = _rotation(rng.uniform(0.0, 1.0, size=3))
        for a, z in enumerate((8, 1, 1)):
            ids.append(z)
            xyz.append(site + jit + rot @ local[a])
    return Molecule(ids, np.array(xyz), 'angstrom')


def random_density(nao, nocc, seed):
    """D = C C^T, C = Q of QR(N(0,1)^{nao x nocc}), FP64."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((nao, nocc))
    q, _ = np.linalg.qr(c)
    return q @ q.T


def batch_clusters(count=256, nmax=16, seed=7, lattice=(3, 3, 2)):
    """``count`` independent water clusters for batched builds: cluster i has
    n_i ~ U{1..nmax} waters on the first n_i sites of ``lattice`` (x fastest)
    and geometry seed ``seed + 1 + i``; returns (molecules, n_i list)."""
    if nmax > lattice[0] * lattice[1] * lattice[2]:
        raise ValueError('batch_clusters: lattice too small for nmax')
    rng = np.random.default_rng(seed)
    ns = [int(v) for v in rng.integers(1, nmax + 1, size=count)]
    return [water_cluster(lattice, seed + 1 + i, n) for i, n in enumerate(ns)], ns


# Named workloads (lattice, seed).
CLUSTERS = {
    'h2o4': ((2, 2, 1), 1),
    'h2o8': ((2, 2, 2), 1),     # small profiling case
    'h2o32': ((4, 4, 2), 1),
    'h2o64': ((4, 4, 4), 1),
}
