"""Writes h2o64_tzvp_jk.npz: a compact fixture of the reference FockDriver's
J and K for the seeded (H2O)_64 / def2-TZVP workload (2,752 functions,
ithreshold 12), so that the GPU build can be checked against the reference at
that size without re-running the reference (about 20 min per label on 8 host
cores).

Inputs: ``water_cluster((4, 4, 4), 1)``, def2-TZVP, D = ``random_density(nao,
320, 1)`` (symmetric).  The reference is the compiled oracle
(oracle/_ref/libvlxref.so, built by oracle/Makefile from the reference
sources), called with labels "j" and "k", exchange factor 1, omega 0.

Stored: checksums of D (to detect a drift of the density generator), the
per-row max |J| and |K|, and full rows of J and K for 48 seeded row indices.

    python tests/golden/make_c3_fixture.py [threads]
"""

import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

LATTICE, SEED, NOCC, ITH, NROWS = (4, 4, 4), 1, 320, 12, 48


def density_checksums(d):
    return np.array([d.sum(), (d * d).sum(), np.abs(d).max(), d.trace()])


def rows_of(nao):
    return np.sort(np.random.default_rng(2024).choice(nao, size=NROWS, replace=False))


def main():
    from oracle.oracle import RefOracle
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200.geometry import random_density, water_cluster
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 4)
    mol = water_cluster(LATTICE, SEED)
    bas = MolecularBasis.read(mol, 'def2-tzvp')
    nao = bas.get_dimensions_of_basis()
    d = random_density(nao, NOCC, SEED)
    RefOracle.set_threads(threads)
    ref = RefOracle(mol, bas)
    out = {}
    for label in ('j', 'k'):
        t0 = time.time()
        m = ref.fock(d, label, 1.0, 0.0, ITH, True)
        print('%s: %.1f s on %d threads' % (label, time.time() - t0, threads), flush=True)
        out[label] = m
    rows = rows_of(nao)
    np.savez_compressed(HERE / 'h2o64_tzvp_jk.npz', lattice=np.array(LATTICE), seed=SEED, nocc=NOCC,
                        ithreshold=ITH, basis='def2-tzvp', nao=nao, d_checksums=density_checksums(d),
                        rows=rows, j_rows=out['j'][rows], k_rows=out['k'][rows],
                        j_rowmax=np.abs(out['j']).max(axis=1), k_rowmax=np.abs(out['k']).max(axis=1),
                        threads=threads)


if __name__ == '__main__':
    main()
