"""Regenerates the golden fixtures in this directory (run where the reference
checkout and the compiled reference oracle are available).

* ``h2o_sto3g.npz``, ``h2o_dimer_svpd.npz``, ``h2o_dimer_tzvp.npz``: the
  reference's own golden J/K/ERI matrices and densities (its tests/data/*.npy,
  used by tests/test_fock_driver.py, test_fock_eri.py) plus the test molecules'
  geometries (tests/test_fock_driver.py:16-56), repacked as npz.
* ``screener_sto3g.json``: the known-answer max (ab|ab) values per pair block
  of tests/test_t4c_screener.py:47-67 (read from that file as text).
* ``h2o4_svp.npz``: the (H2O)_4 / def2-SVP workload (96 functions) with its
  seeded random density, and J, K, 2J-K at ithreshold 12 from the reference
  FockDriver compiled from source (oracle/_ref/libvlxref.so).

    python tests/golden/make_golden.py [/path/to/reference]   (default: $VLX_REFERENCE_DIR)
"""

import json
import os
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

H2O = """
O    0.000000000000        0.000000000000        0.000000000000
H    0.000000000000        0.740848095288        0.582094932012
H    0.000000000000       -0.740848095288        0.582094932012
"""

H2O_DIMER = """
O -1.464  0.099  0.300
H -1.956  0.624 -0.340
H -1.797 -0.799  0.206
O  1.369  0.146 -0.395
H  1.894  0.486  0.335
H  0.451  0.163 -0.083
"""


def _geom(text):
    ids, xyz = [], []
    for line in text.strip().splitlines():
        p = line.split()
        ids.append({'O': 8, 'H': 1}[p[0]])
        xyz.append([float(v) for v in p[1:4]])
    return np.array(ids, dtype=np.int32), np.array(xyz)


def reference_dir():
    """The reference checkout: $VLX_REFERENCE_DIR, else a directory named
    ``reference`` next to this repository."""
    env = os.environ.get('VLX_REFERENCE_DIR')
    ref = Path(env) if env else HERE.parents[2] / 'reference'
    if not (ref / 'tests' / 'data').is_dir():
        raise SystemExit('reference checkout not found at %s: set VLX_REFERENCE_DIR' % ref)
    return ref


def main():
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else reference_dir()
    data = ref / 'tests' / 'data'

    z, xyz = _geom(H2O)
    np.savez_compressed(HERE / 'h2o_sto3g.npz', z=z, xyz_angstrom=xyz, basis='STO-3G',
                        density=np.load(data / 'h2o.sto3g.density.npy'),
                        j=np.load(data / 'h2o.sto3g.j.npy'), k=np.load(data / 'h2o.sto3g.k.npy'),
                        eri=np.load(data / 'h2o.sto3g.eri.npy'))
    z, xyz = _geom(H2O_DIMER)
    np.savez_compressed(HERE / 'h2o_dimer_svpd.npz', z=z, xyz_angstrom=xyz, basis='DEF2-SVPD',
                        density=np.load(data / 'h2o.dimer.svpd.density.npy'),
                        density_gen=np.load(data / 'h2o.dimer.svpd.density.gen.npy'),
                        j=np.load(data / 'h2o.dimer.svpd.j.npy'), k=np.load(data / 'h2o.dimer.svpd.k.npy'),
                        j_gen=np.load(data / 'h2o.dimer.svpd.j.gen.npy'),
                        k_gen=np.load(data / 'h2o.dimer.svpd.k.gen.npy'))
    np.savez_compressed(HERE / 'h2o_dimer_tzvp.npz', z=z, xyz_angstrom=xyz, basis='DEF2-TZVP',
                        density=np.load(data / 'h2o.dimer.tzvp.density.npy'),
                        j=np.load(data / 'h2o.dimer.tzvp.j.npy'), k=np.load(data / 'h2o.dimer.tzvp.k.npy'),
                        erf_k=np.load(data / 'h2o.dimer.tzvp.erf.k.npy'))

    # screener known answers, read from the reference test as text
    text = (ref / 'tests' / 'test_t4c_screener.py').read_text()
    kat = {}
    for name in ('tints_ss', 'tints_sp', 'tints_pp'):
        body = re.search(name + r'\s*=\s*\[(.*?)\]', text, re.S).group(1)
        kat[name[6:]] = [float(v) for v in body.replace('\n', ' ').split(',') if v.strip()]
    (HERE / 'screener_sto3g.json').write_text(json.dumps(kat, indent=1))

    # (H2O)_4 / def2-SVP from the compiled reference
    from oracle.oracle import RefOracle
    from veloxchem_b200.geometry import CLUSTERS, random_density, water_cluster
    from veloxchem_b200.molecularbasis import MolecularBasis
    lattice, seed = CLUSTERS['h2o4']
    mol = water_cluster(lattice, seed)
    bas = MolecularBasis.read(mol, 'def2-svp')
    orc = RefOracle(mol, bas)
    nao = orc.nao
    dens = random_density(nao, 5 * 4, seed)
    out = {}
    for lab in ('j', 'k', '2jk'):
        out[lab.replace('2jk', 'f2jk')] = orc.fock(dens, lab, 1.0, 0.0, 12)
    np.savez_compressed(HERE / 'h2o4_svp.npz', z=mol.get_element_ids(), xyz_bohr=mol.get_coordinates_in_bohr(),
                        basis='DEF2-SVP', ithreshold=12, density=dens, **out)
    print('nao', nao)


if __name__ == '__main__':
    main()
