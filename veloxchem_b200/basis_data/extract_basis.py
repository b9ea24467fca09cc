"""Regenerates the basis-set data files shipped in this directory.

The GPU host has no copy of the reference checkout, so the few basis sets the
Fock-build tests and workloads need (elements H..Ne) are converted once from the
reference's plain-text basis library (``basis/<NAME>``, format read by
``src/pymodule/molecularbasis.py:112-169``: ``@ATOMBASIS X`` blocks with
``<L> <nprim> 1`` shell titles followed by ``exponent coefficient`` lines) into
JSON.  Coefficients are stored raw; normalisation happens at load time exactly
as the reference does it (``CBasisFunction::normalize``).

Usage (in a checkout that has the reference):
    python veloxchem_b200/basis_data/extract_basis.py /path/to/reference/basis
"""

import json
import os
import sys
from pathlib import Path

BASIS_SETS = ['STO-3G', 'DEF2-SVP', 'DEF2-SVPD', 'DEF2-TZVP', 'AO-START-GUESS']
ELEMENTS = ['H', 'HE', 'LI', 'BE', 'B', 'C', 'N', 'O', 'F', 'NE']
ANGL = {'S': 0, 'P': 1, 'D': 2, 'F': 3, 'G': 4, 'H': 5, 'I': 6}


def parse_basis_file(path):
    atoms = {}
    lines = Path(path).read_text().splitlines()
    i = 0
    while i < len(lines):
        line = lines[i].strip()
        if line.startswith('@ATOMBASIS'):
            elem = line.split()[1].upper()
            shells = []
            i += 1
            while not lines[i].strip().startswith('@END'):
                title = lines[i].split()
                i += 1
                if not title:
                    continue
                if title[0] == 'ECP':
                    continue
                lval = ANGL[title[0].upper()]
                nprim = int(title[1])
                exps, coefs = [], []
                for _ in range(nprim):
                    e, c = lines[i].split()[:2]
                    exps.append(float(e))
                    coefs.append(float(c))
                    i += 1
                shells.append([lval, exps, coefs])
            atoms[elem] = shells
        i += 1
    return atoms


def reference_dir():
    """The reference checkout: $VLX_REFERENCE_DIR, else a directory named
    ``reference`` next to this repository."""
    env = os.environ.get('VLX_REFERENCE_DIR')
    ref = Path(env) if env else Path(__file__).resolve().parents[3] / 'reference'
    if not (ref / 'basis').is_dir():
        raise SystemExit('reference checkout not found at %s: set VLX_REFERENCE_DIR' % ref)
    return ref


def main():
    src = Path(sys.argv[1]) if len(sys.argv) > 1 else reference_dir() / 'basis'
    out = Path(__file__).parent
    for name in BASIS_SETS:
        atoms = parse_basis_file(src / name)
        data = {e: atoms[e] for e in ELEMENTS if e in atoms}
        (out / (name.lower() + '.json')).write_text(json.dumps(data, indent=0))
        print(name, sorted(data))


if __name__ == '__main__':
    main()
