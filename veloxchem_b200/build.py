"""Builds the native library veloxchem_b200/lib/libvlx_b200.so for sm_100a.

Steps: generate the per-class recursions (csrc/gen_eri.py) into csrc/_gen,
compile every translation unit with nvcc in parallel (incremental: a unit is
rebuilt when its source or any shared header changed), embed the warp-cooperative
program blob, link one shared library with the static CUDA runtime.

    python -m veloxchem_b200.build [--jobs N] [--lmax 3]
"""

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / 'csrc'
GEN = CSRC / '_gen'
OBJ = CSRC / '_build'
LIB = PKG / 'lib' / 'libvlx_b200.so'
INCLUDE = PKG.parent / 'include'

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ARCH + ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
                     '-I' + str(CSRC), '-I' + str(GEN), '-I' + str(INCLUDE)]


def nvcc():
    exe = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    return exe


def _headers_digest(abi=False):
    """Digest of the headers a unit may include: the device headers for every
    unit, plus the public C header (abi=True) for the units that include it
    (the host orchestration and the guess-network kernels; the per-class
    units do not)."""
    h = hashlib.sha256()
    files = list(CSRC.glob('*.cuh')) + list(CSRC.glob('*.h')) + \
        [GEN / 'dispatch.inc', GEN / 'sph_table.inc', GEN / 'xform.inc', GEN / 'coop_classes.inc']
    if abi:
        files.append(INCLUDE / 'vlx_b200.h')
    for p in sorted(files):
        if p.exists():
            h.update(p.read_bytes())
    # flags with the tree's own location left out, so that a copy of the tree
    # keeps its objects
    h.update(' '.join(f.replace(str(PKG.parent), '<root>') for f in NVCC_FLAGS).encode())
    return h.hexdigest()[:16]


def _compile(src, obj, hdr):
    stamp = obj.with_suffix('.stamp')
    key = hdr + hashlib.sha256(src.read_bytes()).hexdigest()[:16]
    if obj.exists() and stamp.exists() and stamp.read_text() == key:
        return src.name, 0.0, False
    cmd = [nvcc()] + NVCC_FLAGS + ['-c', str(src), '-o', str(obj)]
    import time
    t0 = time.time()
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError('nvcc failed for %s:\n%s\n%s' % (src.name, res.stdout, res.stderr))
    stamp.write_text(key)
    return src.name, time.time() - t0, True


def build(jobs=None, lmax=3, verbose=True):
    GEN.mkdir(parents=True, exist_ok=True)
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    sys.path.insert(0, str(CSRC))
    import gen_eri
    sys.argv = ['gen_eri.py', str(GEN), str(lmax)]
    gen_eri.main()
    blob = GEN / 'coop_programs.bin'
    asm = GEN / 'vlx_blob.S'
    asm_text = ('    .section .rodata\n    .global vlx_coop_blob_start\n    .global vlx_coop_blob_end\n'
                '    .balign 16\nvlx_coop_blob_start:\n    .incbin "%s"\nvlx_coop_blob_end:\n'
                '    .byte 0\n    .section .note.GNU-stack,"",@progbits\n' % blob)
    if not asm.exists() or asm.read_text() != asm_text:
        asm.write_text(asm_text)
    hdr, hdr_abi = _headers_digest(), _headers_digest(abi=True)
    abi_units = {'vlx_host', 'vlx_mlp', 'vlx_onee', 'vlx_coop'}
    sources = sorted(GEN.glob('class_*.cu')) + [CSRC / 'vlx_coop.cu', CSRC / 'vlx_onee.cu', CSRC / 'vlx_mlp.cu',
                                                CSRC / 'vlx_host.cu']
    objs = [OBJ / (s.stem + '.o') for s in sources]
    jobs = jobs or os.cpu_count() or 4
    # the longest units first, so that they do not finish last on one core
    order = sorted(range(len(sources)), key=lambda k: -sources[k].stat().st_size)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, sources[k], objs[k], hdr_abi if sources[k].stem in abi_units else hdr)
                for k in order]
        for f in cf.as_completed(futs):
            name, dt, built = f.result()
            if verbose and built:
                print('  nvcc %-22s %6.1fs' % (name, dt), flush=True)
    blob_obj = OBJ / 'vlx_blob.o'
    blob_key = hashlib.sha256(blob.read_bytes() + asm_text.encode()).hexdigest()[:16]
    blob_stamp = OBJ / 'vlx_blob.stamp'
    if not blob_obj.exists() or not blob_stamp.exists() or blob_stamp.read_text() != blob_key:
        subprocess.run(['gcc', '-c', str(asm), '-o', str(blob_obj)], check=True)
        blob_stamp.write_text(blob_key)
    # only the objects of the current class list are linked
    link = [nvcc()] + ARCH + ['-shared', '-o', str(LIB)] + [str(o) for o in objs] + [str(blob_obj)]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError('link failed:\n%s\n%s' % (res.stdout, res.stderr))
    if verbose:
        print('built', LIB, '%.1f MB' % (LIB.stat().st_size / 1e6))
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--jobs', type=int, default=None)
    ap.add_argument('--lmax', type=int, default=3)
    args = ap.parse_args()
    build(args.jobs, args.lmax)


if __name__ == '__main__':
    main()
