"""Measurement workloads beyond the single-build bench line.

    python -m veloxchem_b200.workloads c3 [--out FILE]     # (H2O)64 / def2-TZVP builds and SCF
    python -m veloxchem_b200.workloads c4 [--out FILE]     # 256 small clusters, batched builds
    python -m veloxchem_b200.workloads c2scf [--out FILE]  # (H2O)32 / def2-SVP SCF, plain and mixed
    python -m veloxchem_b200.workloads c3h / c4h           # the north-star comparison (bench.py's north_star)
    python -m veloxchem_b200.workloads build|onee|guess --cluster NAME [--basis B] [--repeat N]

Each prints one JSON object (and writes it to --out).  Times are CUDA-event
device times for builds and wall-clock times for SCF runs (which include the
host-side linear algebra and synchronisation of the driver).
"""

import argparse
import json
import time

import numpy as np


def _torch():
    import torch
    return torch


def _cluster(name, basis):
    from . import MolecularBasis
    from .geometry import CLUSTERS, water_cluster
    lat, seed = CLUSTERS[name]
    mol = water_cluster(lat, seed)
    return mol, MolecularBasis.read(mol, basis)


def _build_ms(scr, d, f, reps=3, enqueue=None):
    """Device time (ms, best of reps) of one 2J-K build at ithreshold 12;
    enqueue (a list) receives the host time of each call, which returns once
    all the build's launches are enqueued."""
    import ctypes
    from . import _native as nat
    torch = _torch()
    st = torch.cuda.Stream()
    best = 1e30
    with torch.cuda.stream(st):
        for _ in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            t0 = time.perf_counter()
            nat.check(nat.lib().vlx_b200_fock_build_device(scr.handle, ctypes.c_void_p(d.data_ptr()), 1, b'2jk', 1.0,
                                                            0.0, 12, ctypes.c_void_p(f.data_ptr()),
                                                            ctypes.c_void_p(st.cuda_stream)), 'fock_build')
            if enqueue is not None:
                enqueue.append(1e3 * (time.perf_counter() - t0))
            e1.record(st)
            st.synchronize()
            best = min(best, e0.elapsed_time(e1))
    return best


def c3(cutoffs=(1e-9, 1e-8, 1e-7, 1e-6, 1e-5), scf=True, variants=None, builds=True, autotune=False,
       density_screening=None):
    """(H2O)64 / def2-TZVP builds, per-class profile (every class), the mixed
    cutoffs and the SCF variants.  density_screening = (fp32_cutoff,
    skip_cutoff): profile the density-screened kernels instead of the plain
    ones (vlx_b200_set_density_screening)."""
    from . import T4CScreener
    from . import _native as nat
    from .geometry import random_density
    from .scf import ScfRestrictedDriver
    torch = _torch()
    mol, bas = _cluster('h2o64', 'def2-tzvp')
    scr = T4CScreener()
    scr.partition(bas, mol, 'eri')
    d = torch.from_numpy(random_density(scr.nao, 320, 1)).cuda()
    f64 = torch.empty_like(d)
    out = {'workload': '(H2O)64 / def2-TZVP, 2J-K, ithreshold 12', 'nao': scr.nao}
    if not builds:
        cutoffs = ()
    if autotune:
        out['fp64_build_ms_untuned'] = _build_ms(scr, d, torch.empty_like(d), reps=1)
        t0 = time.perf_counter()
        out['autotune'] = nat.autotune(scr, d.data_ptr(), 12)
        out['autotune_s'] = time.perf_counter() - t0
    if density_screening is not None:
        scr.set_density_screening(*density_screening)
        out['density_screening'] = list(density_screening)
    t64 = _build_ms(scr, d, f64, reps=3 if builds else 0)
    prof = nat.fock_profile(scr, d.data_ptr(), f64.data_ptr(), '2jk', 1.0, 12)
    flops = sum(p['flops'] for p in prof)
    out['fp64'] = {'build_ms': t64, 'flops': flops, 'tflops': flops / t64 / 1e9,
                   'classes': sorted([{'cls': '%d%d%d%d' % (p['la'], p['lb'], p['lc'], p['ld']),
                                       'table_driven': p['table_driven'], 'ms': p['device_ms'],
                                       'quartets': p['shell_quartets'], 'prim_quartets': p['prim_quartets'],
                                       'tflops': p['flops'] / max(p['device_ms'], 1e-9) / 1e9} for p in prof],
                                     key=lambda r: -r['ms'])}
    dmax = float(d.abs().max())
    out['mixed'] = []
    for cut in cutoffs:
        scr.set_fp32_threshold(cut, dmax)
        fm = torch.empty_like(d)
        tm = _build_ms(scr, d, fm)
        prof = nat.fock_profile(scr, d.data_ptr(), fm.data_ptr(), '2jk', 1.0, 12)
        n32 = sum(p['fp32_quartets'] for p in prof)
        nq = sum(p['shell_quartets'] for p in prof)
        out['mixed'].append({'cutoff': cut, 'build_ms': tm, 'speedup': t64 / tm, 'fp32_share': n32 / max(nq, 1),
                             'max_abs_fock_error': float((fm - f64).abs().max()),
                             'class_ms': {'%d%d%d%d' % (p['la'], p['lb'], p['lc'], p['ld']): p['device_ms']
                                          for p in prof}})
    scr.set_fp32_threshold(0.0, 0.0)
    if scf:
        runs = {}
        # plain: FP64 builds from the full density every iteration, SAD guess
        for name, cut, guess, inc, early in (('plain_fp64_sad', 0.0, 'sad', False, None),
                                             ('fp64_sad_incremental', 0.0, 'sad', True, None),
                                             ('mixed_1e-6_sad', 1e-6, 'sad', False, None),
                                             ('fp64_learned', 0.0, 'learned', False, None),
                                             ('mixed_learned_incremental', 1e-6, 'learned', True, None),
                                             ('mixed_learned_incremental_early8', 1e-6, 'learned', True, 8)):
            if variants and name not in variants:
                continue
            drv = ScfRestrictedDriver()
            drv.fp32_cutoff = cut
            drv.guess = guess
            drv.incremental = inc
            drv.early_ithreshold = early
            t0 = time.perf_counter()
            res = drv.compute(mol, bas, screener=scr)
            runs[name] = {'energy': res['scf_energy'], 'iterations': res['iterations'],
                          'converged': res['converged'], 'wall_s': time.perf_counter() - t0,
                          'fock_ms_total': res['timings']['fock_ms_total'], 'guess_used': res['guess_used'],
                          'timings': {k: v for k, v in res['timings'].items() if isinstance(v, float)},
                          'history': [(h['iteration'], h['energy'], h['e_grad'], h['time_s'], h['mixed'],
                                       h['ithreshold'], h['incremental']) for h in res['history']]}
        # E_ref: the plain FP64 run (or, if it was not run, the last variant's energy)
        e_ref = runs['plain_fp64_sad']['energy'] if 'plain_fp64_sad' in runs else list(runs.values())[-1]['energy']
        for r in runs.values():
            r['energy_error'] = r['energy'] - e_ref
            r['time_to_1e-6_s'] = next((h[3] for k, h in enumerate(r['history'])
                                        if all(abs(x[1] - e_ref) < 1e-6 for x in r['history'][k:])), None)
        out['scf'] = runs
    return out


def c4(count=256, nmax=16, reps=5):
    from . import MolecularBasis, T4CScreener
    from .batch import FockBatch
    from .geometry import batch_clusters, random_density
    torch = _torch()
    mols, ns = batch_clusters(count, nmax, 7)
    scrs, dens = [], []
    for i, (m, n) in enumerate(zip(mols, ns)):
        b = MolecularBasis.read(m, 'def2-svp')
        s = T4CScreener()
        s.partition(b, m, 'eri')
        scrs.append(s)
        dens.append(random_density(s.nao, 5 * n, 1000 + i))
    batch = FockBatch(scrs)
    d = torch.from_numpy(batch.pack(dens)).cuda()
    f = torch.empty_like(d)
    st = torch.cuda.Stream()
    res = {'workload': '%d water clusters, n ~ U{1..%d}, def2-SVP, 2J-K, ithreshold 12' % (count, nmax),
           'nao_total': int(sum(s.nao for s in scrs)), 'nao_range': [min(s.nao for s in scrs),
                                                                    max(s.nao for s in scrs)]}
    with torch.cuda.stream(st):
        for graph in (True, False):
            batch.build_device(d, f, stream=st, use_graph=graph)
            st.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                batch.build_device(d, f, stream=st, use_graph=graph)
            e1.record(st)
            st.synchronize()
            ms = e0.elapsed_time(e1) / reps
            res['batched_graph' if graph else 'batched_nograph'] = {
                'ms_per_batch': ms, 'builds_per_s': count / (ms * 1e-3),
                'kernel_launches': batch.last_stats['kernel_launches']}
        # one molecule per call through the single-molecule entry point
        import ctypes
        from . import _native as nat
        fs = [torch.empty((s.nao, s.nao), dtype=torch.float64, device='cuda') for s in scrs]
        ds = [d[batch.offsets[k]:batch.offsets[k + 1]].view(s.nao, s.nao) for k, s in enumerate(scrs)]
        for k, s in enumerate(scrs):  # work lists
            nat.check(nat.lib().vlx_b200_fock_build_device(s.handle, ctypes.c_void_p(ds[k].data_ptr()), 1, b'2jk',
                                                            1.0, 0.0, 12, ctypes.c_void_p(fs[k].data_ptr()),
                                                            ctypes.c_void_p(st.cuda_stream)), 'fock_build')
        st.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for k, s in enumerate(scrs):
            nat.check(nat.lib().vlx_b200_fock_build_device(s.handle, ctypes.c_void_p(ds[k].data_ptr()), 1, b'2jk',
                                                            1.0, 0.0, 12, ctypes.c_void_p(fs[k].data_ptr()),
                                                            ctypes.c_void_p(st.cuda_stream)), 'fock_build')
        e1.record(st)
        st.synchronize()
        ms = e0.elapsed_time(e1)
        res['one_per_call'] = {'ms_per_batch': ms, 'builds_per_s': count / (ms * 1e-3)}
    err = max(float((f[batch.offsets[k]:batch.offsets[k + 1]].view(s.nao, s.nao) - fs[k]).abs().max())
              for k, s in enumerate(scrs))
    res['max_abs_error_vs_single'] = err
    return res


def c2scf(conv=1e-8):
    """(H2O)32 / def2-SVP RHF from SAD to an electronic gradient (DIIS error)
    of `conv`: plain FP64 with the reference's C2-DIIS and with Pulay DIIS,
    then the mixed / incremental / early variants (C2-DIIS); per run the
    iterations, wall time, Fock-build time, iterations to a 1e-6 gradient and
    the energy error against the plain run."""
    from .scf import ScfRestrictedDriver
    mol, bas = _cluster('h2o32', 'def2-svp')
    runs = {}
    for name, cut, inc, early, acc in (('warmup', 0.0, False, None, 'c2diis'),
                                       ('plain_fp64', 0.0, False, None, 'c2diis'),
                                       ('plain_fp64_pulay', 0.0, False, None, 'diis'),
                                       ('mixed_1e-4', 1e-4, False, None, 'c2diis'),
                                       ('fp64_incremental', 0.0, True, None, 'c2diis'),
                                       ('mixed_incremental', 1e-4, True, None, 'c2diis'),
                                       ('mixed_incremental_early8', 1e-4, True, 8, 'c2diis')):
        drv = ScfRestrictedDriver()
        drv.conv_thresh = conv
        drv.max_iter = 80
        drv.fp32_cutoff = cut
        drv.incremental = inc
        drv.early_ithreshold = early
        drv.acc_type = acc
        if inc:
            drv.full_skip_factor = 1e-2
            drv.early_skip_factor = 1e-1
        t0 = time.perf_counter()
        res = drv.compute(mol, bas)
        if name == 'warmup':
            continue
        hist = res['history']
        runs[name] = {'energy': res['scf_energy'], 'converged': res['converged'], 'iterations': res['iterations'],
                      'iterations_to_grad_1e-6': next((h['iteration'] for h in hist if h['e_grad'] < 1e-6), None),
                      'wall_s': time.perf_counter() - t0, 'fock_ms_total': res['timings']['fock_ms_total']}
    for k in runs:
        runs[k]['energy_error'] = runs[k]['energy'] - runs['plain_fp64']['energy']
    return {'workload': '(H2O)32 / def2-SVP RHF from SAD, electronic gradient < %g' % conv, **runs}


def build(cluster, basis, repeat=1, fp32_cutoff=0.0):
    """Screener + `repeat` plain builds of a named cluster (the command the
    profiles under profiles/ are taken on)."""
    from . import T4CScreener
    from .geometry import random_density
    torch = _torch()
    mol, bas = _cluster(cluster, basis)
    scr = T4CScreener()
    scr.partition(bas, mol, 'eri')
    d = torch.from_numpy(random_density(scr.nao, 5 * mol.number_of_atoms() // 3, 1)).cuda()
    if fp32_cutoff > 0:
        scr.set_fp32_threshold(fp32_cutoff, float(d.abs().max()))
    f = torch.empty_like(d)
    ms = [_build_ms(scr, d, f, reps=0) for _ in range(repeat)]
    return {'workload': '%s / %s, 2J-K, ithreshold 12' % (cluster, basis), 'nao': scr.nao, 'build_ms': ms,
            'fp32_cutoff': fp32_cutoff}


def _time_to(history, e_ref, tol=1e-6):
    """Wall time (s) after which every later iteration's energy stays within
    tol of e_ref, from an SCF history (None if it never does)."""
    for k, h in enumerate(history):
        if all(abs(x['energy'] - e_ref) < tol for x in history[k:]):
            return h['time_s']
    return None


def _warm_fast_path(scr, d):
    """One-time per-process costs of the fast SCF path, paid before either
    timed run (as the library load and the plain kernels' first launches are):
    the guess network (weights, first inference, on (H2O)_2) and the first
    launches of the density-screened kernel variants (one screened build of
    the workload's own density; the variants load lazily on first launch)."""
    from . import _native as nat
    from . import MolecularBasis
    from .geometry import water_cluster
    from .guess import learned_guess_driver
    mol = water_cluster((2, 1, 1), 3)
    bas = MolecularBasis.read(mol, 'def2-tzvp')
    learned_guess_driver().predict_any(mol, bas, nat.one_electron(0, mol, bas), mol.number_of_electrons() // 2)
    if scr is not None:
        torch = _torch()
        scr.set_density_screening(1e-4, 1e-10)
        _build_ms(scr, d, torch.empty_like(d), reps=0)
        scr.set_density_screening(0.0, 0.0)


def c3_headline(cutoffs=(1e-9, 1e-8, 1e-7, 1e-6, 1e-5, 1e-4), max_fock_error=1e-6, scf=True, log=None,
                full_skip_factor=1e-2, early_skip_factor=1e-1, fp32_cutoff=1e-4, acc_type='c2diis',
                full_fp32_digestion_cutoff=1e-6):
    """The north-star comparison on (H2O)64 / def2-TZVP in one process:

    * builds: the plain FP64 2J-K build (device ms, CUDA events, best of 2
      after one warm-up), then the mixed-precision build at each cutoff (one
      timed build each, FP32 share, max |F_mixed - F_FP64|); the chosen cutoff
      is the fastest one whose Fock error stays within ``max_fock_error``;
    * SCF: plain (FP64 full builds every iteration, SAD guess, electronic
      gradient 1e-6, whose final energy E_ref is the FP64 reference: the
      energy error at that gradient is far below 1e-9 Eh) against mixed
      (FP32 below fp32_cutoff while the gradient is above 1e-4, and in the
      incremental builds) + learned + incremental + early iterations with
      per-quartet density screening (gradient 1e-6), back to back on one
      screener, both with the accelerator acc_type; per run the wall time to
      |E - E_ref| < 1e-6 Eh for good, the time to its declared convergence,
      iterations and the final energy error."""
    from . import T4CScreener
    from . import _native as nat
    from .geometry import random_density
    from .scf import ScfRestrictedDriver
    torch = _torch()
    say = log or (lambda *a: None)
    mol, bas = _cluster('h2o64', 'def2-tzvp')
    t0 = time.perf_counter()
    scr = T4CScreener()
    scr.partition(bas, mol, 'eri')
    out = {'workload': '(H2O)64 / def2-TZVP, 2J-K, ithreshold 12', 'nao': scr.nao,
           'screener_s': time.perf_counter() - t0}
    d = torch.from_numpy(random_density(scr.nao, 320, 1)).cuda()
    f64 = torch.empty_like(d)
    enq = []
    t64 = _build_ms(scr, d, f64, reps=2, enqueue=enq)
    prof = nat.fock_profile(scr, d.data_ptr(), f64.data_ptr(), '2jk', 1.0, 12)
    flops = sum(p['flops'] for p in prof)
    out['fp64_build_ms'] = t64
    # host time to enqueue one build (work list cached): the launch overhead a
    # CUDA graph of the build would remove
    out['enqueue_ms'] = min(enq[1:]) if len(enq) > 1 else None
    out['kernel_launches_per_build'] = len(prof) + 1  # class kernels + symmetrisation
    out['fp64_tflops'] = flops / t64 / 1e9
    say('c3 fp64 build %.1f ms' % t64)
    dmax = float(d.abs().max())
    sweep = []
    for cut in cutoffs:
        scr.set_fp32_threshold(cut, dmax)
        fm = torch.empty_like(d)
        tm = _build_ms(scr, d, fm, reps=0)
        prof = nat.fock_profile(scr, d.data_ptr(), fm.data_ptr(), '2jk', 1.0, 12)
        n32 = sum(p['fp32_quartets'] for p in prof)
        nq = sum(p['shell_quartets'] for p in prof)
        sweep.append({'cutoff': cut, 'build_ms': tm, 'speedup': t64 / tm, 'fp32_share': n32 / max(nq, 1),
                      'max_abs_fock_error': float((fm - f64).abs().max())})
        say('c3 mixed %.0e: %.1f ms, err %.2e' % (cut, tm, sweep[-1]['max_abs_fock_error']))
    scr.set_fp32_threshold(0.0, 0.0)
    ok = [s for s in sweep if s['max_abs_fock_error'] <= max_fock_error] or sweep[:1]
    best = min(ok, key=lambda s: s['build_ms'])
    out['mixed_sweep'] = sweep
    out['mixed_chosen'] = best
    if scf:
        _warm_fast_path(scr, d)
        runs = {}
        for name, cut, guess, inc, early, conv in (('plain_fp64_sad', 0.0, 'sad', False, None, 1e-6),
                                                  ('mixed_learned_incremental_early', fp32_cutoff, 'learned',
                                                   True, 8, 1e-6)):
            drv = ScfRestrictedDriver()
            drv.fp32_cutoff = cut
            drv.guess = guess
            drv.incremental = inc
            drv.early_ithreshold = early
            drv.conv_thresh = conv
            drv.acc_type = acc_type
            if inc:
                drv.full_skip_factor = full_skip_factor
                drv.early_skip_factor = early_skip_factor
                drv.full_fp32_digestion_cutoff = full_fp32_digestion_cutoff
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = drv.compute(mol, bas, screener=scr)
            wall = time.perf_counter() - t0
            hist = [h for h in res['history']]
            t_conv6 = next((h['time_s'] for h in hist if h['e_grad'] < 1e-6 and not h.get('mixed')), None)
            runs[name] = {'energy': res['scf_energy'], 'iterations': res['iterations'], 'converged': res['converged'],
                          'conv_thresh': conv, 'wall_s': wall, 'fock_s': res['timings']['fock_ms_total'] / 1e3,
                          'timings': {k: v for k, v in res['timings'].items() if isinstance(v, float)},
                          'time_to_grad_1e-6_s': t_conv6, 'guess_used': res['guess_used'], '_history': hist}
            say('c3 scf %s: %d it, %.1f s' % (name, res['iterations'], wall))
        e_ref = runs['plain_fp64_sad']['energy']
        for r in runs.values():
            hist = r.pop('_history')
            r['energy_error'] = r['energy'] - e_ref
            r['time_to_1e-6_Eh_s'] = _time_to(hist, e_ref)
            # per iteration: time (s), |E - E_ref|, gradient, ithreshold, incremental, mixed
            r['history'] = [[round(h['time_s'], 3), float('%.3g' % abs(h['energy'] - e_ref)),
                             float('%.3g' % h['e_grad']), h['ithreshold'], int(h['incremental']),
                             int(h['mixed'])] for h in hist]
        out['scf'] = runs
        out['scf_reference_energy'] = e_ref
        p, m = runs['plain_fp64_sad'], runs['mixed_learned_incremental_early']
        out['scf_speedup_time_to_1e-6_Eh'] = ((p['time_to_1e-6_Eh_s'] / m['time_to_1e-6_Eh_s'])
                                              if p['time_to_1e-6_Eh_s'] and m['time_to_1e-6_Eh_s'] else None)
        out['scf_speedup_to_declared_convergence'] = (p['time_to_grad_1e-6_s'] / m['wall_s']
                                                      if p['time_to_grad_1e-6_s'] else None)
    return out


def c3scf_variants(variants, log=None):
    """(H2O)64 / def2-TZVP SCF: the plain FP64 run (C2-DIIS, E_ref, gradient
    1e-6) and fast variants given as dicts of ScfRestrictedDriver attributes on top of
    mixed 1e-4 + learned + incremental + early 8 with per-quartet density
    screening (full skip 1e-2, early skip 1e-1) and C2-DIIS; per run the time to
    |E - E_ref| < 1e-6 Eh for good, the wall time and the energy error."""
    from . import T4CScreener
    from .geometry import random_density
    from .scf import ScfRestrictedDriver
    torch = _torch()
    say = log or (lambda *a: None)
    mol, bas = _cluster('h2o64', 'def2-tzvp')
    scr = T4CScreener()
    scr.partition(bas, mol, 'eri')
    d = torch.from_numpy(random_density(scr.nao, 320, 1)).cuda()
    _build_ms(scr, d, torch.empty_like(d), reps=0)  # work list of threshold 12
    _warm_fast_path(scr, d)
    base = dict(fp32_cutoff=1e-4, guess='learned', incremental=True, early_ithreshold=8, full_skip_factor=1e-2,
                early_skip_factor=1e-1, acc_type='c2diis', full_fp32_digestion_cutoff=1e-6)
    out = {}
    for name, attrs in [('plain', dict(fp32_cutoff=0.0, guess='sad', incremental=False, acc_type='c2diis'))] + \
            list(variants):
        drv = ScfRestrictedDriver()
        for k, v in (attrs if name == 'plain' else {**base, **attrs}).items():
            setattr(drv, k, v)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = drv.compute(mol, bas, screener=scr)
        out[name] = {'attrs': attrs, 'wall_s': time.perf_counter() - t0, 'energy': res['scf_energy'],
                     'iterations': res['iterations'], 'converged': res['converged'], '_h': res['history'],
                     'timings': dict(drv.timings)}
        say('%s: %d it, %.1f s' % (name, res['iterations'], out[name]['wall_s']))
    e_ref = out['plain']['energy']
    for r in out.values():
        h = r.pop('_h')
        r['energy_error'] = r['energy'] - e_ref
        r['time_to_1e-6_Eh_s'] = _time_to(h, e_ref)
        r['history'] = [[round(x['time_s'], 3), float('%.3g' % abs(x['energy'] - e_ref)), x['ithreshold'],
                         int(x['incremental'])] for x in h]
    for r in out.values():
        r['speedup'] = (out['plain']['time_to_1e-6_Eh_s'] / r['time_to_1e-6_Eh_s']) if r['time_to_1e-6_Eh_s'] else None
    return out


def c4_headline(count=256, nmax=16, reps=3):
    """Batched builds/s of the 256-cluster workload (graph replay) and the
    one-molecule-per-call rate, device time."""
    r = c4(count, nmax, reps)
    return {'workload': r['workload'], 'nao_total': r['nao_total'],
            'batched_builds_per_s': r['batched_graph']['builds_per_s'],
            'batched_ms': r['batched_graph']['ms_per_batch'],
            'one_per_call_builds_per_s': r['one_per_call']['builds_per_s'],
            'max_abs_error_vs_single': r['max_abs_error_vs_single']}


def onee(cluster, basis, repeat=1):
    """Overlap, kinetic and nuclear-attraction matrices of a named cluster
    (the SCF's one-electron integrals), `repeat` times; wall seconds each."""
    from . import _native as nat
    mol, bas = _cluster(cluster, basis)
    times = []
    for _ in range(repeat):
        t0 = time.perf_counter()
        for which in range(3):
            nat.one_electron(which, mol, bas)
        times.append(time.perf_counter() - t0)
    return {'workload': '%s / %s S, T, V' % (cluster, basis), 'nao': bas.get_dimensions_of_basis(), 'seconds': times}


def guess(cluster, repeat=1):
    """Learned-guess inference (descriptors, BF16 network on the tensor
    cores, assembly, idempotent projection) for a named def2-SVP cluster."""
    from . import _native as nat
    from .guess import learned_guess_driver
    from .scf import SadGuessDriver
    from . import MolecularBasis
    mol, bas = _cluster(cluster, 'def2-svp')
    S = nat.one_electron(0, mol, bas)
    sad = SadGuessDriver().compute(mol, MolecularBasis.read(mol, 'ao-start-guess'), bas, overlap=S)
    drv = learned_guess_driver()
    nocc = mol.number_of_electrons() // 2
    times = []
    for _ in range(repeat):
        t0 = time.perf_counter()
        drv.predict(mol, bas, sad, S, nocc)
        times.append(time.perf_counter() - t0)
    return {'workload': '%s / def2-SVP learned guess' % cluster, 'seconds': times}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('which', choices=['c3', 'c4', 'c2scf', 'build', 'c3h', 'c4h', 'c3scf', 'onee', 'guess'])
    ap.add_argument('--out', default=None)
    ap.add_argument('--no-scf', action='store_true')
    ap.add_argument('--cluster', default='h2o64')
    ap.add_argument('--basis', default='def2-tzvp')
    ap.add_argument('--repeat', type=int, default=1)
    ap.add_argument('--fp32-cutoff', type=float, default=0.0)
    ap.add_argument('--scf-variants', default=None, help='comma-separated subset of the C3 SCF variants')
    ap.add_argument('--no-builds', action='store_true', help='C3: skip the per-cutoff build table')
    ap.add_argument('--autotune', action='store_true', help='C3: autotune the classes first')
    ap.add_argument('--density-screening', type=float, nargs=2, default=None, metavar=('FP32', 'SKIP'),
                    help='C3: profile the density-screened kernels with these cutoffs')
    a = ap.parse_args(argv)
    if a.which == 'build':
        res = build(a.cluster, a.basis, a.repeat, a.fp32_cutoff)
    elif a.which == 'c3h':
        import sys
        res = c3_headline(cutoffs=(1e-5,) if a.no_builds else (1e-9, 1e-8, 1e-7, 1e-6, 1e-5), scf=not a.no_scf,
                          log=lambda m: print(m, file=sys.stderr, flush=True))
    elif a.which == 'c4h':
        res = c4_headline()
    elif a.which == 'c3scf':
        import sys
        res = c3scf_variants([('fast', {}),
                              ('fast_fp64_full_digestion', dict(full_fp32_digestion_cutoff=None)),
                              ('fast_full_fp32_digestion_1e-5', dict(full_fp32_digestion_cutoff=1e-5))],
                             log=lambda m: print(m, file=sys.stderr, flush=True))
    elif a.which == 'onee':
        res = onee(a.cluster, a.basis, a.repeat)
    elif a.which == 'guess':
        res = guess(a.cluster, a.repeat)
    else:
        res = (c3(scf=not a.no_scf, variants=a.scf_variants.split(',') if a.scf_variants else None,
                  builds=not a.no_builds, autotune=a.autotune, density_screening=a.density_screening)
               if a.which == 'c3'
               else (c4() if a.which == 'c4' else c2scf()))
    text = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, 'w') as fh:
            fh.write(text)
    print(text)


if __name__ == '__main__':
    main()
