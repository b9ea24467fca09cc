"""Benchmark of the B200 Fock build.

One step = one restricted 2J-K Fock build (label "2jk", ithreshold 12, i.e.
Schwarz 1e-12) of a seeded (H2O)_32 / def2-SVP cluster (768 spherical basis
functions) with a seeded random closed-shell FP64 density, inputs resident on
the GPU.  The metric is Fock builds per second (whole job).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torch.distributed.run, one rank per GPU: the ranks shard the
one build (cost-balanced work items per rank, vlx_b200_set_partition) and sum
their FP64 partial Fock matrices with one NCCL all-reduce inside the step
(strong scaling); the timing takes the max over ranks.

At N = 1 the line also carries ``north_star``: the (H2O)64 / def2-TZVP build
(FP64 and mixed precision per cutoff), the SCF time to 1e-6 Eh of the plain
FP64 path against mixed + learned + incremental builds on the same screener,
and the 256-cluster batched builds/s (--no-north-star skips it).

--impl reference times the reference's own FockDriver (compiled from source,
oracle/_ref/libvlxref.so) on the host cores with all threads, on rank 0: one
full build per step.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = 'h2o32'
BASIS = 'def2-svp'
ITHRESHOLD = 12
METRIC = 'fock_builds_per_s'
UNIT = 'builds/s'


def _env():
    return int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1)), int(os.environ.get('LOCAL_RANK', 0))


def _system(rank):
    from veloxchem_b200 import MolecularBasis
    from veloxchem_b200.geometry import CLUSTERS, random_density, water_cluster
    lattice, seed = CLUSTERS[WORKLOAD]
    mol = water_cluster(lattice, seed + rank)
    bas = MolecularBasis.read(mol, BASIS)
    nw = mol.number_of_atoms() // 3
    dens = random_density(bas.get_dimensions_of_basis(), 5 * nw, seed + rank)
    return mol, bas, dens


def _config(extra=None):
    lattice, seed = __import__('veloxchem_b200.geometry', fromlist=['CLUSTERS']).CLUSTERS[WORKLOAD]
    cfg = {'workload': '(H2O)_32 / def2-SVP restricted 2J-K Fock build, 768 functions, ithreshold 12',
           'molecule': 'seeded water cluster %dx%dx%d lattice, 3.0 A spacing, seed %d + rank' % (lattice + (seed,)),
           'basis': BASIS, 'label': '2jk', 'ithreshold': ITHRESHOLD,
           'density': 'C C^T, C = Q(QR(N(0,1)^{768x160})), FP64',
           'l2': 'L2 flushed between timed steps (256 MB write, outside the per-step events)'}
    if extra:
        cfg.update(extra)
    return cfg


class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.QUERY,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.lines:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': smax, 'reasons': sorted(reasons),
                'samples': len(sm)}


def _profiled_traffic(cls):
    """DRAM bytes per launch of a class kernel from its committed ncu summary
    (profiles/quartet_kernel_<class>_h2o32_svp.md), or None."""
    import re
    name = '%d%d%d%d' % (cls['la'], cls['lb'], cls['lc'], cls['ld'])
    path = ROOT / 'profiles' / ('quartet_kernel_%s_h2o32_svp.md' % name)
    if not path.exists():
        return None
    m = re.search(r'dram_bytes_per_launch:\s*(\d+)', path.read_text())
    return int(m.group(1)) if m else None


def cpu_reference_build(mol, bas, dens, nodes=1, threads=None):
    """Seconds for the reference FockDriver share (rank 0 of `nodes`) on host cores."""
    from oracle.oracle import RefOracle
    threads = threads or os.cpu_count()
    RefOracle.set_threads(threads)
    t0 = time.perf_counter()
    ref = RefOracle(mol, bas, partition=False)
    ref.partition()
    t_screen = time.perf_counter() - t0
    t0 = time.perf_counter()
    f = ref.fock(dens, '2jk', 1.0, 0.0, ITHRESHOLD, True, 0, nodes)
    return time.perf_counter() - t0, t_screen, threads, f


def run_reference(args):
    rank, world, _ = _env()
    if rank != 0:
        return 0
    from oracle.oracle import ref_available
    if not ref_available():
        print(json.dumps({'impl': 'reference', 'unavailable': 'oracle/_ref/libvlxref.so not built'}))
        return 0
    mol, bas, dens = _system(0)
    # one full build of the workload per step (FockDriver::compute with
    # rank 0 of 1 node), all host threads; warm-up capped at one build so
    # that the arm stays within a few minutes (a build takes seconds)
    for _ in range(min(args.warmup, 1)):
        cpu_reference_build(mol, bas, dens, 1)
    times = []
    threads = os.cpu_count()
    for _ in range(args.steps):
        dt, _, threads, _ = cpu_reference_build(mol, bas, dens, 1)
        times.append(dt)
    total = sum(times)
    value = args.steps / total
    sample = ('one full build of the workload per step by the reference FockDriver compiled from source '
              '(FockDriver::compute(screener, D, "2jk", 1, 0, 12), -O3 -march=x86-64-v3 OpenMP, %d threads); '
              'builds/s = steps / seconds; warm-up %d build(s)' % (threads, min(args.warmup, 1)))
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * total / args.steps,
            'higher_is_better': True, 'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic', 'config': _config({'threads': threads}),
            'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': threads, 'kind': 'reference', 'sample': sample},
            'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import ctypes

    import torch
    import torch.distributed as dist
    from veloxchem_b200 import FockDriver, T4CScreener, make_matrix, mat_t
    from veloxchem_b200 import _native as nat
    from veloxchem_b200.distributed import distributed_fock

    rank, world, local = _env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group('nccl', timeout=timedelta(seconds=300), device_id=torch.device('cuda', local))
    # one build of one cluster per step; with N ranks every rank evaluates its
    # cost-balanced share of the work items and the FP64 partial Fock
    # matrices are summed by one NCCL all-reduce inside the step
    mol, bas, dens = _system(0)
    scr = T4CScreener(device=local)
    t0 = time.perf_counter()
    scr.partition(bas, mol, 'eri')
    t_screen = time.perf_counter() - t0
    nao = scr.nao
    if world > 1:
        scr.set_partition('balanced')
    # one explicit stream for the copies, the L2 flush, the library's kernels and the events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    d_D = torch.from_numpy(dens).to('cuda')
    d_F = torch.empty_like(d_D)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device='cuda')  # 256 MB > 126 MB L2
    assert stream.cuda_stream != 0
    lib = nat.lib()

    def build():
        if world > 1:
            nat.check(lib.vlx_b200_fock_build_local_device(scr.handle, rank, world, ctypes.c_void_p(d_D.data_ptr()),
                                                            1, b'2jk', 1.0, 0.0, ITHRESHOLD,
                                                            ctypes.c_void_p(d_F.data_ptr()),
                                                            ctypes.c_void_p(stream.cuda_stream)), 'fock_build_local')
            dist.all_reduce(d_F, op=dist.ReduceOp.SUM)
        else:
            nat.check(lib.vlx_b200_fock_build_device(scr.handle, ctypes.c_void_p(d_D.data_ptr()), 1, b'2jk', 1.0,
                                                     0.0, ITHRESHOLD, ctypes.c_void_p(d_F.data_ptr()),
                                                     ctypes.c_void_p(stream.cuda_stream)), 'fock_build_device')

    # one-time set-up outside the timed region: per-class work-item lengths
    tuned = [] if args.no_autotune else nat.autotune(scr, d_D.data_ptr(), ITHRESHOLD, stream.cuda_stream)
    # per-class profile (one full build) -> launches per build and the dominant kernel
    prof = nat.fock_profile(scr, d_D.data_ptr(), d_F.data_ptr(), '2jk', 1.0, ITHRESHOLD, True, stream.cuda_stream)
    launches_per_build = len(prof) + 1  # class kernels + symmetrisation
    for _ in range(max(3, args.warmup)):
        flush.fill_(1.0)
        build()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.fill_(float(k))
        starts[k].record(stream)
        build()
        ends[k].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    t = torch.tensor([total_ms], device='cuda', dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = args.steps / (total_ms / 1e3)

    # roofline of the dominant class kernel (profiled full build, CUDA events per launch)
    prof = nat.fock_profile(scr, d_D.data_ptr(), d_F.data_ptr(), '2jk', 1.0, ITHRESHOLD, True, stream.cuda_stream)
    peak = nat.fp64_peak(local)
    top = max(prof, key=lambda p: p['device_ms'])
    tot_prof_ms = sum(p['device_ms'] for p in prof)
    achieved = top['flops'] / (top['device_ms'] * 1e-3) / 1e12
    all_flops = sum(p['flops'] for p in prof)
    roofline = {'bound': 'fp64', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s', 'frac': achieved / peak,
                'traffic': _profiled_traffic(top),
                'traffic_source': 'dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of this kernel '
                                  'on this workload, summarised under profiles/ (null: no capture of this kernel)',
                'kernel': ('coop_quartet_kernel<double,%d,%d,%d,%d>' if top['table_driven'] else
                           'quartet_kernel<%d,%d,%d,%d>') % (top['la'], top['lb'], top['lc'], top['ld']),
                'kernel_share': top['device_ms'] / tot_prof_ms,
                'peak_source': 'measured: FP64 FMA-chain probe kernel (vlx_b200_fp64_peak), burst; '
                               'MEASURED_PEAKS.json has no FP64 figure',
                'build_achieved_tflops': all_flops / (total_ms / args.steps * 1e-3) / 1e12 / world,
                'build_frac': all_flops / (total_ms / args.steps * 1e-3) / 1e12 / peak / world}

    # end to end through the public API: host Matrix in, host Matrix out
    dm = make_matrix(bas, mat_t.symmetric)
    dm.set_values(dens)
    drv = FockDriver()

    def e2e_build():
        if world > 1:
            return distributed_fock(scr, dm, '2jk', 1.0, 0.0, ITHRESHOLD, partition='balanced')
        return drv.compute(scr, dm, '2jk', 1.0, 0.0, ITHRESHOLD)

    e2e_build()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ne2e = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(ne2e):
        fock = e2e_build()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], device='cuda', dtype=torch.float64)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e = {'value': ne2e / float(te.item()), 'unit': UNIT, 'h2d_bytes_per_step': nao * nao * 8,
           'd2h_bytes_per_step': nao * nao * 8,
           'path': ('distributed_fock(screener, Matrix, "2jk", 1.0, 0.0, 12, partition="balanced"): host Matrix in, '
                    'rank share on each GPU, all-reduce, host Matrix out' if world > 1 else
                    'FockDriver.compute(screener, Matrix, "2jk", 1.0, 0.0, 12): host Matrix in, host Matrix out; '
                    'the copies go through page-locked staging buffers of the driver')}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        from oracle.oracle import ref_available
        if ref_available():
            dt, t_ref_screen, threads, fref = cpu_reference_build(mol, bas, dens, 1)
            err = float(np.max(np.abs(fref - fock.full_matrix().to_numpy())))
            cpu = {'value': 1.0 / dt, 'unit': UNIT, 'cores': threads, 'kind': 'reference',
                   'sample': 'one full build of the same workload by the reference FockDriver compiled from source '
                             '(-O3 -march=x86-64-v3 OpenMP), %d threads; screener %.2f s extra; '
                             'max|F_gpu - F_ref| = %.2e' % (threads, t_ref_screen, err)}

    # the north-star comparison (BASELINE metric: SCF time-to-1e-6 Eh and
    # builds/s, mixed + batched + learned vs plain FP64), on one GPU
    north = None
    if world == 1 and not args.no_north_star:
        from veloxchem_b200 import workloads
        ns_clocks = ClockSampler(local)
        ns_clocks.start()
        t0 = time.perf_counter()
        north = {'c3': workloads.c3_headline(log=lambda m: print(m, file=sys.stderr, flush=True)),
                 'c4': workloads.c4_headline()}
        north['wall_s'] = time.perf_counter() - t0
        north['clocks'] = ns_clocks.stop()

    classes = [{'class': '%d%d%d%d' % (p['la'], p['lb'], p['lc'], p['ld']),
                'kernel': 'coop' if p['table_driven'] else 'compiled',
                'ms': round(p['device_ms'], 4), 'tflops': round(p['flops'] / max(p['device_ms'], 1e-9) / 1e9, 3),
                'fp64_frac': round(p['flops'] / max(p['device_ms'], 1e-9) / 1e9 / peak, 4),
                'quartets': p['shell_quartets']} for p in sorted(prof, key=lambda p: -p['device_ms'])]
    line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': total_ms / args.steps, 'higher_is_better': True,
            'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': _config({'nao': nao, 'screener_s': t_screen,
                               'parallelism': ('one build sharded over %d GPUs (cost-balanced work items, NCCL '
                                               'all-reduce of the FP64 partials)' % world) if world > 1
                               else 'single GPU',
                               'autotuned_classes': sum(1 for t in tuned if t['best_ms'] < t['default_ms']),
                               'autotune': ['%d%d%d%d:%d/%d' % (t['la'], t['lb'], t['lc'], t['ld'], t['segment'],
                                                                t['blocks_per_sm']) for t in tuned]}),
            'roofline': roofline, 'cpu_baseline': cpu, 'e2e': e2e,
            'gpu_launches': launches_per_build * args.steps, 'clocks': clk,
            'quartets_per_build': int(sum(p['shell_quartets'] for p in prof)),
            'classes': classes, 'north_star': north}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-autotune', action='store_true')
    ap.add_argument('--no-north-star', action='store_true', help='skip the (H2O)64 / def2-TZVP and batched workloads')
    args = ap.parse_args()
    if args.impl == 'reference':
        return run_reference(args)
    return run_ours(args)


if __name__ == '__main__':
    sys.exit(main())
