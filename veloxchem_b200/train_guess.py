"""Train and evaluate the learned initial guess (def2-SVP water clusters).

    python -m veloxchem_b200.train_guess --clusters 2000 --out weights.npz --report report.json

1. Data: seeded water clusters with n ~ U{nmin..nmax} waters on the first n
   sites of a 4 x 3 x 2 lattice (the cluster generator of geometry.py); each
   is converged with this package's FP64 SCF from SAD; the pair descriptors
   and the local-frame blocks of (D_converged - D_SAD) are the samples.
2. Training: the three-layer network of guess_net.GuessMLP (width 128, SiLU),
   FP32, masked mean squared error (on-site blocks weighted SELF_WEIGHT),
   Adam with cosine-decayed step size, all through the library's own
   kernels; 5% of the clusters are held out.
3. Evaluation: held-out (H2O)_n clusters on a 4 x 4 x 3 lattice, SCF from SAD
   and from the learned guess (with the SAD fallback of the SCF driver);
   reports iterations and time to |E - E_ref| < 1e-6 Eh, E_ref being the FP64
   energy of full builds converged to a 1e-8 gradient from SAD.
"""

import argparse
import json
import math
import time

import numpy as np

SELF_WEIGHT = 10.0  # loss weight of the on-site (i = j) blocks


def _scf(mol, bas, guess, conv=1e-6, weights=None, guess_density=None, incremental=True):
    from .scf import ScfRestrictedDriver
    drv = ScfRestrictedDriver()
    drv.conv_thresh = conv
    drv.incremental = incremental
    drv.guess = guess
    drv.guess_weights = weights
    t0 = time.perf_counter()
    res = drv.compute(mol, bas, guess_density=guess_density)
    res['wall_s'] = time.perf_counter() - t0
    return res


def generate(clusters, nmin, nmax, seed, log=print):
    from . import MolecularBasis
    from .geometry import water_cluster
    from .guess import ClusterLayout
    from .scf import SadGuessDriver
    rng = np.random.default_rng(seed)
    X, T, M, owner = [], [], [], []
    t0 = time.perf_counter()
    for c in range(clusters):
        n = int(rng.integers(nmin, nmax + 1))
        mol = water_cluster((4, 3, 2), seed + 1 + c, n)
        bas = MolecularBasis.read(mol, 'def2-svp')
        minb = MolecularBasis.read(mol, 'ao-start-guess')
        d_sad = SadGuessDriver().compute(mol, minb, bas)
        res = _scf(mol, bas, 'sad', guess_density=d_sad)
        if not res['converged']:
            continue
        lay = ClusterLayout(mol, bas)
        tc, m = lay.local_blocks(res['D_alpha'])
        ts, _ = lay.local_blocks(d_sad)
        X.append(lay.descriptors())
        T.append(tc - ts)
        # on-site blocks weigh more: the energy is most sensitive to them
        m[lay.pairs[:, 0] == lay.pairs[:, 1]] *= SELF_WEIGHT
        M.append(m)
        owner.append(np.full(len(lay.pairs), c, dtype=np.int64))
        if (c + 1) % 100 == 0:
            log('data %d / %d clusters, %.1f s' % (c + 1, clusters, time.perf_counter() - t0))
    return np.concatenate(X), np.concatenate(T), np.concatenate(M), np.concatenate(owner)


def train(X, T, M, owner, epochs=120, batch=4096, lr=2e-3, scale=10.0, seed=0, log=print):
    import torch
    from .guess import NFEAT, NOUT
    from .guess_net import GuessMLP
    dev = torch.device('cuda', 0)
    mu = X.mean(axis=0)
    sd = X.std(axis=0)
    sd[sd < 1e-6] = 1.0
    rng = np.random.default_rng(seed)
    clusters = np.unique(owner)
    val_c = set(rng.choice(clusters, size=max(1, len(clusters) // 20), replace=False).tolist())
    is_val = np.array([o in val_c for o in owner])
    Xd = torch.tensor((X - mu) / sd, dtype=torch.float32, device=dev)
    Td = torch.tensor(T * scale, dtype=torch.float32, device=dev)
    Md = torch.tensor(M, dtype=torch.float32, device=dev)
    tr_idx = torch.tensor(np.where(~is_val)[0], device=dev)
    va_idx = torch.tensor(np.where(is_val)[0], device=dev)
    net = GuessMLP(NFEAT, NOUT, 128, 3, seed=seed)
    steps_per_epoch = max(1, len(tr_idx) // batch)
    total = epochs * steps_per_epoch
    hist = []
    t0 = time.perf_counter()
    step = 0
    for ep in range(epochs):
        perm = tr_idx[torch.randperm(len(tr_idx), device=dev)]
        tl = 0.0
        for s in range(steps_per_epoch):
            idx = perm[s * batch:(s + 1) * batch]
            xb, tb, mb = Xd[idx], Td[idx], Md[idx]
            y, cache = net.forward(xb, keep=True)
            loss, dy = net.mse(y, tb, mb)
            grads = net.backward(dy, cache)
            cur = 1e-5 + 0.5 * (lr - 1e-5) * (1.0 + math.cos(math.pi * step / total))
            net.adam_step(grads, lr=cur)
            tl += float(loss.item()) if s % 20 == 0 else 0.0
            step += 1
        vl = 0.0
        for s in range(0, len(va_idx), 65536):
            idx = va_idx[s:s + 65536]
            y = net.forward(Xd[idx])
            l, _ = net.mse(y, Td[idx], Md[idx])
            vl += float(l.item()) * float(Md[idx].sum().item())
        vl /= max(float(Md[va_idx].sum().item()), 1.0)
        hist.append({'epoch': ep + 1, 'val_mse': vl})
        if (ep + 1) % 5 == 0 or ep == 0:
            log('epoch %d  val mse (scaled) %.3e  %.1f s' % (ep + 1, vl, time.perf_counter() - t0))
    state = net.state_dict()
    state.update(mu=mu.astype(np.float32), sd=sd.astype(np.float32), target_scale=np.float64(scale))
    return state, hist, time.perf_counter() - t0


def _time_to(res, e_ref, tol=1e-6):
    """(iterations, seconds) until |E - E_ref| < tol for good (None if never)."""
    hist = res['history']
    for k in range(len(hist)):
        if all(abs(h['energy'] - e_ref) < tol for h in hist[k:]):
            return hist[k]['iteration'], hist[k]['time_s']
    return None, None


def evaluate(weights, count, nwaters, seed, log=print):
    from . import MolecularBasis
    from .geometry import water_cluster
    rows = []
    for k in range(count):
        mol = water_cluster((4, 4, 3), seed + k, nwaters)
        bas = MolecularBasis.read(mol, 'def2-svp')
        if k == 0:
            _scf(mol, bas, 'sad')  # warm-up: CUDA context, kernels, basis files
        # E_ref: full FP64 builds every iteration, converged to a 1e-8 gradient
        ref = _scf(mol, bas, 'sad', conv=1e-8, incremental=False)
        sad = _scf(mol, bas, 'sad')
        lrn = _scf(mol, bas, 'learned', weights=weights)
        e_ref = ref['scf_energy']
        row = {'seed': seed + k, 'e_ref': e_ref}
        for name, r in (('sad', sad), ('learned', lrn)):
            it, ts = _time_to(r, e_ref)
            conv_it = next((h['iteration'] for h in r['history'] if h['e_grad'] < 1e-6), None)
            row[name] = {'iterations_to_grad_1e-6': conv_it, 'converged': r['converged'], 'wall_s': r['wall_s'],
                         'iters_to_1e-6': it, 'time_to_1e-6_s': ts, 'energy_error': r['scf_energy'] - e_ref,
                         'guess_used': r.get('guess_used'), 'learned_guess_s': r['timings'].get('learned_guess_s')}
        row['learned']['guess_energies'] = lrn['timings'].get('guess_energies')
        rows.append(row)
        log('eval %d: SAD %s it %.2f s | learned (%s) %s it %.2f s' %
            (k, row['sad']['iters_to_1e-6'], row['sad']['time_to_1e-6_s'] or -1, row['learned']['guess_used'],
             row['learned']['iters_to_1e-6'], row['learned']['time_to_1e-6_s'] or -1))
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--clusters', type=int, default=2000)
    ap.add_argument('--nmin', type=int, default=2)
    ap.add_argument('--nmax', type=int, default=24)
    ap.add_argument('--seed', type=int, default=100000)
    ap.add_argument('--epochs', type=int, default=120)
    ap.add_argument('--out', default='guess_mlp_svp.npz')
    ap.add_argument('--eval', type=int, default=100)
    ap.add_argument('--eval-waters', type=int, default=48)
    ap.add_argument('--eval-seed', type=int, default=900000)
    ap.add_argument('--report', default='guess_report.json')
    ap.add_argument('--eval-only', default=None, help='evaluate this weights file, no training')
    a = ap.parse_args(argv)

    def log(msg):
        print(msg, flush=True)

    if a.eval_only:
        X, t_data, t_train, hist = np.zeros((0, 1)), 0.0, 0.0, []
        weights = a.eval_only
    else:
        t0 = time.perf_counter()
        X, T, M, owner = generate(a.clusters, a.nmin, a.nmax, a.seed, log)
        t_data = time.perf_counter() - t0
        log('samples %d pairs from %d clusters, %.1f s' % (len(X), len(np.unique(owner)), t_data))
        state, hist, t_train = train(X, T, M, owner, epochs=a.epochs, log=log)
        np.savez(a.out, **state)
        weights = a.out
    rows = evaluate(weights, a.eval, a.eval_waters, a.eval_seed, log) if a.eval > 0 else []
    summary = {}
    for name in ('sad', 'learned'):
        its = [r[name]['iters_to_1e-6'] for r in rows if r[name]['iters_to_1e-6']]
        tts = [r[name]['time_to_1e-6_s'] for r in rows if r[name]['time_to_1e-6_s']]
        summary[name] = {'mean_iters_to_1e-6': float(np.mean(its)) if its else None,
                         'mean_time_to_1e-6_s': float(np.mean(tts)) if tts else None,
                         'max_abs_energy_error': float(max(abs(r[name]['energy_error']) for r in rows))
                         if rows else None}
    summary['fallback_to_sad'] = sum(1 for r in rows if r['learned']['guess_used'] == 'sad')
    rep = {'clusters': a.clusters, 'nmin': a.nmin, 'nmax': a.nmax, 'seed': a.seed, 'samples': int(len(X)),
           'data_s': t_data, 'train_s': t_train, 'epochs': a.epochs, 'history': hist,
           'eval': {'count': a.eval, 'waters': a.eval_waters, 'seed': a.eval_seed, 'summary': summary,
                    'rows': rows}}
    with open(a.report, 'w') as f:
        json.dump(rep, f, indent=1)
    log(json.dumps(summary))


if __name__ == '__main__':
    main()
