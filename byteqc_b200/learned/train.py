"""Train the density-guess MLP on converged densities of the plain SCF.

    python -m byteqc_b200.learned.train --nsys 300 --epochs 200 \
        --out byteqc_b200/learned/weights_ccpvdz.npz --report report.json

Training systems: seeded (H2O)_k, k uniform in [2, 16], and all-trans
CnH(2n+2), n uniform in [4, 20], in the cc-pVDZ-shaped basis; each is solved
by the plain FP64 RHF of this package (SAD guess, |Delta E| < 1e-9) and every
atom pair within the cutoff becomes a sample.  Evaluation: held-out (H2O)_32
and C40H82: SCF cycles and wall time from SAD and from the learned guess,
with the converged energies compared.
"""
import argparse
import json
import time

import numpy as np
import torch

from ..gto.mole import Mole
from ..gto.basis import synthetic_basis
from ..gto.geom import water_cluster, linear_alkane
from ..scf import hf
from ..scf.guess import init_guess
from . import dataset
from .model import DensityMLP

BASIS = 'cc-pvdz'


def training_systems(nsys, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for s in range(nsys):
        if s % 2 == 0:
            k = int(rng.integers(2, 17))
            out.append(('water', k, 1000 + s, water_cluster(k, seed=1000 + s)))
        else:
            n = int(rng.integers(4, 21))
            out.append(('alkane', n, 0, linear_alkane(n)))
    return out


def make_mol(atoms, basis=None):
    els = sorted(set(a[0] for a in atoms))
    mol = Mole(atoms, synthetic_basis(basis or BASIS, els))
    mol.basis_name = (basis or BASIS).lower()
    return mol


def converged(mol, conv=1e-9):
    mf = hf.RHF(mol)
    mf.conv_tol = conv
    mf.kernel()
    sad = init_guess(mf, 'sad')
    return mf, mf.dm.cpu().numpy(), sad.cpu().numpy()


def collect(systems, log=print, basis=None):
    from .features import OUT_DIMS
    out_dim = OUT_DIMS[(basis or BASIS).lower()]
    F, T, K = [], [], []
    t0 = time.time()
    cache = {}
    for i, (kind, size, seed, atoms) in enumerate(systems):
        key = (kind, size, seed)
        if key not in cache:
            mol = make_mol(atoms, basis)
            mf, dm, sad = converged(mol)
            cache[key] = dataset.samples(mol, dm, sad, out_dim, np.float32)
        f, t, k = cache[key]
        F.append(f)
        T.append(t)
        K.append(k)
        if (i + 1) % 25 == 0:
            log('collected %d systems, %.0f s' % (i + 1, time.time() - t0))
    return np.vstack(F), np.vstack(T), np.vstack(K)


def fit(F, T, K, epochs=200, batch=4096, lr=1e-3, seed=0, log=print):
    dev = torch.device('cuda')
    model = DensityMLP(seed=seed, out_dim=T.shape[1])
    Fd = torch.as_tensor(F, dtype=torch.float32, device=dev)
    Td = torch.as_tensor(T, dtype=torch.float32, device=dev)
    Kd = torch.as_tensor(K, dtype=torch.float32, device=dev)
    n = len(F)
    g = torch.Generator(device='cpu').manual_seed(seed)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(dev)
        tot = 0.
        cur_lr = lr * 0.5 * (1 + np.cos(np.pi * ep / epochs))
        for s in range(0, n - batch + 1 if n >= batch else 1, batch):
            idx = perm[s:s + batch]
            m = (len(idx) // 16) * 16
            idx = idx[:m]
            y = model.forward(Fd[idx], keep=True)
            diff = (y - Td[idx]) * Kd[idx]
            norm = Kd[idx].sum()
            loss = (diff * diff).sum() / norm
            dy = 2. * diff / norm
            grads = model.backward(dy)
            model.adam(grads, lr=cur_lr)
            tot += float(loss) * m
        hist.append(tot / max(n, 1))
        if ep % 20 == 0 or ep == epochs - 1:
            log('epoch %d loss %.3e' % (ep, hist[-1]))
    return model, hist


def evaluate(model_path, log=print, basis=None):
    """SCF cycles and time from SAD and from the learned guess on held-out
    (H2O)_32 (seed 7) and C40H82."""
    out = {}
    for name, atoms in (('(H2O)32', water_cluster(32, seed=7)), ('C40H82', linear_alkane(40))):
        mol = make_mol(atoms, basis)
        rec = {}
        for guess in ('sad', 'mlp'):
            from ..learned import infer
            infer._MODELS.clear()
            mf = hf.RHF(mol)
            mf.conv_tol = 1e-9
            mf.init_guess = guess
            mf.mlp_weights = model_path
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e = mf.kernel()
            torch.cuda.synchronize()
            rec[guess] = {'energy': e, 'cycles': mf.cycles, 'seconds': time.perf_counter() - t0,
                          'converged': bool(mf.converged),
                          'fallback': bool(getattr(mf, 'guess_fallback', False))}
        rec['energy_diff'] = abs(rec['mlp']['energy'] - rec['sad']['energy'])
        out[name] = rec
        log(name, json.dumps(rec))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--nsys', type=int, default=300)
    ap.add_argument('--epochs', type=int, default=200)
    ap.add_argument('--out', default=None)
    ap.add_argument('--report', default=None)
    ap.add_argument('--basis', default=BASIS)
    a = ap.parse_args(argv)
    t0 = time.time()
    F, T, K = collect(training_systems(a.nsys), basis=a.basis)
    t_data = time.time() - t0
    print('samples', F.shape, 'data %.0f s' % t_data, flush=True)
    t0 = time.time()
    model, hist = fit(F, T, K, epochs=a.epochs)
    t_fit = time.time() - t0
    out = a.out or __import__('os').path.join(__import__('os').path.dirname(__file__),
                                              'weights_%s.npz' % a.basis.replace('-', ''))
    np.savez(out, **model.state())
    ev = evaluate(out, basis=a.basis)
    rep = {'nsys': a.nsys, 'samples': int(F.shape[0]), 'epochs': a.epochs,
           'data_seconds': t_data, 'fit_seconds': t_fit, 'loss_first': hist[0],
           'loss_last': hist[-1], 'eval': ev}
    print(json.dumps(rep))
    if a.report:
        json.dump(rep, open(a.report, 'w'), indent=1)


if __name__ == '__main__':
    main()
