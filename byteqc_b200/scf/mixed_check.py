"""Accuracy and speed of the mixed-precision form against plain FP64 on one
molecule: J/K max-abs error of an FP32-band build, and the converged SCF
energy and wall time of both forms.

    python -m byteqc_b200.scf.mixed_check --alkane 60 --basis 6-31g**
    python -m byteqc_b200.scf.mixed_check --water 32 --basis cc-pvtz

Prints one JSON object.  J/K errors are measured on two densities: the
converged one (a full build, the form's FP64 rebuild replaces it) and the
difference density of the second SCF cycle (the incremental build the FP32
band is for).
"""
import argparse
import json
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--alkane', type=int, default=0, help='all-trans CnH(2n+2)')
    ap.add_argument('--water', type=int, default=0, help='(H2O)_n cluster, seed 0')
    ap.add_argument('--basis', default='6-31g**')
    ap.add_argument('--fp32-below', type=float, default=1e-6)
    ap.add_argument('--early-tol', type=float, default=0.)
    ap.add_argument('--conv', type=float, default=1e-8)
    a = ap.parse_args(argv)
    import torch
    from ..gto.mole import Mole
    from ..gto.basis import synthetic_basis
    from ..gto.geom import water_cluster, linear_alkane
    from . import hf, guess
    if a.alkane:
        atoms, elems, name = linear_alkane(a.alkane), ['C', 'H'], 'C%dH%d' % (a.alkane, 2 * a.alkane + 2)
    else:
        atoms, elems, name = water_cluster(a.water or 4, seed=0), ['O', 'H'], '(H2O)%d' % (a.water or 4)
    mol = Mole(atoms, synthetic_basis(a.basis, elems))

    def solve(mixed):
        guess._SAD_CACHE.clear()
        mf = hf.RHF(mol)
        mf.conv_tol = a.conv
        if mixed:
            mf.fp32_threshold = a.fp32_below
            mf.early_tol = a.early_tol
        ddm = []
        mf.jk_hook = lambda d, f: ddm.append(d) if len(ddm) < 2 else None
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        e = mf.kernel()
        e1.record()
        torch.cuda.synchronize()
        return mf, e, e0.elapsed_time(e1) / 1e3, ddm

    solve(False)                      # warm-up (library load, caches)
    mf0, e0, t0, ddm = solve(False)
    mf1, e1, t1, _ = solve(True)
    opt = mf0.opt
    out = {'molecule': name, 'basis': a.basis + ' (synthetic, same shell shapes)', 'nao': mol.nao,
           'fp32_below': a.fp32_below, 'early_tol': a.early_tol,
           'plain': {'energy': e0, 'cycles': mf0.cycles, 'seconds': round(t0, 3)},
           'mixed': {'energy': e1, 'cycles': mf1.cycles, 'seconds': round(t1, 3),
                     'builds': [r[:2] for r in mf1.build_log]},
           'abs_dE': abs(e1 - e0), 'speedup': round(t0 / t1, 3)}
    for label, d in (('converged', mf0.dm), ('cycle2_difference', ddm[1] if len(ddm) > 1 else None)):
        if d is None:
            continue
        d = d[None] if d.dim() == 2 else d
        vj0, vk0 = opt.jk_ao(d)
        vj1, vk1 = opt.jk_ao(d, fp32_below=a.fp32_below)
        out['jk_error_' + label] = {
            'J_maxabs': float((vj1 - vj0).abs().max()), 'K_maxabs': float((vk1 - vk0).abs().max()),
            'J_max': float(vj0.abs().max()), 'K_max': float(vk0.abs().max())}
    print(json.dumps(out))
    return 0


if __name__ == '__main__':
    sys.exit(main())
