"""Profiling harness: one full J/K build of a water cluster, for ncu.

    python -m byteqc_b200.profile_jk --nwater 16 [--basis cc-pvtz] [--only 2,1,1,0]

Builds (H2O)_n (seed 0) in a synthetic basis, a random symmetric density
(the recipe of the reference's timing script: rand + rand^T, seed 2341,
scaled by 0.1) and runs ``--builds`` J/K builds through BQCbuild_jk, or, with
``--only li,lj,lk,ll``, only the class pairs of that shape through
BQCbuild_jk_class.  Prints the build times measured with CUDA events.
"""
import argparse
import ctypes
import sys

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--nwater', type=int, default=16)
    ap.add_argument('--basis', default='cc-pvtz')
    ap.add_argument('--builds', type=int, default=1)
    ap.add_argument('--only', default=None)
    a = ap.parse_args(argv)
    import torch
    from byteqc_b200 import lib as L
    from byteqc_b200.gto.mole import Mole
    from byteqc_b200.gto.basis import synthetic_basis
    from byteqc_b200.gto.geom import water_cluster
    from byteqc_b200.scf import hf
    from byteqc_b200.scf.hf import _ptr, _stream
    lib = L.load_library()
    mol = Mole(water_cluster(a.nwater, seed=0), synthetic_basis(a.basis, ['O', 'H']))
    opt = hf._VHFOpt(mol).build()
    rng = np.random.default_rng(2341)
    dm = rng.random((mol.nao, mol.nao))
    dm = 0.1 * (dm + dm.T)
    dm = torch.as_tensor(dm, device='cuda')
    C = opt.coeff_dev
    dmc = (C @ dm @ C.T)[None].contiguous()
    nao = dmc.shape[-1]
    dm_cond = torch.empty((opt.mol.nbas, opt.mol.nbas), dtype=torch.float64, device='cuda')
    lib.BQCdm_cond(_ptr(dmc), 1, nao, _ptr(opt._mem['ao_loc']), opt.mol.nbas, _ptr(dm_cond),
                   _stream())
    dm_max = float(dm_cond.max())
    qh = opt.pair_q_host.ctypes.data_as(ctypes.c_void_p)
    bp = ctypes.cast(opt.bpcache, ctypes.c_void_p)
    shape = tuple(int(x) for x in a.only.split(',')) if a.only else None
    for b in range(a.builds):
        vj = torch.zeros_like(dmc)
        vk = torch.zeros_like(dmc)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        if shape is None:
            err = lib.BQCbuild_jk(bp, _ptr(opt.pair_q), qh, _ptr(dm_cond), dm_max, _ptr(vj),
                                  _ptr(vk), _ptr(dmc), nao, 1, opt.direct_scf_tol, 0., None,
                                  _stream())
        else:
            err = 0
            for cij in range(opt.ncptype):
                for ckl in range(cij + 1):
                    li, lj = opt.cptype[cij][:2]
                    lk, ll = opt.cptype[ckl][:2]
                    if shape in ((li, lj, lk, ll), (lk, ll, li, lj)) and \
                            opt.cptype[cij][3] and opt.cptype[ckl][3]:
                        err |= lib.BQCbuild_jk_class(bp, cij, ckl, _ptr(opt.pair_q), qh,
                                                     _ptr(dm_cond), dm_max, _ptr(vj), _ptr(vk),
                                                     _ptr(dmc), nao, 1, opt.direct_scf_tol, 0.,
                                                     None, _stream())
        e1.record()
        torch.cuda.synchronize()
        if err:
            raise RuntimeError('build failed (%d)' % err)
        print('build %d: %.3f ms' % (b, e0.elapsed_time(e1)))
    return 0


if __name__ == '__main__':
    sys.exit(main())
