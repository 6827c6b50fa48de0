"""Per-class kernel autotuner of the J/K engine.

Some shell-quartet classes have two kernels (jk_kernels.cuh, launch_class):
the group kernel (several threads per quartet share the 2D tables in shared
memory) and ket-split tile launches (one thread per quartet, shell k's
components spread over up to three launches).  ``tune`` times both on the
class pairs of a basis, with the caller's density or the density of the
reference's timing script, and keeps the faster one per class through
BQCset_class_variant.  The choice changes speed only; results are the same
to rounding.

    from byteqc_b200 import autotune
    choice = autotune.tune(opt)          # opt: a built scf.hf._VHFOpt
    autotune.save(choice, 'variants.json'); autotune.apply(autotune.load(...))
"""
import ctypes
import json

import numpy as np

SMALL_NF = 54          # jk_kernels.cuh SMALL_NF
MAX_SPLIT = 3          # jk_kernels.cuh MAX_SPLIT
GROUP, SPLIT = 1, 2    # BQC_VARIANT_GROUP, BQC_VARIANT_SPLIT


def _nc(l):
    return (l + 1) * (l + 2) // 2


def canonical(li, lj, lk, ll):
    """The class as the library dispatches it: li >= lj, lk >= ll, bra pair
    index >= ket pair index."""
    if li < lj:
        li, lj = lj, li
    if lk < ll:
        lk, ll = ll, lk
    if li * (li + 1) // 2 + lj < lk * (lk + 1) // 2 + ll:
        li, lj, lk, ll = lk, ll, li, lj
    return li, lj, lk, ll


def has_variants(li, lj, lk, ll):
    """True when the class has both kernels (the rule of launch_class)."""
    l1, l2, l3, l4 = canonical(li, lj, lk, ll)
    n12, n34 = _nc(l1) * _nc(l2), _nc(l3) * _nc(l4)
    if n12 * n34 <= SMALL_NF:
        return False
    ck = SMALL_NF // (n12 * _nc(l4))
    if ck >= 1 and -(-_nc(l3) // ck) <= MAX_SPLIT:
        return True
    # an s-s ket: the bra's first shell splits with bra and ket exchanged
    cks = SMALL_NF // (n34 * _nc(l2))
    return ck == 0 and n34 == 1 and cks >= 1 and -(-_nc(l1) // cks) <= MAX_SPLIT


def apply(choice):
    from . import lib as L
    lib = L.load_library()
    for key, v in choice.items():
        err = lib.BQCset_class_variant(*[int(x) for x in key], int(v))
        if err:
            raise ValueError('BQCset_class_variant%s failed (%d)' % (tuple(key), err))


def save(choice, path):
    with open(path, 'w') as f:
        json.dump({''.join(str(x) for x in k): v for k, v in choice.items()}, f, indent=1)


def load(path):
    with open(path) as f:
        return {tuple(int(c) for c in k): v for k, v in json.load(f).items()}


def tune(opt, dmc=None, reps=3, tol=None):
    """Time both kernels of every class with two; set and return the faster
    one per canonical class {(li, lj, lk, ll): variant}."""
    import torch
    from . import lib as L
    from .scf.hf import _ptr, _stream
    lib = L.load_library()
    if dmc is None:
        rng = np.random.default_rng(2341)
        n0 = opt.coeff.shape[1]
        dm = rng.random((n0, n0))
        dm = torch.as_tensor(0.1 * (dm + dm.T), device=opt.pair_q.device)
        C = opt.coeff_dev
        dmc = (C @ dm @ C.T)[None].contiguous()
    n_dm, nao = dmc.shape[0], dmc.shape[-1]
    tol = opt.direct_scf_tol if tol is None else tol
    dm_cond = torch.empty((opt.mol.nbas, opt.mol.nbas), dtype=torch.float64, device=dmc.device)
    err = lib.BQCdm_cond(_ptr(dmc), ctypes.c_int(n_dm), ctypes.c_int(nao),
                         _ptr(opt._mem['ao_loc']), ctypes.c_int(opt.mol.nbas), _ptr(dm_cond),
                         _stream())
    if err:
        raise RuntimeError('BQCdm_cond failed (%d)' % err)
    dm_max = float(dm_cond.max())
    vj = torch.zeros_like(dmc)
    vk = torch.zeros_like(dmc)
    qh = opt.pair_q_host.ctypes.data_as(ctypes.c_void_p)
    bp = ctypes.cast(opt.bpcache, ctypes.c_void_p)
    pairs = {}
    for cij in range(opt.ncptype):
        for ckl in range(cij + 1):
            if not (opt.cptype[cij][3] and opt.cptype[ckl][3]):
                continue
            li, lj = opt.cptype[cij][:2]
            lk, ll = opt.cptype[ckl][:2]
            if has_variants(li, lj, lk, ll):
                pairs.setdefault(canonical(li, lj, lk, ll), []).append((cij, ckl))

    def run():
        for cij, ckl in cls_pairs:
            err = lib.BQCbuild_jk_class(bp, cij, ckl, _ptr(opt.pair_q), qh, _ptr(dm_cond), dm_max,
                                        _ptr(vj), _ptr(vk), _ptr(dmc), nao, n_dm, tol, 0., None,
                                        _stream())
            if err:
                raise RuntimeError('BQCbuild_jk_class failed (%d)' % err)

    choice = {}
    for key, cls_pairs in pairs.items():
        best = {}
        for v in (GROUP, SPLIT):
            lib.BQCset_class_variant(*key, v)
            run()                                   # warm-up (module load)
        for _ in range(reps):
            for v in (GROUP, SPLIT):
                lib.BQCset_class_variant(*key, v)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                run()
                e1.record()
                torch.cuda.synchronize()
                best[v] = min(best.get(v, 1e30), e0.elapsed_time(e1))
        choice[key] = min(best, key=best.get)
        lib.BQCset_class_variant(*key, choice[key])
    return choice
