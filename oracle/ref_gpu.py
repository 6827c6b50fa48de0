"""The reference's own GPU J/K kernels, driven from Python.

Test and measurement infrastructure only: a second checker for the engine's
J/K and the reference timing beside it.  Nothing in the engine imports it.

libgint.so and libgvhf.so are compiled from the reference's cuobc/lib sources
for sm_100a by oracle/build_ref.sh into oracle/_ref/.  RefJK restates the host
side that drives them in the reference:

* pair lists: cuobc/scf/hf.py:341-397 (_VHFOpt.build) -- per (l, nprim)
  group pair, the shell pairs with Schwarz factor above the cutoff, sorted by
  descending factor, log q clipped at 0;
* basis-product cache: cuobc/scf/hf.py:410-436 (initBpcache) --
  GINTinit_basis_prod_cpu, then GINTinit_basis_prod_gpu on device copies of
  ao_loc, bas_coords, aexyz and the pair list;
* J/K: cuobc/scf/hf.py:91-180 (get_jk) -- class-level density screen
  (absmax over (l, nprim) group blocks), log q bins down to tol / dm_cond
  (_make_s_index_offsets, hf.py:567-578), nbins = max(10, pairs_max // 1e5),
  one GINTbuild_jk per class pair, then J = 2 (V + V^T), K = V + V^T.

pyscf is absent, so the basis decontraction and shell sort (restated in
byteqc_b200.scf.hf) and the Schwarz factors (the engine's device kernel; the
reference reads them from pyscf's CVHFsetnr_direct_scf) come from the
engine's _VHFOpt, whose lists hold exactly the pairs above the cutoff.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, '_ref')

_LIBS = None


def available():
    return all(os.path.exists(os.path.join(REF, n)) for n in ('libgint.so', 'libgvhf.so'))


def load():
    """(libgint, libgvhf) from oracle/_ref; raises if they were not built."""
    global _LIBS
    if _LIBS is None:
        if not available():
            raise FileNotFoundError('reference libraries not built (oracle/build_ref.sh)')
        lg = ctypes.CDLL(os.path.join(REF, 'libgint.so'), mode=ctypes.RTLD_GLOBAL)
        lv = ctypes.CDLL(os.path.join(REF, 'libgvhf.so'))
        _LIBS = (lg, lv)
    return _LIBS


def make_s_index_offsets(log_q, nbins, cutoff):
    """cuobc/scf/hf.py:567-578, including its bin-size limit."""
    scale = nbins / np.log(min(cutoff, .1))
    s_index = np.floor(scale * log_q).astype(np.int32)
    bins = np.bincount(s_index, minlength=nbins)[:nbins]
    if bins.size and bins.max() >= 65536 * 8:
        raise ValueError('a bin holds more pairs than the reference kernel accepts')
    return np.append(0, np.cumsum(bins)).astype(np.int32)


class RefJK:
    """The reference J/K builder over the engine's sorted, decontracted basis."""

    def __init__(self, opt):
        import torch
        from byteqc_b200 import lib as L
        lg, lv = load()
        self.lg, self.lv = lg, lv
        self.opt = opt
        pmol = opt.mol
        dev = opt.pair_q.device
        # lists in the reference's order: descending q inside each class
        locs = opt.bas_pairs_locs
        keep = ~opt.pair_dummy
        bra, ket, self.log_qs = [], [], []
        for c in range(opt.ncptype):
            sl = slice(locs[c], locs[c + 1])
            k = keep[sl]
            q = opt.pair_q_host[sl][k]
            order = np.argsort(-q, kind='stable')
            bra.append(opt.bas_pair2shls[0, sl][k][order])
            ket.append(opt.bas_pair2shls[1, sl][k][order])
            self.log_qs.append(np.minimum(np.log(q[order]), 0.))
        self.pair2shls = np.ascontiguousarray(np.vstack([np.hstack(bra), np.hstack(ket)]),
                                              dtype=np.int32)
        self.pairs_locs = np.append(0, np.cumsum([len(b) for b in bra])).astype(np.int32)
        self.ncptype = opt.ncptype
        self.atm = np.ascontiguousarray(pmol._atm, dtype=np.int32)
        self.bas = np.ascontiguousarray(pmol._bas, dtype=np.int32)
        self.env = np.ascontiguousarray(pmol._env)
        self.bas_coords = np.empty(pmol.nbas * 3)
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        tp = lambda t: ctypes.c_void_p(t.data_ptr())
        bp = ctypes.POINTER(L.BasisProdCache)()
        diag_fac = 0.5
        lg.GINTinit_basis_prod_cpu(ctypes.byref(bp), ctypes.c_double(diag_fac), vp(self.bas_coords),
                                   vp(self.pair2shls), vp(self.pairs_locs), ctypes.c_int(self.ncptype),
                                   vp(self.atm), ctypes.c_int(pmol.natm), vp(self.bas),
                                   ctypes.c_int(pmol.nbas), vp(self.env))
        nprim = bp.contents.primitive_pairs_locs[self.ncptype]
        aexyz = np.ctypeslib.as_array(bp.contents.aexyz, (nprim * 5,)).copy()
        self.mem = {
            'ao_loc': torch.as_tensor(pmol.ao_loc_nr(cart=True), dtype=torch.int32, device=dev),
            'bas_coords': torch.as_tensor(self.bas_coords, device=dev),
            'aexyz': torch.as_tensor(aexyz, device=dev),
            'pair2shls': torch.as_tensor(self.pair2shls.ravel(), device=dev),
        }
        self.bp_cpu = bp
        self.bp_gpu = ctypes.POINTER(L.BasisProdCache)()
        lg.GINTinit_basis_prod_gpu(ctypes.byref(bp), ctypes.byref(self.bp_gpu),
                                   tp(self.mem['ao_loc']), tp(self.mem['bas_coords']),
                                   tp(self.mem['aexyz']), tp(self.mem['pair2shls']))
        self.ao_loc = pmol.ao_loc_nr(cart=True)
        self.group_ao_loc = self.ao_loc[opt.l_ctr_offsets]
        self.uniq_l = opt.uniq_l_ctr[:, 0]
        pairs_max = int((self.pairs_locs[1:] - self.pairs_locs[:-1]).max())
        self.nbins = max(10, pairs_max // 100000)

    def close(self):
        # as cuobc/scf/hf.py does, release through the device copy only (it
        # owns the class table and pair block it shares with the host cache)
        if self.bp_gpu is not None:
            self.lg.GINTdel_basis_prod(ctypes.byref(self.bp_gpu))
            self.bp_gpu = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def dm_cond(self, dmc):
        """Absmax of each (l, nprim) group block over all densities (host)."""
        d = np.abs(dmc.cpu().numpy()).max(axis=0)
        g = self.group_ao_loc[:-1]
        return np.maximum.reduceat(np.maximum.reduceat(d, g, axis=0), g, axis=1)

    def tasks(self, dmc, tol=1e-13):
        """The (cp_ij, cp_kl, bins_ij, bins_kl) launches of one build."""
        cond = self.dm_cond(dmc)
        cp_idx, cp_jdx = np.tril_indices(self.ncptype)
        out = []
        for n in range(self.ncptype * (self.ncptype + 1) // 2):
            cij = int(np.floor(np.sqrt(2 * n)))
            if cij * (cij + 1) // 2 > n:
                cij -= 1
            ckl = n - cij * (cij + 1) // 2
            lq_ij, lq_kl = self.log_qs[cij], self.log_qs[ckl]
            if lq_ij.size == 0 or lq_kl.size == 0:
                continue
            i, j, k, l = cp_idx[cij], cp_jdx[cij], cp_idx[ckl], cp_jdx[ckl]
            sub = max(cond[i, j], cond[k, l], cond[i, k], cond[j, k], cond[i, l], cond[j, l])
            if sub < tol:
                continue
            cutoff = tol / sub
            out.append((cij, ckl, make_s_index_offsets(lq_ij, self.nbins, cutoff),
                        make_s_index_offsets(lq_kl, self.nbins, cutoff)))
        return out

    def jk_cart(self, dmc, tol=1e-13, tasks=None):
        """J' = 2 (V_J + V_J^T), K' = V_K + V_K^T over the engine's Cartesian
        basis, like _VHFOpt.jk_cart; dmc is (n_dm, nao, nao) on the device."""
        import torch
        dmc = dmc.contiguous()
        n_dm, nao = dmc.shape[0], dmc.shape[-1]
        vj = torch.zeros_like(dmc)
        vk = torch.zeros_like(dmc)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        tp = lambda t: ctypes.c_void_p(t.data_ptr())
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        if tasks is None:
            tasks = self.tasks(dmc, tol)
        for cij, ckl, bi, bk in tasks:
            err = self.lv.GINTbuild_jk(self.bp_gpu, tp(vj), tp(vk), tp(dmc), ctypes.c_int(nao),
                                       ctypes.c_int(n_dm), vp(bi), vp(bk), ctypes.c_int(self.nbins),
                                       ctypes.c_int(cij), ctypes.c_int(ckl), stream)
            if err != 0:
                raise RuntimeError('reference GINTbuild_jk failed for class pair (%d, %d)'
                                   % (cij, ckl))
        J = 2 * (vj + vj.transpose(-1, -2))
        K = vk + vk.transpose(-1, -2)
        return J, K
