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

RefVHFOpt restates the set-up of cuobc/scf/hf.py without the engine: the
basis decontraction (basis_seg_contraction, hf.py:481-564), the shell sort
by (l, nprim) and the Schwarz pair lists (_VHFOpt.build, hf.py:288-397).
pyscf is absent, so the Schwarz factors come from the CPU oracle's (ij|ij)
in place of pyscf's CVHFsetnr_direct_scf.  RefJK also accepts the engine's
own _VHFOpt, so that a test can run both builders on identical pair lists.
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


class ContractionProdType(ctypes.Structure):
    """cuobc/lib/gint/gint.h:101-107."""
    _fields_ = [('l_bra', ctypes.c_int), ('l_ket', ctypes.c_int), ('nprim_12', ctypes.c_int),
                ('npairs', ctypes.c_int)]


class BasisProdCache(ctypes.Structure):
    """cuobc/lib/gint/gint.h:118-147."""
    _fields_ = [('nbas', ctypes.c_int), ('ncptype', ctypes.c_int),
                ('cptype', ctypes.POINTER(ContractionProdType)),
                ('bas_pairs_locs', ctypes.POINTER(ctypes.c_int)),
                ('primitive_pairs_locs', ctypes.POINTER(ctypes.c_int)),
                ('bas_pair2shls', ctypes.POINTER(ctypes.c_int)),
                ('aexyz', ctypes.POINTER(ctypes.c_double)),
                ('bas_coords', ctypes.POINTER(ctypes.c_double)),
                ('bas_pair2bra', ctypes.POINTER(ctypes.c_int)),
                ('bas_pair2ket', ctypes.POINTER(ctypes.c_int)),
                ('ao_loc', ctypes.POINTER(ctypes.c_int))] + \
        [(n, ctypes.POINTER(ctypes.c_double)) for n in ('a12', 'e12', 'x12', 'y12', 'z12')]


def make_s_index_offsets(log_q, nbins, cutoff):
    """cuobc/scf/hf.py:567-578, including its bin-size limit."""
    scale = nbins / np.log(min(cutoff, .1))
    s_index = np.floor(scale * log_q).astype(np.int32)
    bins = np.bincount(s_index, minlength=nbins)[:nbins]
    if bins.size and bins.max() >= 65536 * 8:
        raise ValueError('a bin holds more pairs than the reference kernel accepts')
    return np.append(0, np.cumsum(bins)).astype(np.int32)


ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, PTR_EXP, PTR_COEFF = 0, 1, 2, 3, 5, 6


def _gto_norm(l, expnt):
    """Radial normalisation 1 / sqrt(int r^(2l+2) exp(-2 a r^2) dr)."""
    from math import gamma
    e = np.asarray(expnt, dtype=float)
    n1 = l + 1.5
    return 1. / np.sqrt(gamma(n1) / (2. * (2. * e) ** n1))


def seg_contraction(mol):
    """cuobc/scf/hf.py:481-564 (allow_replica=False): a shell with nctr > 1
    becomes nprim single-primitive shells carrying the primitive radial
    normalisation, the contraction (divided by that normalisation) moves into
    coeff; the returned molecule is Cartesian and coeff includes the
    Cartesian-to-spherical transformation of mol."""
    import copy
    env = mol._env.copy()
    bas, blocks = [], []
    for sh in mol._bas:
        l, nprim, nctr = int(sh[ANG_OF]), int(sh[NPRIM_OF]), int(sh[NCTR_OF])
        nf = (l + 1) * (l + 2) // 2
        if nctr == 1:
            bas.append(sh[None].copy())
            blocks.append(np.eye(nf))
            continue
        pexp, pcoeff = int(sh[PTR_EXP]), int(sh[PTR_COEFF])
        norm = _gto_norm(l, env[pexp:pexp + nprim])
        c = mol._env[pcoeff:pcoeff + nprim * nctr].reshape(nctr, nprim) / norm[None, :]
        # rows (primitive p, component f), columns (contraction i, component f)
        blocks.append(np.kron(c.T, np.eye(nf)))
        env[pcoeff:pcoeff + nprim] = norm
        bs = np.repeat(sh[None], nprim, axis=0)
        bs[:, NPRIM_OF] = 1
        bs[:, NCTR_OF] = 1
        bs[:, PTR_EXP] = np.arange(pexp, pexp + nprim)
        bs[:, PTR_COEFF] = np.arange(pcoeff, pcoeff + nprim)
        bas.append(bs)
    pmol = copy.copy(mol)
    pmol.cart = True
    pmol._bas = np.ascontiguousarray(np.vstack(bas), dtype=np.int32)
    pmol._env = env
    rows = sum(b.shape[0] for b in blocks)
    cols = sum(b.shape[1] for b in blocks)
    coeff = np.zeros((rows, cols))
    r = c = 0
    for b in blocks:
        coeff[r:r + b.shape[0], c:c + b.shape[1]] = b
        r += b.shape[0]
        c += b.shape[1]
    if not mol.cart:
        coeff = coeff @ mol.cart2sph_coeff()
    return pmol, coeff


class RefVHFOpt:
    """The set-up of cuobc/scf/hf.py:_VHFOpt restated without the engine:
    decontraction, sort of the shells by unique (l, nprim) (hf.py:296-320),
    Schwarz factors (the CPU oracle's sqrt max |(ij|ij)|, hf.py:341), and per
    pair of groups p >= q the shell pairs with q > cutoff sorted by
    descending q (upper triangle dropped on diagonal blocks), log q clipped
    at 0 (hf.py:343-397)."""

    def __init__(self, mol):
        self.mol0 = mol
        self.mol, self.coeff = seg_contraction(mol)

    def build(self, cutoff=1e-13, nthreads=0):
        from oracle import oracle
        mol = self.mol
        l_ctrs = mol._bas[:, [ANG_OF, NPRIM_OF]]
        uniq, inv, counts = np.unique(l_ctrs, axis=0, return_inverse=True, return_counts=True)
        inv = np.asarray(inv).ravel()
        order = np.argsort(inv, kind='stable')
        ao_loc = mol.ao_loc_nr(cart=True)
        ao_idx = np.hstack([np.arange(ao_loc[i], ao_loc[i + 1]) for i in order])
        self.coeff = self.coeff[ao_idx]
        mol._bas = np.ascontiguousarray(mol._bas[order])
        self.direct_scf_tol = cutoff
        q_cond = oracle.q_cond(mol)
        offs = np.append(0, np.cumsum(counts))
        bra, ket, log_qs = [], [], []
        for i in range(len(uniq)):
            p0, p1 = offs[i], offs[i + 1]
            for j in range(i + 1):
                q0, q1 = offs[j], offs[j + 1]
                sub = q_cond[p0:p1, q0:q1].ravel()
                idx = sub.argsort()[::-1]
                qs = sub[idx]
                ish, jsh = np.unravel_index(idx, (p1 - p0, q1 - q0))
                mask = qs > cutoff
                if i == j:
                    mask &= ish >= jsh
                bra.append(ish[mask] + p0)
                ket.append(jsh[mask] + q0)
                log_qs.append(np.minimum(np.log(qs[mask]), 0.))
        self.uniq_l_ctr = uniq
        self.l_ctr_offsets = offs
        self.log_qs = log_qs
        self.ncptype = len(log_qs)
        self.bas_pair2shls = np.ascontiguousarray(np.vstack([np.hstack(bra), np.hstack(ket)]),
                                                  dtype=np.int32)
        self.bas_pairs_locs = np.append(0, np.cumsum([len(b) for b in bra])).astype(np.int32)
        return self


class RefJK:
    """The reference J/K builder (its libgint/libgvhf) over the pair lists of
    a RefVHFOpt, or over the engine's sorted, decontracted basis and lists
    (padding pairs removed, reference order restored)."""

    def __init__(self, opt, device='cuda', libs=None):
        """libs: (libgint, libgvhf) to drive; default the reference's own from
        oracle/_ref.  A test passes this package's library for both to run
        it as the drop-in under the reference's host logic."""
        import torch
        lg, lv = load() if libs is None else libs
        self.lg, self.lv = lg, lv
        self.opt = opt
        pmol = opt.mol
        if isinstance(opt, RefVHFOpt):
            dev = torch.device(device)
            self.pair2shls = opt.bas_pair2shls
            self.pairs_locs = opt.bas_pairs_locs
            self.log_qs = opt.log_qs
        else:
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
        self.device = dev
        self.ncptype = opt.ncptype
        self.atm = np.ascontiguousarray(pmol._atm, dtype=np.int32)
        self.bas = np.ascontiguousarray(pmol._bas, dtype=np.int32)
        self.env = np.ascontiguousarray(pmol._env)
        self.bas_coords = np.empty(pmol.nbas * 3)
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        tp = lambda t: ctypes.c_void_p(t.data_ptr())
        bp = ctypes.POINTER(BasisProdCache)()
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
        self.bp_gpu = ctypes.POINTER(BasisProdCache)()
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
