"""Three- and two-centre Coulomb integrals for density fitting on one B200.

Mirrors cuobc/lib/int3c.py:177-373, which drives the same Rys engine as the
J/K builder through GINTfill_int2e with an auxiliary basis:

* the orbital basis and the auxiliary basis are decontracted and sorted by
  (l, nprim) (``sort_mol``, int3c.py:93-118);
* a one-shell "fake" molecule holds an s function that is the constant 1
  (exponent 0, int3c.py:47-60), so that the four-index kernel evaluates
  (ij|k) = (ij|k 1) and (k|l) = (k 1|l 1);
* ``VHFOpt3c`` pairs the orbital shells among themselves and every auxiliary
  shell with the fake shell (both orientations on diagonal blocks,
  ``get_pairing``, int3c.py:121-172), keeping pairs with Schwarz factor
  above 1e-11, and builds one basis-product cache over the concatenated
  molecule [orbital | fake | auxiliary];
* ``get_int2c`` fills the auxiliary metric (k|l), transforms it to the
  caller's auxiliary basis and returns its Cholesky factor (or, for a
  numerically singular metric, the eigenvectors scaled by 1/sqrt(e) of the
  eigenvalues above a threshold) (int3c.py:283-322);
* ``get_int3c`` fills one (orbital class pair, auxiliary class) block of
  (ij|k) (int3c.py:325-368).

The Schwarz factors come from the device (BQCschwarz) instead of libcint on
the CPU.  Everything stays on the device (torch tensors).
"""
import ctypes

import numpy as np
import torch

from .. import lib as _libmod
from ..gto import mole as gto
from ..scf.hf import (_dev, _ptr, _stream, basis_cache, basis_seg_contraction,
                      free_basis_cache, schwarz_factors)

PAIR_CUTOFF = 1e-11          # get_pairing's default (int3c.py:121)
FAC_SP_S = 0.282094791773878143   # the common factor of a Cartesian s function


def make_fake_mol():
    """One atom carrying one s shell that is the constant function 1:
    exponent 0 and coefficient 1/FAC_SP_S, which the kernels' s-shell factor
    cancels (int3c.py:47-60)."""
    fake = gto.Mole([('He', (0., 0., 0.))], {'He': [[0, [1., 1.]]]}, unit='Bohr')
    fake._env[fake._bas[0, gto.PTR_EXP]] = 0.
    fake._env[fake._bas[0, gto.PTR_COEFF]] = 1. / FAC_SP_S
    fake.cart = True
    return fake


def conc_mol(m1, m2):
    """Concatenated molecule: atoms, shells and env of m1 then m2, the env
    pointers of m2 shifted (pyscf's gto.conc_mol)."""
    out = m1.copy()
    off = len(m1._env)
    atm2 = m2._atm.copy()
    atm2[:, gto.PTR_COORD] += off
    atm2[:, gto.PTR_ZETA] += off
    bas2 = m2._bas.copy()
    bas2[:, gto.ATOM_OF] += m1.natm
    bas2[:, gto.PTR_EXP] += off
    bas2[:, gto.PTR_COEFF] += off
    out._atm = np.vstack([m1._atm, atm2]).astype(np.int32)
    out._bas = np.vstack([m1._bas, bas2]).astype(np.int32)
    out._env = np.hstack([m1._env, m2._env])
    out.atom = list(m1.atom) + list(m2.atom)
    out.cart = True
    return out


def sort_mol(mol):
    """Sort the shells of a decontracted Cartesian molecule by (l, nprim)
    in place (int3c.py:93-118).  Returns (mol, ao_idx, uniq (l, nprim),
    shells per group)."""
    l_ctrs = mol._bas[:, [gto.ANG_OF, gto.NPRIM_OF]]
    uniq, inv, counts = np.unique(l_ctrs, axis=0, return_inverse=True, return_counts=True)
    order = np.argsort(np.asarray(inv).ravel(), kind='stable').astype(np.int32)
    ao_loc = mol.ao_loc_nr(cart=True)
    ao_idx = np.hstack([np.arange(ao_loc[i], ao_loc[i + 1]) for i in order])
    mol._bas = np.ascontiguousarray(mol._bas[order])
    return mol, ao_idx, uniq, counts


def _group_pairs(p_offsets, q_offsets):
    """Candidate pairs of get_pairing (int3c.py:121-172): for every bra
    group p and ket group q that starts before p, all (i, j); for q == p,
    all (i, j) of the block (both orientations).  Returns [(p, q, i, j)]."""
    out = []
    for p in range(len(p_offsets) - 1):
        p0, p1 = p_offsets[p], p_offsets[p + 1]
        for q in range(len(q_offsets) - 1):
            q0, q1 = q_offsets[q], q_offsets[q + 1]
            if q0 < p0 or (q0 == p0 and q1 == p1):
                i, j = np.meshgrid(np.arange(p0, p1), np.arange(q0, q1), indexing='ij')
                out.append((p, q, i.ravel().astype(np.int32), j.ravel().astype(np.int32)))
    return out


class VHFOpt3c:
    """Pair lists and basis-product cache of the 3-centre integrals
    (VHFOpt3c, int3c.py:175-280) over [orbital | fake | auxiliary] shells.

    After build(): coeff (nao_cart_sorted, nao) and auxcoeff (naux_cart_sorted,
    naux) map the sorted decontracted Cartesian functions to the caller's
    bases; log_qs / aux_log_qs hold the pair classes of orbital pairs and of
    (auxiliary, fake) pairs; l_ctr_offsets / aux_l_ctr_offsets the shell
    groups."""

    def __init__(self, mol, auxmol):
        self.mol, self.coeff = basis_seg_contraction(mol)
        self.auxmol, self.auxcoeff = basis_seg_contraction(auxmol)
        self._bp = None

    def build(self, cutoff=PAIR_CUTOFF):
        mol, ao_idx, uniq, counts = sort_mol(self.mol)
        self.coeff = self.coeff[ao_idx]
        fake, _, _, fake_counts = sort_mol(make_fake_mol())
        aux, aux_idx, aux_uniq, aux_counts = sort_mol(self.auxmol)
        self.auxcoeff = self.auxcoeff[aux_idx]
        tot = conc_mol(mol, conc_mol(fake, aux))
        self.tot_mol = tot
        if tot._bas[:, gto.ANG_OF].max() > 3:
            raise NotImplementedError('shells beyond f are not supported on the device')
        offs = np.append(0, np.cumsum(counts))
        fake_offs = np.append(0, np.cumsum(fake_counts)) + offs[-1]
        aux_offs = np.append(0, np.cumsum(aux_counts))
        self.aux_l_ctr_offsets = aux_offs.copy()
        aux_offs_tot = aux_offs + fake_offs[-1]
        cand = _group_pairs(offs, offs) + _group_pairs(aux_offs_tot, fake_offs)
        norb_classes = len(_group_pairs(offs, offs))
        # Schwarz factors of every candidate pair (diagonal factor 1: both
        # orientations of a diagonal block are kept)
        qs = schwarz_factors(tot, [(i, j) for _, _, i, j in cand], 1.)
        bra, ket, log_qs, self.class_groups = [], [], [], []
        for (p, q, i, j), qv in zip(cand, qs):
            o = np.argsort(-qv, kind='stable')
            keep = qv[o] > cutoff
            bra.append(i[o][keep])
            ket.append(j[o][keep])
            log_qs.append(np.minimum(np.log(qv[o][keep]), 0.))
            self.class_groups.append((p, q))
        self.log_qs = log_qs[:norb_classes]
        self.aux_log_qs = log_qs[norb_classes:]
        self.l_ctr_offsets = offs
        self.bas_pair2shls = np.ascontiguousarray(np.vstack([np.hstack(bra), np.hstack(ket)]),
                                                  dtype=np.int32)
        self.bas_pairs_locs = np.append(0, np.cumsum([len(b) for b in bra])).astype(np.int32)
        self.ncptype = len(bra)
        self._bp = basis_cache(tot, self.bas_pair2shls, self.bas_pairs_locs, self.ncptype, 1.)
        self.ao_loc = mol.ao_loc_nr(cart=True)
        self.aux_ao_loc = aux.ao_loc_nr(cart=True)
        self.nao = int(self.ao_loc[-1])
        self.naux = int(self.aux_ao_loc[-1])
        self.coeff_dev = torch.as_tensor(self.coeff, device=_dev())
        self.auxcoeff_dev = torch.as_tensor(self.auxcoeff, device=_dev())
        return self

    @property
    def bpcache(self):
        return self._bp[1]

    def clear(self):
        if self._bp is not None:
            free_basis_cache(self._bp[0], self._bp[1])
            self._bp = None

    def __del__(self):
        try:
            self.clear()
        except Exception:
            pass


def _fill(opt, out, strides, ao_offsets, cp_ij, cp_kl, nij, nkl):
    lib = _libmod.load_library()
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    bins_ij = np.array([0, nij], dtype=np.int32)
    bins_kl = np.array([0, nkl], dtype=np.int32)
    norb = opt.nao + opt.naux + 1
    err = lib.GINTfill_int2e(ctypes.cast(opt.bpcache, ctypes.c_void_p), _ptr(out), ctypes.c_int(norb),
                             vp(strides), vp(ao_offsets), vp(bins_ij), vp(bins_kl), ctypes.c_int(1),
                             ctypes.c_int(cp_ij), ctypes.c_int(cp_kl), _stream())
    if err:
        raise RuntimeError('GINTfill_int2e failed (%d)' % err)


def get_int2c(opt, j2c_eig_always=False, linear_dep_threshold=1e-13):
    """Factor of the auxiliary Coulomb metric (int3c.py:283-322): the metric
    (k|l) over the caller's auxiliary basis, then its lower Cholesky factor
    L (metric = L L^T); with j2c_eig_always, or when the metric is not
    positive definite, the eigenvectors with eigenvalue e above
    linear_dep_threshold scaled by 1/sqrt(e)."""
    nao, naux = opt.nao, opt.naux
    # column-major (k, l): the k index has stride 1
    int2c = torch.zeros((naux, naux), dtype=torch.float64, device=_dev())
    ao_offsets = np.array([nao + 1, nao, nao + 1, nao], dtype=np.int32)
    strides = np.array([1, naux, naux, naux * naux], dtype=np.int32)
    norb_cls = len(opt.log_qs)
    for k, lq_k in enumerate(opt.aux_log_qs):
        for l, lq_l in enumerate(opt.aux_log_qs):
            if len(lq_k) == 0 or len(lq_l) == 0:
                continue
            _fill(opt, int2c, strides, ao_offsets, norb_cls + k, norb_cls + l, len(lq_k), len(lq_l))
    int2c = int2c.T                      # the filled array is (l, k) row-major
    C = opt.auxcoeff_dev
    int2c = C.T @ int2c @ C
    if not j2c_eig_always:
        L, info = torch.linalg.cholesky_ex(int2c)
        if int(info) == 0:
            return L
    e, v = torch.linalg.eigh(int2c)
    mask = e > linear_dep_threshold
    return v[:, mask] * torch.rsqrt(e[mask])[None, :]


def get_int3c(cp_ij_id, cp_aux_id, opt, out=None):
    """(ij|k) of one orbital class (pairs of groups cpi >= cpj) and one
    auxiliary class (int3c.py:325-368), as (slice_i, slice_j, slice_k,
    block) over the sorted decontracted Cartesian functions; block is
    (ni, nj, nk), i and j over the AO ranges of the two groups."""
    p, q = opt.class_groups[cp_ij_id]
    ao, aux_ao = opt.ao_loc, opt.aux_ao_loc
    offs, aoffs = opt.l_ctr_offsets, opt.aux_l_ctr_offsets
    i0, i1 = ao[offs[p]], ao[offs[p + 1]]
    j0, j1 = ao[offs[q]], ao[offs[q + 1]]
    k0, k1 = aux_ao[aoffs[cp_aux_id]], aux_ao[aoffs[cp_aux_id + 1]]
    ni, nj, nk = i1 - i0, j1 - j0, k1 - k0
    if out is None:
        out = torch.zeros((ni, nj, nk), dtype=torch.float64, device=_dev())
    else:
        out.zero_()
    ao_offsets = np.array([i0, j0, opt.nao + 1 + k0, opt.nao], dtype=np.int32)
    strides = np.array([nj * nk, nk, 1, 1], dtype=np.int32)
    nij = len(opt.log_qs[cp_ij_id])
    nk_pairs = len(opt.aux_log_qs[cp_aux_id])
    if nij and nk_pairs:
        _fill(opt, out, strides, ao_offsets, cp_ij_id, len(opt.log_qs) + cp_aux_id, nij, nk_pairs)
    return slice(i0, i1), slice(j0, j1), slice(k0, k1), out


def int3c_cart(opt):
    """All (ij|k) over the sorted decontracted Cartesian functions,
    (nao, nao, naux), assembled from the class blocks (off-diagonal group
    blocks mirrored to (ji|k))."""
    full = torch.zeros((opt.nao, opt.nao, opt.naux), dtype=torch.float64, device=_dev())
    for c in range(len(opt.log_qs)):
        p, q = opt.class_groups[c]
        for a in range(len(opt.aux_log_qs)):
            si, sj, sk, blk = get_int3c(c, a, opt)
            full[si, sj, sk] += blk
            if p != q:
                full[sj, si, sk] += blk.transpose(0, 1)
    return full


def int3c_ao(opt):
    """(ij|k) over the caller's orbital and auxiliary bases, (nao0, nao0, naux0)."""
    full = int3c_cart(opt)
    C, Ca = opt.coeff_dev, opt.auxcoeff_dev
    return torch.einsum('pqr,pi,qj,rk->ijk', full, C, C, Ca)
