"""Direct-SCF J/K builder and restricted/unrestricted Hartree-Fock on one B200.

Mirrors the interface of the reference module cuobc/scf/hf.py:

* ``get_jk(mol, dm, hermi=1, vhfopt=None, with_j=True, with_k=True, omega=None,
  verbose=None, group_size=None, gpus=None, prescreen=True, nbins=None)``
  (hf.py:53-227): same arguments, same return convention (host numpy arrays of
  the shape of ``dm``), same errors (``NotImplementedError`` for hermi != 1 or
  omega, ``RuntimeError`` for a nonzero library status);
* ``_VHFOpt`` (hf.py:277-448): basis decontraction and sort, Schwarz pair lists,
  device cache;
* ``RHF`` (hf.py:272-274) with ``get_jk`` and ``_eigh`` (``eig``, hf.py:253-265);
* ``UHF``, which the reference lacks, built on the n_dm batch dimension.

Device memory is held in torch tensors; the kernels are reached through the
C ABI of libbyteqc_b200 (include/byteqc_b200.h).  Unlike the reference, one
library call covers every class pair of a build, the density screening is
per quartet on the device, and the SCF loop (Fock build, DIIS, eigensolver,
energy) runs on the device too.
"""
import ctypes
import math
import time

import numpy as np
import torch

from .. import lib as _libmod
from ..gto import mole as gto

LMAX_ON_GPU = 3


def _dev():
    if not torch.cuda.is_available():
        raise RuntimeError('byteqc_b200 needs a CUDA device (no CPU fallback)')
    return torch.device('cuda', torch.cuda.current_device())


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def basis_seg_contraction(mol):
    """Decontract generally contracted shells into primitive shells.

    Returns (pmol, coeff): a Cartesian molecule whose shells each hold one
    contraction, and coeff (nao_cart(pmol), mol.nao) with AO = pmol AO @ coeff.
    Same transformation as cuobc/scf/hf.py:481-564: shells with nctr == 1 are
    kept; a shell with nctr > 1 becomes nprim single-primitive shells with the
    radial normalisation of each primitive, and the contraction coefficients
    (divided by that normalisation) move into coeff.  coeff includes the
    Cartesian-to-spherical transformation unless mol.cart.
    """
    bas_out = []
    env = mol._env.copy()
    blocks = []
    for shell in mol._bas:
        l, nprim, nctr = shell[gto.ANG_OF], shell[gto.NPRIM_OF], shell[gto.NCTR_OF]
        nf = gto.ncart(l)
        if nctr == 1:
            bas_out.append(shell.copy())
            blocks.append(np.eye(nf))
            continue
        pexp, pcoeff = shell[gto.PTR_EXP], shell[gto.PTR_COEFF]
        exps = env[pexp:pexp + nprim]
        norm = gto.gto_norm(l, exps)
        c = mol._env[pcoeff:pcoeff + nprim * nctr].reshape(nctr, nprim)
        # block[(p, f), (i, f')] = delta_ff' c[i, p] / norm[p]
        blk = np.einsum('ip,p,ef->pfie', c, 1. / norm, np.eye(nf)).reshape(nprim * nf, nctr * nf)
        blocks.append(blk)
        env[pcoeff:pcoeff + nprim] = norm
        for p in range(nprim):
            s = shell.copy()
            s[gto.NPRIM_OF] = 1
            s[gto.NCTR_OF] = 1
            s[gto.PTR_EXP] = pexp + p
            s[gto.PTR_COEFF] = pcoeff + p
            bas_out.append(s)
    pmol = mol.copy()
    pmol.cart = True
    pmol._bas = np.asarray(bas_out, dtype=np.int32).reshape(-1, gto.BAS_SLOTS)
    pmol._env = env
    nr = sum(b.shape[0] for b in blocks)
    nc = sum(b.shape[1] for b in blocks)
    coeff = np.zeros((nr, nc))
    r0 = c0 = 0
    for b in blocks:
        coeff[r0:r0 + b.shape[0], c0:c0 + b.shape[1]] = b
        r0 += b.shape[0]
        c0 += b.shape[1]
    if not mol.cart:
        coeff = coeff @ mol.cart2sph_coeff()
    return pmol, coeff


def _make_s_index_offsets(log_q, nbins=10, cutoff=1e-12):
    """Bin sorted log q into nbins down to cutoff (cuobc/scf/hf.py:567-578)."""
    scale = nbins / np.log(min(cutoff, .1))
    s_index = np.floor(scale * log_q).astype(np.int32)
    bins = np.bincount(s_index, minlength=nbins)[:nbins]
    return np.append(0, np.cumsum(bins)).astype(np.int32)


PAIR_TILE = 16


def _tiles_by_first_q(tb, tk, tq, dummy):
    """Sort the pairs inside each tile by q descending, then the tiles by
    their first (largest) q, stably."""
    oi = np.argsort(-tq, axis=1, kind='stable')
    rows = np.arange(len(tq))[:, None]
    tb, tk, tq, dummy = tb[rows, oi], tk[rows, oi], tq[rows, oi], dummy[rows, oi]
    ot = np.argsort(-tq[:, 0], kind='stable')
    return tb[ot].ravel(), tk[ot].ravel(), tq[ot].ravel(), dummy[ot].ravel()


def _tile_order(bra, ket, q, layout='q'):
    """Order the pairs of one class in tiles of PAIR_TILE pairs.

    layout 'q': all pairs sorted by q descending, the last tile padded with
    pairs of q = 0.  Every tile spans a narrow range of q, so almost every
    quartet of a launched tile pair passes the device screen.
    layout 'shell': tiles of pairs that share the bra shell: pairs grouped by
    bra shell, sorted by q descending within a group, cut into tiles (the
    last tile of a group padded), tiles sorted by their largest q.  A J/K
    kernel can then sum the K contributions that share a shell across the
    tile before its atomics, but small groups leave tiles mostly padding.

    layout 'hybrid': the full tiles of the 'shell' layout (bra-shell groups
    of at least PAIR_TILE pairs), all remaining pairs packed in the 'q'
    layout, tiles sorted by their largest q.

    In every layout q is descending within a tile and the first q of every
    tile is descending along the list, which keeps the tile pruning of
    BQCbuild_jk valid.  Returns (bra, ket, q, is_padding)."""
    n = len(q)
    if n == 0 and layout in ('q', 'hybrid'):
        return bra, ket, q, np.zeros(0, bool)
    if layout in ('q', 'hybrid'):
        if layout == 'hybrid':
            o = np.lexsort((-q, bra))
            starts = np.flatnonzero(np.r_[True, bra[o][1:] != bra[o][:-1]])
            sizes = np.diff(np.r_[starts, n])
            gid = np.repeat(np.arange(len(starts)), sizes)
            rank = np.arange(n) - starts[gid]
            full = o[rank < (sizes[gid] // PAIR_TILE) * PAIR_TILE]
            rest = o[rank >= (sizes[gid] // PAIR_TILE) * PAIR_TILE]
        else:
            full = np.zeros(0, np.int64)
            rest = np.arange(n)
        rest = rest[np.argsort(-q[rest], kind='stable')]
        pad = (-len(rest)) % PAIR_TILE
        idx = np.r_[full, rest, np.full(pad, rest[-1] if len(rest) else 0)].astype(np.int64)
        tb = bra[idx].reshape(-1, PAIR_TILE)
        tk = ket[idx].reshape(-1, PAIR_TILE)
        tq = np.r_[q[idx[:n]], np.zeros(pad)].reshape(-1, PAIR_TILE)
        dummy = np.r_[np.zeros(n, bool), np.ones(pad, bool)].reshape(-1, PAIR_TILE)
        return _tiles_by_first_q(tb, tk, tq, dummy)
    if layout != 'shell':
        raise ValueError('unknown tile layout %r' % layout)
    n = len(q)
    if n == 0:
        return bra, ket, q, np.zeros(0, bool)
    order = np.lexsort((-q, bra))
    b, k, qq = bra[order], ket[order], q[order]
    starts = np.flatnonzero(np.r_[True, b[1:] != b[:-1]])
    sizes = np.diff(np.r_[starts, n])
    gid = np.repeat(np.arange(len(starts)), sizes)
    rank = np.arange(n) - starts[gid]
    ntile_g = (sizes + PAIR_TILE - 1) // PAIR_TILE
    tile_off = np.r_[0, np.cumsum(ntile_g)[:-1]]
    tile = tile_off[gid] + rank // PAIR_TILE
    slot = rank % PAIR_TILE
    ntile = int(ntile_g.sum())
    first = slot == 0
    tq = np.empty(ntile)
    tq[tile[first]] = qq[first]
    tb = np.empty(ntile, dtype=b.dtype)
    tb[tile[first]] = b[first]
    tk = np.empty(ntile, dtype=k.dtype)
    tk[tile[first]] = k[first]
    pos = np.empty(ntile, dtype=np.int64)
    pos[np.argsort(-tq, kind='stable')] = np.arange(ntile)
    out_b = np.repeat(tb[np.argsort(pos)], PAIR_TILE)
    out_k = np.repeat(tk[np.argsort(pos)], PAIR_TILE)
    out_q = np.zeros(ntile * PAIR_TILE)
    dummy = np.ones(ntile * PAIR_TILE, bool)
    dst = pos[tile] * PAIR_TILE + slot
    out_b[dst] = b
    out_k[dst] = k
    out_q[dst] = qq
    dummy[dst] = False
    return out_b, out_k, out_q, dummy


def schwarz_factors(mol, pair_lists, diag_fac):
    """Schwarz factors sqrt(max |(ij|ij)|) of every pair of the given lists,
    one list (bra shells, ket shells) per class of pairs sharing
    (l, nprim) on each side, computed on the device (BQCschwarz); the e12
    diagonal factor diag_fac is undone.  Returns one array per list."""
    lib = _libmod.load_library()
    ncptype = len(pair_lists)
    locs = np.append(0, np.cumsum([len(x[0]) for x in pair_lists])).astype(np.int32)
    p2s = np.vstack([np.hstack([x[0] for x in pair_lists]),
                     np.hstack([x[1] for x in pair_lists])]).astype(np.int32)
    bp_cpu, bp_gpu, mem, keep = basis_cache(mol, p2s, locs, ncptype, diag_fac)
    q_all = torch.zeros(max(int(locs[-1]), 1), dtype=torch.float64, device=_dev())
    for c in range(ncptype):
        if locs[c + 1] > locs[c]:
            err = lib.BQCschwarz(bp_gpu, ctypes.c_int(c), ctypes.c_double(diag_fac),
                                 _ptr(q_all[locs[c]:]), _stream())
            if err:
                raise RuntimeError('BQCschwarz failed (%d)' % err)
    q_all = q_all.cpu().numpy()
    free_basis_cache(bp_cpu, bp_gpu)
    del mem, keep
    return [q_all[locs[c]:locs[c + 1]] for c in range(ncptype)]


def make_plan(bp_gpu, pair_q_host, pair_mol_host=None):
    """The device schedule of J/K builds over a basis-product cache
    (BQCplan_create); released with BQCplan_destroy before the cache."""
    lib = _libmod.load_library()
    plan = ctypes.c_void_p()
    mol = pair_mol_host.ctypes.data_as(ctypes.c_void_p) if pair_mol_host is not None else None
    err = lib.BQCplan_create(ctypes.cast(bp_gpu, ctypes.c_void_p),
                             pair_q_host.ctypes.data_as(ctypes.c_void_p), mol, ctypes.byref(plan))
    if err:
        raise RuntimeError('BQCplan_create failed (%d)' % err)
    return plan


def free_basis_cache(bp_cpu, bp_gpu):
    """Release both structs.  The device copy shares the host blocks of
    the cpu cache, so deleting it frees them (cuobc/scf/hf.py:439-442
    deletes only that copy); the cpu struct is then released with its
    shared pointers cleared."""
    lib = _libmod.load_library()
    shared = bool(bp_gpu)
    if shared:
        lib.GINTdel_basis_prod(ctypes.byref(bp_gpu))
    if bp_cpu:
        if shared:
            c = bp_cpu.contents
            c.cptype = None
            c.primitive_pairs_locs = None
            c.aexyz = None
        lib.GINTdel_basis_prod(ctypes.byref(bp_cpu))


def basis_cache(mol, pair2shls, pairs_locs, ncptype, diag_fac, dummy=None):
    """The basis-product cache of a pair list (GINTinit_basis_prod_cpu, then
    GINTinit_basis_prod_gpu on device copies of ao_loc, shell coordinates,
    primitive-pair block and pair list, as cuobc/scf/hf.py:410-437).  Pairs
    flagged in dummy get e12 = 0.  Returns (cpu cache, device cache, device
    buffers, host arrays the caches borrow)."""
    lib = _libmod.load_library()
    bp_cpu = ctypes.POINTER(_libmod.BasisProdCache)()
    bas_coords = np.empty(mol.nbas * 3)
    pair2shls = np.ascontiguousarray(pair2shls, dtype=np.int32)
    pairs_locs = np.ascontiguousarray(pairs_locs, dtype=np.int32)
    atm = np.ascontiguousarray(mol._atm, dtype=np.int32)
    bas = np.ascontiguousarray(mol._bas, dtype=np.int32)
    env = np.ascontiguousarray(mol._env)
    lib.GINTinit_basis_prod_cpu(
        ctypes.byref(bp_cpu), ctypes.c_double(diag_fac),
        bas_coords.ctypes.data_as(ctypes.c_void_p),
        pair2shls.ctypes.data_as(ctypes.c_void_p), pairs_locs.ctypes.data_as(ctypes.c_void_p),
        ctypes.c_int(ncptype), atm.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(mol.natm),
        bas.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(mol.nbas),
        env.ctypes.data_as(ctypes.c_void_p))
    nprim = bp_cpu.contents.primitive_pairs_locs[ncptype]
    aexyz = np.ctypeslib.as_array(bp_cpu.contents.aexyz, (max(nprim, 1) * 5,)).copy()
    if dummy is not None and dummy.any():
        # padding pairs contribute exactly zero: e12 = 0 for all their primitives
        e12 = aexyz[nprim:2 * nprim]
        for c in range(ncptype):
            p0, p1 = pairs_locs[c], pairs_locs[c + 1]
            d = np.flatnonzero(dummy[p0:p1])
            if len(d):
                n12 = bp_cpu.contents.cptype[c].nprim_12
                base = bp_cpu.contents.primitive_pairs_locs[c]
                idx = (base + d[:, None] * n12 + np.arange(n12)[None, :]).ravel()
                e12[idx] = 0.
    dev = _dev()
    mem = {
        'ao_loc': torch.as_tensor(mol.ao_loc_nr(cart=True), dtype=torch.int32, device=dev),
        'bas_coords': torch.as_tensor(bas_coords, device=dev),
        'aexyz': torch.as_tensor(aexyz, device=dev),
        'pair2shls': torch.as_tensor(pair2shls.ravel(), device=dev),
    }
    bp_gpu = ctypes.POINTER(_libmod.BasisProdCache)()
    lib.GINTinit_basis_prod_gpu(ctypes.byref(bp_cpu), ctypes.byref(bp_gpu),
                                _ptr(mem['ao_loc']), _ptr(mem['bas_coords']),
                                _ptr(mem['aexyz']), _ptr(mem['pair2shls']))
    # keep host arrays alive: the cache borrows them
    keep = (pair2shls, pairs_locs, atm, bas, env)
    return bp_cpu, bp_gpu, mem, keep


class _VHFOpt:
    """Basis sort, Schwarz pair lists and the device basis-product cache.

    build() follows cuobc/scf/hf.py:288-408: shells are grouped by unique
    (l, nprim); for every pair of groups p >= q the shell pairs (ish in p,
    jsh in q; ish >= jsh on a diagonal block) with q_ij > cutoff are kept,
    sorted by q_ij descending.  The Schwarz factors q_ij are computed on the
    device (BQCschwarz) instead of by libcint on the CPU.
    """

    def __init__(self, mol, intor='int2e', prescreen='CVHFnoscreen',
                 qcondname='CVHFsetnr_direct_scf', dmcondname=None):
        self.mol0 = mol
        self.mol, self.coeff = basis_seg_contraction(mol)
        self._intor = intor
        self.direct_scf_tol = 1e-13
        # pair layout of the tiles (see _tile_order)
        self.tile_layout = 'hybrid'
        self._bp_cpu = None
        self._bp_gpu = None

    # -- helpers ---------------------------------------------------------------
    def _init_cache(self, pair2shls, pairs_locs, ncptype, diag_fac, dummy=None):
        return basis_cache(self.mol, pair2shls, pairs_locs, ncptype, diag_fac, dummy)

    def _free_cache(self, bp_cpu, bp_gpu):
        free_basis_cache(bp_cpu, bp_gpu)

    # -- build -----------------------------------------------------------------
    def build(self, cutoff=1e-13, group_size=None, diag_block_with_triu=False, gpus=None):
        lib = _libmod.load_library()
        mol = self.mol
        self.direct_scf_tol = cutoff
        l_ctrs = mol._bas[:, [gto.ANG_OF, gto.NPRIM_OF]]
        if l_ctrs[:, 0].max() > LMAX_ON_GPU:
            raise NotImplementedError('shells beyond f are not supported on the device')
        uniq_l_ctr, inv_idx, l_ctr_counts = np.unique(l_ctrs, axis=0, return_inverse=True,
                                                     return_counts=True)
        inv_idx = inv_idx.ravel()
        sorted_idx = np.argsort(inv_idx, kind='stable').astype(np.int32)
        ao_loc = mol.ao_loc_nr(cart=True)
        ao_idx = np.hstack([np.arange(ao_loc[i], ao_loc[i + 1]) for i in sorted_idx])
        self.coeff = self.coeff[ao_idx]
        mol._bas = mol._bas[sorted_idx]
        self.uniq_l_ctr = uniq_l_ctr
        self.l_ctr_offsets = np.append(0, np.cumsum(l_ctr_counts))
        offs = self.l_ctr_offsets
        scale_diag = 1. if diag_block_with_triu else .5

        # pass 1: every pair of every class, Schwarz factors on the device
        pair_lists = []
        for p in range(len(uniq_l_ctr)):
            p0, p1 = offs[p], offs[p + 1]
            for q in range(p + 1):
                q0, q1 = offs[q], offs[q + 1]
                i, j = np.meshgrid(np.arange(p0, p1), np.arange(q0, q1), indexing='ij')
                i, j = i.ravel(), j.ravel()
                if p == q and not diag_block_with_triu:
                    m = i >= j
                    i, j = i[m], j[m]
                pair_lists.append((i, j))
        q_all = schwarz_factors(mol, pair_lists, scale_diag)

        # pass 2: keep q > cutoff and lay every class out in tiles of 16 pairs
        # (see _tile_order)
        ncptype = len(pair_lists)
        pair2bra, pair2ket, qs, log_qs, dummies = [], [], [], [], []
        for c in range(ncptype):
            b, k = pair_lists[c]
            q = q_all[c]
            keep = q > cutoff
            b, k, q = b[keep].astype(np.int32), k[keep].astype(np.int32), q[keep]
            b, k, q, dummy = _tile_order(b, k, q, self.tile_layout)
            pair2bra.append(b)
            pair2ket.append(k)
            qs.append(q)
            dummies.append(dummy)
            with np.errstate(divide='ignore'):
                lq = np.log(np.maximum(q, cutoff)) if len(q) else np.zeros(0)
            log_qs.append(np.minimum(lq, 0))
        self.log_qs = log_qs
        self.bas_pairs_locs = np.append(0, np.cumsum([len(x) for x in pair2bra])).astype(np.int32)
        self.bas_pair2shls = np.vstack([np.hstack(pair2bra), np.hstack(pair2ket)]).astype(np.int32)
        self.pair_dummy = np.hstack(dummies) if dummies else np.zeros(0, bool)
        self.ncptype = ncptype
        self._bp_cpu, self._bp_gpu, self._mem, self._keep = self._init_cache(
            self.bas_pair2shls, self.bas_pairs_locs, ncptype, scale_diag, self.pair_dummy)
        self.pair_q_host = np.ascontiguousarray(np.hstack(qs) if qs else np.zeros(1))
        self.pair_q = torch.as_tensor(self.pair_q_host, device=_dev())
        self.coeff_dev = torch.as_tensor(self.coeff, device=_dev())
        self.nao_cart = int(self.coeff.shape[0])
        self.cptype = [(self._bp_cpu.contents.cptype[c].l_bra, self._bp_cpu.contents.cptype[c].l_ket,
                        self._bp_cpu.contents.cptype[c].nprim_12,
                        self._bp_cpu.contents.cptype[c].npairs) for c in range(ncptype)]
        self._plan = make_plan(self._bp_gpu, self.pair_q_host)
        return self

    @property
    def bpcache(self):
        return self._bp_gpu

    def clear(self):
        if getattr(self, '_plan', None):
            _libmod.load_library().BQCplan_destroy(self._plan)
            self._plan = None
        if self._bp_cpu is not None:
            self._free_cache(self._bp_cpu, self._bp_gpu)
            self._bp_cpu = self._bp_gpu = None

    def __del__(self):
        try:
            self.clear()
        except Exception:
            pass

    # -- device J/K ------------------------------------------------------------
    def jk_cart(self, dmc, with_j=True, with_k=True, tol=None, fp32_below=0.):
        """V_J, V_K contributions over the internal Cartesian basis.

        dmc: (n_dm, nao_cart, nao_cart) device tensor (symmetric densities).
        Returns device tensors J', K' (already symmetrised: J' = 2(V+V^T),
        K' = V + V^T) or None for a disabled output.
        """
        lib = _libmod.load_library()
        n_dm, nao = dmc.shape[0], dmc.shape[-1]
        dmc = dmc.contiguous()
        dm_cond = torch.empty((self.mol.nbas, self.mol.nbas), dtype=torch.float64,
                              device=dmc.device)
        err = lib.BQCdm_cond(_ptr(dmc), ctypes.c_int(n_dm), ctypes.c_int(nao),
                             _ptr(self._mem['ao_loc']), ctypes.c_int(self.mol.nbas),
                             _ptr(dm_cond), _stream())
        if err:
            raise RuntimeError('BQCdm_cond failed (%d)' % err)
        vj = torch.zeros_like(dmc) if with_j else None
        vk = torch.zeros_like(dmc) if with_k else None
        tol = self.direct_scf_tol if tol is None else tol
        # the device-scheduled build: no host round trip, no allocation
        err = lib.BQCbuild_jk_plan(self._plan, _ptr(self.pair_q), _ptr(dm_cond), _ptr(vj), _ptr(vk),
                                   _ptr(dmc), nao, n_dm, tol, fp32_below, _stream())
        if err:
            raise RuntimeError('BQCbuild_jk_plan failed (%d)' % err)
        if vj is not None:
            vj = 2. * (vj + vj.transpose(-1, -2))
        if vk is not None:
            vk = vk + vk.transpose(-1, -2)
        return vj, vk

    def jk_ao(self, dm, with_j=True, with_k=True, **kw):
        """J, K in the AO basis of the original molecule for device densities
        dm (n_dm, nao0, nao0)."""
        C = self.coeff_dev
        dmc = torch.matmul(torch.matmul(C, dm), C.T)
        vj, vk = self.jk_cart(dmc, with_j, with_k, **kw)
        if vj is not None:
            vj = torch.matmul(torch.matmul(C.T, vj), C)
        if vk is not None:
            vk = torch.matmul(torch.matmul(C.T, vk), C)
        return vj, vk

    # -- one-electron integrals --------------------------------------------------
    def int1e(self):
        """Overlap, kinetic and nuclear attraction in the AO basis (device)."""
        lib = _libmod.load_library()
        mol = self.mol
        dev = _dev()
        n = self.nao_cart
        atm = torch.as_tensor(np.ascontiguousarray(mol._atm), device=dev)
        bas = torch.as_tensor(np.ascontiguousarray(mol._bas), device=dev)
        env = torch.as_tensor(np.ascontiguousarray(mol._env), device=dev)
        S = torch.zeros((n, n), dtype=torch.float64, device=dev)
        T = torch.zeros_like(S)
        V = torch.zeros_like(S)
        err = lib.BQCint1e(_ptr(atm), ctypes.c_int(mol.natm), _ptr(bas), ctypes.c_int(mol.nbas),
                           _ptr(env), _ptr(self._mem['ao_loc']), ctypes.c_int(n), _ptr(S),
                           _ptr(T), _ptr(V), _stream())
        if err:
            raise RuntimeError('BQCint1e failed (%d)' % err)
        C = self.coeff_dev
        tr = lambda M: torch.matmul(torch.matmul(C.T, M), C)
        return tr(S), tr(T), tr(V)


def get_jk(mol, dm, hermi=1, vhfopt=None, with_j=True, with_k=True, omega=None,
           verbose=None, group_size=None, gpus=None, prescreen=True, nbins=None, fp32_below=0.,
           tol=None):
    """Coulomb and exchange matrices for symmetric densities (host arrays in/out).

    Same signature and return convention as cuobc/scf/hf.py:53-227.
    ``prescreen=False`` disables the density screening (Schwarz only).
    ``fp32_below`` (an addition, default 0 = all FP64) evaluates the quartets
    whose bound q_ij q_kl max|D| is below it in FP32; ``tol`` (an addition)
    overrides the screening threshold of vhfopt.
    """
    if hermi != 1:
        raise NotImplementedError('JK-builder only supports hermitian density matrix')
    if omega is not None:
        raise NotImplementedError('Range separated Coulomb integrals')
    if vhfopt is None:
        vhfopt = _VHFOpt(mol, 'int2e').build(group_size=group_size)
    dm0 = np.asarray(dm) if not torch.is_tensor(dm) else dm
    nao0 = vhfopt.coeff.shape[1]
    dms = torch.as_tensor(dm0, dtype=torch.float64, device=_dev()).reshape(-1, nao0, nao0)
    if prescreen:
        vj, vk = vhfopt.jk_ao(dms, with_j, with_k, fp32_below=fp32_below, tol=tol)
    else:
        C = vhfopt.coeff_dev
        dmc = torch.matmul(torch.matmul(C, dms), C.T)
        vj, vk = _jk_schwarz_only(vhfopt, dmc, with_j, with_k)
        if vj is not None:
            vj = torch.matmul(torch.matmul(C.T, vj), C)
        if vk is not None:
            vk = torch.matmul(torch.matmul(C.T, vk), C)
    shape = dm0.shape
    vj = vj.reshape(shape).cpu().numpy() if vj is not None else None
    vk = vk.reshape(shape).cpu().numpy() if vk is not None else None
    return vj, vk


def _jk_schwarz_only(vhfopt, dmc, with_j, with_k):
    lib = _libmod.load_library()
    n_dm, nao = dmc.shape[0], dmc.shape[-1]
    vj = torch.zeros_like(dmc) if with_j else None
    vk = torch.zeros_like(dmc) if with_k else None
    err = lib.BQCbuild_jk(ctypes.cast(vhfopt.bpcache, ctypes.c_void_p), _ptr(vhfopt.pair_q),
                          vhfopt.pair_q_host.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(0),
                          ctypes.c_double(1.), _ptr(vj),
                          _ptr(vk), _ptr(dmc.contiguous()), ctypes.c_int(nao), ctypes.c_int(n_dm),
                          ctypes.c_double(vhfopt.direct_scf_tol ** 2), ctypes.c_double(0.),
                          ctypes.c_void_p(0), _stream())
    if err:
        raise RuntimeError('BQCbuild_jk failed (%d)' % err)
    if vj is not None:
        vj = 2. * (vj + vj.transpose(-1, -2))
    if vk is not None:
        vk = vk + vk.transpose(-1, -2)
    return vj, vk


def orthogonalizer(s):
    """The canonical orthogonalisation of the overlap s: its eigenvectors
    scaled by 1/sqrt(eigenvalue), zero columns for eigenvalues below 1e-15
    (cuobc/scf/hf.py:253-265)."""
    s = torch.as_tensor(s, device=_dev())
    seig, t = torch.linalg.eigh(s)
    inv = torch.where(seig < 1e-15, torch.zeros_like(seig), 1. / torch.sqrt(seig))
    return t * inv


def eig(h, s, t=None):
    """Generalized eigenproblem h C = s C e by canonical orthogonalisation
    (cuobc/scf/hf.py:253-265), on the device; t: the orthogonalizer of s
    when the caller already has it."""
    h = torch.as_tensor(h, device=_dev())
    if t is None:
        t = orthogonalizer(s)
    e, c = torch.linalg.eigh(t.T @ h @ t)
    return e, t @ c


class _SCFBase:
    """Shared SCF machinery (device-resident Fock build, DIIS, eigensolver)."""

    def __init__(self, mol):
        self.mol = mol
        self.conv_tol = 1e-9
        self.max_cycle = 60
        self.direct_scf_tol = 1e-13
        self.diis_space = 8
        self.init_guess = 'sad'
        self.verbose = 0
        self.converged = False
        self.e_tot = 0.
        self.cycles = 0
        self.timings = {}
        self._opt_gpu = None
        self._int1e = None

    # -- pyscf-style hooks -----------------------------------------------------
    @property
    def opt(self):
        if self._opt_gpu is None:
            self._opt_gpu = _VHFOpt(self.mol, 'int2e').build(self.direct_scf_tol)
        return self._opt_gpu

    def get_jk(self, mol=None, dm=None, hermi=1, with_j=True, with_k=True, omega=None):
        """Drop-in of cuobc/scf/hf.py:230-250 (host arrays)."""
        if omega is not None:
            raise NotImplementedError('Range separated Coulomb integrals')
        return get_jk(mol or self.mol, dm, hermi, self.opt, with_j, with_k)

    def _eigh(self, h, s):
        # the overlap does not change during an SCF: its orthogonalizer is
        # computed once per overlap object (the reference recomputes it in
        # every call of eig)
        cached = getattr(self, '_orth', None)
        if cached is None or cached[0] is not s:
            cached = self._orth = (s, orthogonalizer(s))
        return eig(h, s, cached[1])

    def get_ovlp(self):
        return self._ints()[0]

    def get_hcore(self):
        S, T, V = self._ints()
        return T + V

    def _ints(self):
        if self._int1e is None:
            self._int1e = self.opt.int1e()
        return self._int1e

    def energy_nuc(self):
        return self.mol.energy_nuc()

    # -- DIIS ------------------------------------------------------------------
    def _diis_reset(self):
        self._diis_f, self._diis_e = [], []

    def _diis(self, F, err):
        self._diis_f.append(F)
        self._diis_e.append(err)
        self._diis_f = self._diis_f[-self.diis_space:]
        self._diis_e = self._diis_e[-self.diis_space:]
        n = len(self._diis_f)
        if n < 2:
            return F
        E = torch.stack([e.reshape(-1) for e in self._diis_e])
        B = torch.empty((n + 1, n + 1), dtype=torch.float64, device=F.device)
        B[:n, :n] = E @ E.T
        B[n, :n] = -1
        B[:n, n] = -1
        B[n, n] = 0
        rhs = torch.zeros(n + 1, dtype=torch.float64, device=F.device)
        rhs[n] = -1
        try:
            c = torch.linalg.solve(B, rhs)[:n]
        except RuntimeError:
            return F
        return torch.einsum('i,i...->...', c, torch.stack(self._diis_f))


class HostDIIS:
    """Pulay DIIS on host numpy arrays, the role pyscf's lib.diis.DIIS plays
    in the reference's CPU SCF loop: the Gram matrix of the error vectors is
    kept and extended by one row per cycle (n dot products instead of an
    n x n product over copies of every stored vector), and the extrapolated
    Fock matrix is accumulated in place."""

    def __init__(self, space=8):
        self.space = space
        self.focks, self.errs = [], []
        self.gram = np.zeros((0, 0))

    def update(self, F, err):
        """Store (F, err) and return the extrapolated Fock matrix."""
        err = np.ascontiguousarray(err).ravel()
        if len(self.focks) == self.space:
            self.focks.pop(0)
            self.errs.pop(0)
            self.gram = self.gram[1:, 1:]
        row = np.array([float(np.dot(e, err)) for e in self.errs] + [float(np.dot(err, err))])
        n = len(row)
        g = np.empty((n, n))
        g[:n - 1, :n - 1] = self.gram
        g[n - 1, :] = row
        g[:, n - 1] = row
        self.gram = g
        self.focks.append(F)
        self.errs.append(err)
        if n < 2:
            return F
        B = -np.ones((n + 1, n + 1))
        B[n, n] = 0
        B[:n, :n] = g
        rhs = np.zeros(n + 1)
        rhs[n] = -1
        try:
            c = np.linalg.solve(B, rhs)[:n]
        except np.linalg.LinAlgError:
            # singular system (repeated error vectors): no extrapolation,
            # as the device DIIS does
            return F
        Fd = self.focks[0] * c[0]
        for ci, Fi in zip(c[1:], self.focks[1:]):
            Fd += ci * Fi
        return Fd


class RHF(_SCFBase):
    """Restricted Hartree-Fock; the J/K builds go through the device engine.

    ``kernel()`` returns the total energy (pyscf convention).  Convergence is
    |Delta E| < conv_tol; incremental (difference-density) Fock builds as in
    pyscf's direct SCF (a full rebuild every ``rebuild_cycle`` cycles when it
    is positive; by default only the first build is a full one).

    Mixed precision (``fp32_threshold > 0``): on the builds before the switch
    (the first, full one and the incremental ones) the quartets whose bound
    q_ij q_kl max|D| is below fp32_threshold are evaluated in FP32 (roots,
    weights, Fock accumulation stay FP64), and with ``early_tol`` >
    direct_scf_tol those builds also drop quartets below early_tol.  Once |Delta E| < ``mixed_switch_tol`` the Fock matrix is
    rebuilt in full in FP64 at direct_scf_tol and the remaining cycles are
    FP64 incremental builds at direct_scf_tol; convergence is only accepted
    between two such final cycles, so the converged energy is an FP64 energy.
    """

    rebuild_cycle = 0
    fp32_threshold = 0.
    mixed_switch_tol = 1e-6
    early_tol = 0.
    guess_fallback = False   # set when a learned guess was abandoned for SAD
    jk_hook = None   # optional callable(density, fp32_below) run after each J/K build

    def init_guess_dm(self):
        from .guess import init_guess
        return init_guess(self, self.init_guess)

    def get_veff(self, mol=None, dm=None, dm_last=0, vhf_last=0, hermi=1):
        """Hartree-Fock potential J - K/2 (host arrays), pyscf's RHF.get_veff,
        which the reference's RHF inherits (cuobc/scf/hf.py:272-274): with a
        previous density and potential only the difference density goes
        through get_jk (direct SCF) and the result is added to vhf_last."""
        if dm is None:
            raise ValueError('get_veff needs a density')
        ddm = np.asarray(dm) - np.asarray(dm_last)
        vj, vk = self.get_jk(mol, ddm, hermi)
        return np.asarray(vhf_last) + vj - .5 * vk

    def make_rdm1(self, mo_coeff, mo_occ):
        c = mo_coeff[:, mo_occ > 0]
        return (c * mo_occ[mo_occ > 0]) @ c.T

    def get_occ(self, mo_energy):
        nocc = self.mol.nelectron // 2
        occ = torch.zeros_like(mo_energy)
        idx = torch.argsort(mo_energy)
        occ[idx[:nocc]] = 2.
        return occ

    def kernel(self, dm0=None):
        t0 = time.perf_counter()
        opt = self.opt
        S = self.get_ovlp()
        h = self.get_hcore()
        e_nuc = self.energy_nuc()
        dm = self.init_guess_dm() if dm0 is None else torch.as_tensor(dm0, device=_dev())
        torch.cuda.synchronize()
        self.timings['setup'] = time.perf_counter() - t0
        self._diis_reset()
        vj = vk = None
        dm_last = None
        e_last = None
        self.converged = False
        mixed = self.fp32_threshold > 0
        final = not mixed          # in the final (all-FP64) phase
        n_final = 0
        t_jk = 0.
        self.build_log = []
        for cycle in range(self.max_cycle):
            tj = time.perf_counter()
            full = dm_last is None or (self.rebuild_cycle > 0 and cycle % self.rebuild_cycle == 0) \
                or (mixed and final and n_final == 0)
            # before the switch every build, the first full one included, takes
            # the FP32 band and the early screen: the full FP64 rebuild at the
            # switch replaces all of it
            fp32_below = 0. if final else self.fp32_threshold
            tol = opt.direct_scf_tol
            if mixed and not final:
                tol = max(tol, self.early_tol)
            if full:
                dm_in = dm
                vj, vk = opt.jk_ao(dm[None], fp32_below=fp32_below, tol=tol)
            else:
                dm_in = dm - dm_last
                dvj, dvk = opt.jk_ao(dm_in[None], fp32_below=fp32_below, tol=tol)
                vj = vj + dvj
                vk = vk + dvk
            torch.cuda.synchronize()
            dt = time.perf_counter() - tj
            t_jk += dt
            self.build_log.append(('full' if full else 'incr', fp32_below, round(dt, 4)))
            if self.jk_hook is not None:
                self.jk_hook(dm_in, fp32_below)
            F = h + vj[0] - .5 * vk[0]
            e = float(.5 * torch.sum(dm * (h + F))) + e_nuc
            self.cycles = cycle + 1
            if final:
                n_final += 1
            de = abs(e - e_last) if e_last is not None else float('inf')
            if de < self.conv_tol and final and (not mixed or n_final >= 2):
                self.converged = True
                self.e_tot = e
                break
            if mixed and not final and de < self.mixed_switch_tol:
                final = True
            e_last = e
            err = F @ dm @ S - S @ dm @ F
            enorm = float(torch.linalg.norm(err))
            if self.init_guess == 'mlp' and cycle == 1 and not self.guess_fallback \
                    and enorm > self._enorm0:
                # the DIIS error rose from the learned guess: restart from SAD
                from .guess import init_guess
                self.guess_fallback = True
                self._diis_reset()
                dm = init_guess(self, 'sad')
                dm_last = None
                e_last = None
                continue
            if cycle == 0:
                self._enorm0 = enorm
            Fd = self._diis(F, err)
            mo_e, mo_c = self._eigh(Fd, S)
            occ = self.get_occ(mo_e)
            dm_last = dm
            dm = self.make_rdm1(mo_c, occ)
            self.mo_energy, self.mo_coeff, self.mo_occ = mo_e, mo_c, occ
        self.e_tot = e
        self.dm = dm
        torch.cuda.synchronize()
        self.timings['jk'] = t_jk
        self.timings['total'] = time.perf_counter() - t0
        return self.e_tot

    scf = kernel

    def kernel_hostloop(self, dm0=None):
        """The reference's arrangement of one SCF: a CPU loop (pyscf's role)
        holding host numpy arrays, calling the drop-in ``get_jk`` with a host
        density every cycle (host->device copy of D, device->host copies of J
        and K) and ``_eigh`` with host matrices (cuobc/scf/hf.py:230-274).
        Returns the energy; ``self.host_bytes`` = (h2d, d2h) bytes moved by
        get_jk and _eigh."""
        t0 = time.perf_counter()
        S = self.get_ovlp().cpu().numpy()
        h = self.get_hcore().cpu().numpy()
        e_nuc = self.energy_nuc()
        dm = (self.init_guess_dm() if dm0 is None else torch.as_tensor(dm0)).cpu().numpy()
        nao = dm.shape[0]
        nocc = self.mol.nelectron // 2
        h2d = d2h = 0
        diis = HostDIIS(self.diis_space)
        e_last = None
        vj = vk = dm_last = co = None
        self.converged = False
        mixed = self.fp32_threshold > 0
        final = not mixed
        n_final = 0
        for cycle in range(self.max_cycle):
            full = dm_last is None or (self.rebuild_cycle > 0 and cycle % self.rebuild_cycle == 0) \
                or (mixed and final and n_final == 0)
            fp32_below = 0. if final else self.fp32_threshold
            tol = None if final else max(self.opt.direct_scf_tol, self.early_tol)
            if full:
                vj, vk = get_jk(self.mol, dm, 1, self.opt, fp32_below=fp32_below, tol=tol)
            else:
                dvj, dvk = get_jk(self.mol, dm - dm_last, 1, self.opt, fp32_below=fp32_below,
                                  tol=tol)
                vj, vk = vj + dvj, vk + dvk
            h2d += dm.nbytes
            d2h += 2 * dm.nbytes
            F = h + vj - .5 * vk
            e = float(.5 * np.sum(dm * (h + F))) + e_nuc
            self.cycles = cycle + 1
            if final:
                n_final += 1
            de = abs(e - e_last) if e_last is not None else float('inf')
            if de < self.conv_tol and final and (not mixed or n_final >= 2):
                self.converged = True
                break
            if mixed and not final and de < self.mixed_switch_tol:
                final = True
            e_last = e
            # F D S - S D F = X - X^T with X = F D S (F, D, S symmetric), as
            # pyscf forms the DIIS error; once D = 2 Co Co^T (after the first
            # diagonalisation) X = 2 (F Co)(S Co)^T, nocc columns wide
            if co is None:
                X = F @ dm @ S
            else:
                X = 2. * (F @ co) @ (S @ co).T
            Fd = diis.update(F, X - X.T)
            mo_e, mo_c = self._eigh(Fd, S)
            mo_e = mo_e.cpu().numpy()
            mo_c = mo_c.cpu().numpy()
            # S crosses once: its orthogonalizer is kept on the device
            h2d += Fd.nbytes + (S.nbytes if cycle == 0 else 0)
            d2h += mo_e.nbytes + mo_c.nbytes
            idx = np.argsort(mo_e)[:nocc]
            dm_last = dm
            co = np.ascontiguousarray(mo_c[:, idx])
            dm = 2. * co @ co.T
        self.e_tot = e
        self.host_bytes = (h2d, d2h)
        self.timings['total'] = time.perf_counter() - t0
        return e


class UHF(_SCFBase):
    """Unrestricted Hartree-Fock: alpha and beta densities share one J/K build
    through the n_dm batch dimension (no reference counterpart)."""

    rebuild_cycle = 8

    def get_veff(self, mol=None, dm=None, dm_last=0, vhf_last=0, hermi=1):
        """Alpha and beta potentials J(total) - K(spin) (host arrays, shape
        (2, nao, nao)), pyscf's UHF.get_veff: the difference of the spin
        densities against dm_last goes through one get_jk call (n_dm = 2)
        and is added to vhf_last."""
        if dm is None:
            raise ValueError('get_veff needs a density')
        dm = np.asarray(dm)
        if dm.ndim != 3 or dm.shape[0] != 2:
            raise ValueError('UHF.get_veff needs alpha and beta densities (2, nao, nao)')
        ddm = dm - np.asarray(dm_last)
        vj, vk = self.get_jk(mol, ddm, hermi)
        return np.asarray(vhf_last) + (vj[0] + vj[1])[None] - vk

    def kernel(self, dm0=None):
        t0 = time.perf_counter()
        opt = self.opt
        S = self.get_ovlp()
        h = self.get_hcore()
        e_nuc = self.energy_nuc()
        na, nb = self.mol.nelec
        if dm0 is None:
            from .guess import init_guess
            d = init_guess(self, self.init_guess)
            dm = torch.stack([d * (na / max(na + nb, 1)), d * (nb / max(na + nb, 1))])
        else:
            dm = torch.as_tensor(dm0, device=_dev())
        self._diis_reset()
        e_last = None
        vj = vk = None
        dm_last = None
        for cycle in range(self.max_cycle):
            if dm_last is None or cycle % self.rebuild_cycle == 0:
                vj, vk = opt.jk_ao(dm)
            else:
                dvj, dvk = opt.jk_ao(dm - dm_last)
                vj, vk = vj + dvj, vk + dvk
            jtot = vj[0] + vj[1]
            F = torch.stack([h + jtot - vk[0], h + jtot - vk[1]])
            e = float(.5 * (torch.sum(dm[0] * (h + F[0])) + torch.sum(dm[1] * (h + F[1])))) + e_nuc
            self.cycles = cycle + 1
            if e_last is not None and abs(e - e_last) < self.conv_tol:
                self.converged = True
                break
            e_last = e
            err = torch.cat([F[s] @ dm[s] @ S - S @ dm[s] @ F[s] for s in range(2)])
            Fd = self._diis(F, err)
            dm_last = dm
            dms = []
            for s, n in enumerate((na, nb)):
                mo_e, mo_c = self._eigh(Fd[s], S)
                idx = torch.argsort(mo_e)[:n]
                c = mo_c[:, idx]
                dms.append(c @ c.T)
            dm = torch.stack(dms)
        self.e_tot = e
        self.dm = dm
        self.timings['total'] = time.perf_counter() - t0
        return e
