"""Batched restricted HF: many independent molecules solved together.

All molecules share one set of pair lists (shells ordered molecule by
molecule; within each (l, nprim) x (l, nprim) class the 16-pair tiles are
grouped by molecule and sorted by their largest Schwarz factor), so one
``BQCbuild_jk_mol`` call builds J and K of every molecule with one launch per
class pair; quartets never mix molecules.  The AO densities and J/K live in
one block-diagonal matrix over all molecules (HBM holds it easily: 51k
Cartesian AOs for 256 (H2O)_k, k <= 12); the SCF linear algebra (DIIS,
density, energy) runs batched over a padded stack, and the new density of
each cycle is the occupied projector of the orthogonalised Fock matrix by
canonical purification, batched GEMMs per molecule size (an eigensolver only
for a molecule without a gap at the Fermi level).
"""
import ctypes
import time

import numpy as np
import torch

from .. import lib as _libmod
from ..gto import mole as gto
from .hf import (_VHFOpt, _dev, _ptr, _stream, basis_seg_contraction, PAIR_TILE,
                 free_basis_cache, make_plan)
from .guess import atomic_density


def _intra_pairs(sp, sq, shell_mol, nmol, diag):
    """Shell pairs (i in sp, j in sq) of the same molecule, i-major then j
    ascending (i >= j when diag).  sp and sq are ascending and the shells of a
    molecule are contiguous, so each molecule's members of sp (and of sq) form
    one run: the pairs are generated molecule by molecule by index arithmetic,
    in time proportional to their number rather than to len(sp) * len(sq)."""
    cp = np.bincount(shell_mol[sp], minlength=nmol)
    cq = np.bincount(shell_mol[sq], minlength=nmol)
    p0 = np.r_[0, np.cumsum(cp)[:-1]]
    q0 = np.r_[0, np.cumsum(cq)[:-1]]
    npair = cp * cq
    m = np.repeat(np.arange(nmol), npair)
    t = np.arange(int(npair.sum())) - np.r_[0, np.cumsum(npair)[:-1]][m]
    i = sp[p0[m] + t // cq[m]]
    j = sq[q0[m] + t % cq[m]]
    if diag:
        keep = i >= j
        i, j = i[keep], j[keep]
    return i, j


def _tile_order_mols(bra, ket, q, mol):
    """The 'q' tile layout of _tile_order applied to each molecule's pairs of
    one class, for all molecules at once: per molecule (ascending) the pairs
    sorted by q descending (stably), the run padded to a multiple of
    PAIR_TILE with copies of its last pair (q = 0, flagged), so no tile mixes
    molecules.  Returns (bra, ket, q, is_padding, molecule) per slot."""
    n = len(q)
    if n == 0:
        z = np.zeros(0, np.int64)
        return bra[z], ket[z], q[z], np.zeros(0, bool), np.zeros(0, np.int32)
    o = np.lexsort((-q, mol))
    bra, ket, q, mol = bra[o], ket[o], q[o], mol[o]
    uniq, cnt = np.unique(mol, return_counts=True)
    pad = (-cnt) % PAIR_TILE
    tot = cnt + pad
    ostart = np.r_[0, np.cumsum(tot)[:-1]]
    istart = np.r_[0, np.cumsum(cnt)[:-1]]
    src = np.empty(int(tot.sum()), np.int64)
    is_pad = np.zeros(len(src), bool)
    g = np.repeat(np.arange(len(uniq)), cnt)
    src[ostart[g] + np.arange(n) - istart[g]] = np.arange(n)
    pg = np.repeat(np.arange(len(uniq)), pad)
    ppos = ostart[pg] + cnt[pg] + np.arange(len(pg)) - np.r_[0, np.cumsum(pad)[:-1]][pg]
    src[ppos] = istart[pg] + cnt[pg] - 1
    is_pad[ppos] = True
    return (bra[src], ket[src], np.where(is_pad, 0., q[src]), is_pad,
            np.repeat(uniq, tot).astype(np.int32))


def _eigh_by_size(A, sizes):
    """Eigenpairs of the padded stack A (B, n, n) solved molecule size by
    molecule size on the leading sizes[b] x sizes[b] blocks (a padded stack
    makes every eigensolve as large as the largest molecule).  Padding
    directions get eigenvalue +inf-like 1e300 and unit eigenvectors, after the
    real ones, so ascending order and occupations are those of the padded
    solve."""
    B, n = A.shape[0], A.shape[-1]
    w = torch.full((B, n), 1e300, dtype=A.dtype, device=A.device)
    V = torch.eye(n, dtype=A.dtype, device=A.device).repeat(B, 1, 1)
    sizes = np.asarray(sizes)
    for s in np.unique(sizes):
        idx = torch.as_tensor(np.flatnonzero(sizes == s), device=A.device)
        ws, vs = torch.linalg.eigh(A[idx][:, :s, :s])
        w[idx, :s] = ws
        blk = V[idx]
        blk[:, :s, :s] = vs
        V[idx] = blk
    return w, V


def _occupied_projector(A, sizes, nocc, max_iter=120, tol=1e-12):
    """P[b] = projector onto the nocc[b] lowest eigenvectors of the leading
    sizes[b] x sizes[b] block of A[b] (zero outside it), by canonical
    purification (Palser and Manolopoulos, Phys. Rev. B 58, 12704 (1998)):
    batched GEMMs per molecule size instead of eigensolves.  Start from the
    Gershgorin-scaled P0 = lam/n (mu - A) + N/n with trace N; each step
    P <- ((1+c) P^2 - P^3)/c (c >= 1/2) or ((1-2c) P + (1+c) P^2 - P^3)/(1-c),
    c = tr(P^2 - P^3)/tr(P - P^2), until P^2 = P.  Molecules whose P is not
    idempotent with trace N to tol after max_iter steps (no gap at the Fermi
    level) are diagonalised instead."""
    B, n = A.shape[0], A.shape[-1]
    dev, dt = A.device, A.dtype
    P = torch.zeros_like(A)
    sizes = np.asarray(sizes)
    nocc = torch.as_tensor(np.asarray(nocc), dtype=dt, device=dev)
    for s in np.unique(sizes):
        idx = torch.as_tensor(np.flatnonzero(sizes == s), device=dev)
        F = A[idx][:, :s, :s]
        N = nocc[idx][:, None, None]
        eye = torch.eye(s, dtype=dt, device=dev)
        d = torch.diagonal(F, dim1=1, dim2=2)
        r = F.abs().sum(-1) - d.abs()
        emin = (d - r).amin(-1)[:, None, None]
        emax = (d + r).amax(-1)[:, None, None]
        mu = d.mean(-1)[:, None, None]
        lam = torch.minimum(N / (emax - mu), (s - N) / (mu - emin))
        Q = lam / s * (mu * eye - F) + N / s * eye
        for it in range(max_iter):
            Q2 = Q @ Q
            Q3 = Q2 @ Q
            trq = torch.diagonal(Q, dim1=1, dim2=2).sum(-1)
            trq2 = torch.diagonal(Q2, dim1=1, dim2=2).sum(-1)
            trq3 = torch.diagonal(Q3, dim1=1, dim2=2).sum(-1)
            den = trq - trq2
            # near convergence tr(P - P^2) -> 0: McWeeny steps (c = 1/2) there
            ok = den.abs() > 1e-10
            c = torch.where(ok, (trq2 - trq3) / torch.where(ok, den, torch.ones_like(den)),
                            torch.full_like(den, .5))[:, None, None]
            hi = ((1 + c) * Q2 - Q3) / c
            lo = ((1 - 2 * c) * Q + (1 + c) * Q2 - Q3) / (1 - c)
            Q = torch.where(c >= .5, hi, lo)
            if it % 10 == 9 and float((Q2 - Q).abs().amax()) < tol:
                break
        bad = ((Q @ Q - Q).abs().amax((1, 2)) > 100 * tol) | \
              ((torch.diagonal(Q, dim1=1, dim2=2).sum(-1) - N[:, 0, 0]).abs() > 1e-8)
        if bool(bad.any()):
            sel = torch.nonzero(bad).ravel()
            w, V = torch.linalg.eigh(F[sel])
            occ = (torch.arange(s, device=dev)[None, :] < N[sel, 0, :]).to(dt)
            Q[sel] = (V * occ[:, None, :]) @ V.transpose(1, 2)
        blk = P[idx]
        blk[:, :s, :s] = Q
        P[idx] = blk
    return P


class BatchedVHFOpt:
    """Combined decontracted basis of many molecules with intra-molecular
    pair lists."""

    def __init__(self, mols, cutoff=1e-13):
        self.mols = mols
        self.direct_scf_tol = cutoff
        parts = [basis_seg_contraction(m) for m in mols]
        self.parts = parts     # per molecule (decontracted molecule, coeff), unsorted
        self.coeffs = [c for _, c in parts]
        # concatenate the Cartesian molecules (pointer offsets into one env)
        atm, bas, env = [], [], [np.zeros(gto.PTR_ENV_START)]
        shell_mol = []
        natm = 0
        off = gto.PTR_ENV_START
        for m, (pmol, _) in enumerate(parts):
            e = pmol._env[gto.PTR_ENV_START:]
            a = pmol._atm.copy()
            a[:, gto.PTR_COORD] += off - gto.PTR_ENV_START
            a[:, 3] += off - gto.PTR_ENV_START
            b = pmol._bas.copy()
            b[:, gto.ATOM_OF] += natm
            b[:, gto.PTR_EXP] += off - gto.PTR_ENV_START
            b[:, gto.PTR_COEFF] += off - gto.PTR_ENV_START
            # (l, nprim) sort inside the molecule keeps classes uniform
            order = np.lexsort((b[:, gto.NPRIM_OF], b[:, gto.ANG_OF]))
            self.coeffs[m] = self._sort_coeff(pmol, order, self.coeffs[m])
            b = b[order]
            atm.append(a)
            bas.append(b)
            env.append(e)
            shell_mol += [m] * len(b)
            natm += len(a)
            off += len(e)
        big = mols[0].copy()
        big._atm = np.vstack(atm).astype(np.int32)
        big._bas = np.vstack(bas).astype(np.int32)
        big._env = np.concatenate(env)
        big.cart = True
        self.mol = big
        self.shell_mol = np.asarray(shell_mol, dtype=np.int32)
        ao_loc = big.ao_loc_nr(cart=True)
        self.ao_off = np.array([ao_loc[np.flatnonzero(self.shell_mol == m)[0]] for m in range(len(mols))]
                               + [ao_loc[-1]])
        self.nao_cart = int(ao_loc[-1])

    @staticmethod
    def _sort_coeff(pmol, order, coeff):
        ao_loc = pmol.ao_loc_nr(cart=True)
        idx = np.hstack([np.arange(ao_loc[i], ao_loc[i + 1]) for i in order])
        return coeff[idx]

    def build(self):
        lib = _libmod.load_library()
        mol = self.mol
        key = mol._bas[:, gto.ANG_OF] * 1000 + mol._bas[:, gto.NPRIM_OF]
        groups = np.unique(key)
        gid = np.searchsorted(groups, key)
        shells_of = [np.flatnonzero(gid == g) for g in range(len(groups))]
        pair_lists = [_intra_pairs(shells_of[p], shells_of[q], self.shell_mol, len(self.mols), p == q)
                      for p in range(len(groups)) for q in range(p + 1)]
        ncp = len(pair_lists)
        locs = np.append(0, np.cumsum([len(x[0]) for x in pair_lists])).astype(np.int32)
        p2s = np.vstack([np.hstack([x[0] for x in pair_lists]),
                         np.hstack([x[1] for x in pair_lists])]).astype(np.int32)
        helper = _VHFOpt.__new__(_VHFOpt)
        helper.mol = mol
        bp_cpu, bp_gpu, mem, keep = helper._init_cache(p2s, locs, ncp, 0.5)
        q_all = torch.zeros(max(int(locs[-1]), 1), dtype=torch.float64, device=_dev())
        for c in range(ncp):
            if locs[c + 1] > locs[c]:
                err = lib.BQCschwarz(bp_gpu, ctypes.c_int(c), ctypes.c_double(0.5),
                                     _ptr(q_all[locs[c]:]), _stream())
                if err:
                    raise RuntimeError('BQCschwarz failed (%d)' % err)
        q_all = q_all.cpu().numpy()
        helper._free_cache(bp_cpu, bp_gpu)
        del mem, keep
        b_all, k_all, q_out, mol_out, dummies, new_locs = [], [], [], [], [], [0]
        for c in range(ncp):
            sl = slice(locs[c], locs[c + 1])
            b, k, q = p2s[0, sl], p2s[1, sl], q_all[sl]
            keepm = q > self.direct_scf_tol
            b, k, q = b[keepm], k[keepm], q[keepm]
            tb, tk, tq, td, tm = _tile_order_mols(b, k, q, self.shell_mol[b])
            b_all.append(tb)
            k_all.append(tk)
            q_out.append(tq)
            dummies.append(td)
            mol_out.append(tm)
            new_locs.append(new_locs[-1] + len(tb))
        self.bas_pairs_locs = np.asarray(new_locs, dtype=np.int32)
        cat = lambda x, dt: np.hstack(x).astype(dt) if x else np.zeros(0, dt)
        self.bas_pair2shls = np.vstack([cat(b_all, np.int32), cat(k_all, np.int32)])
        self.pair_dummy = cat(dummies, bool)
        self.pair_mol_host = np.ascontiguousarray(cat(mol_out, np.int32))
        self.pair_q_host = np.ascontiguousarray(cat(q_out, np.float64))
        self.ncptype = ncp
        self._helper = helper
        self._bp_cpu, self._bp_gpu, self._mem, self._keep = helper._init_cache(
            self.bas_pair2shls, self.bas_pairs_locs, ncp, 0.5, self.pair_dummy)
        self.pair_q = torch.as_tensor(self.pair_q_host, device=_dev())
        self._plan = make_plan(self._bp_gpu, self.pair_q_host, self.pair_mol_host)
        return self

    def clear(self):
        if getattr(self, '_plan', None):
            _libmod.load_library().BQCplan_destroy(self._plan)
            self._plan = None
        if getattr(self, '_bp_cpu', None) is not None:
            free_basis_cache(self._bp_cpu, self._bp_gpu)
            self._bp_cpu = self._bp_gpu = None

    def __del__(self):
        try:
            self.clear()
        except Exception:
            pass

    def jk_cart(self, dmc, tol=None, fp32_below=0.):
        """J', K' of the block-diagonal Cartesian density dmc (1, n, n)."""
        lib = _libmod.load_library()
        n = dmc.shape[-1]
        nbas = self.mol.nbas
        dm_cond = torch.empty((nbas, nbas), dtype=torch.float64, device=dmc.device)
        err = lib.BQCdm_cond(_ptr(dmc), ctypes.c_int(1), ctypes.c_int(n), _ptr(self._mem['ao_loc']),
                             ctypes.c_int(nbas), _ptr(dm_cond), _stream())
        if err:
            raise RuntimeError('BQCdm_cond failed (%d)' % err)
        vj = torch.zeros_like(dmc)
        vk = torch.zeros_like(dmc)
        # device-scheduled over the (molecule, class pair, tile) work of the
        # batch: no host round trip, so the build can be graph-captured
        err = lib.BQCbuild_jk_plan(self._plan, _ptr(self.pair_q), _ptr(dm_cond), _ptr(vj), _ptr(vk),
                                   _ptr(dmc), n, 1, self.direct_scf_tol if tol is None else tol,
                                   fp32_below, _stream())
        if err:
            raise RuntimeError('BQCbuild_jk_plan failed (%d)' % err)
        return vj, vk


class BatchedRHF:
    """RHF of many molecules in lock step: one batched J/K build per cycle,
    padded batched DIIS, density by purification; SAD guess; incremental
    Fock builds.
    Converged molecules keep their Fock matrix (their density no longer
    changes, so the difference density screens their quartets out)."""

    # replay the J/K build of each cycle (density transform, screening table,
    # device-scheduled build, back-transform) as one captured CUDA graph
    use_graph = True

    def __init__(self, mols):
        self.mols = mols
        self.conv_tol = 1e-9
        self.max_cycle = 60
        self.diis_space = 8
        self.timings = {}

    def kernel(self):
        t0 = time.perf_counter()
        dev = _dev()
        mols = self.mols
        B = len(mols)
        opt = self.opt = BatchedVHFOpt(mols).build()
        n0 = np.array([m.nao for m in mols])
        nmax = int(n0.max())
        nc = np.diff(opt.ao_off)
        ncmax = int(nc.max())
        # padded per-molecule matrices
        S = torch.zeros((B, nmax, nmax), dtype=torch.float64, device=dev)
        H = torch.zeros_like(S)
        C = torch.zeros((B, ncmax, nmax), dtype=torch.float64, device=dev)
        D = torch.zeros_like(S)
        e_nuc = torch.tensor([m.energy_nuc() for m in mols], dtype=torch.float64, device=dev)
        for b, m in enumerate(mols):
            single = _VHFOpt.__new__(_VHFOpt)
            single.mol, single.coeff = opt.parts[b]
            single.coeff_dev = torch.as_tensor(single.coeff, device=dev)
            single.nao_cart = single.coeff.shape[0]
            single._mem = {'ao_loc': torch.as_tensor(single.mol.ao_loc_nr(cart=True),
                                                     dtype=torch.int32, device=dev)}
            s, t, v = single.int1e()
            S[b, :n0[b], :n0[b]] = s
            H[b, :n0[b], :n0[b]] = t + v
            C[b, :nc[b], :n0[b]] = torch.as_tensor(opt.coeffs[b], device=dev)
            sl = m.aoslice_by_atom()
            for ia, (sym, _) in enumerate(m.atom):
                D[b, sl[ia, 2]:sl[ia, 3], sl[ia, 2]:sl[ia, 3]] = atomic_density(sym, m.basis)
            ne = float(torch.sum(D[b] * S[b]))
            D[b] *= m.nelectron / ne
        # canonical orthogonalisation, padded rows/columns stay zero
        pad = torch.zeros((B, nmax), dtype=torch.bool, device=dev)
        for b in range(B):
            pad[b, n0[b]:] = True
        w, U = _eigh_by_size(S, n0)
        real = torch.arange(nmax, device=dev)[None, :] < torch.as_tensor(n0, device=dev)[:, None]
        X = U * torch.where(real & (w > 1e-12), 1. / torch.sqrt(w.clamp_min(1e-300)), 0.)[:, None, :]
        nocc_np = np.array([m.nelectron // 2 for m in mols])
        # gather indices of the diagonal blocks of the block-diagonal matrix
        rows, cols, bid, ri, ci = [], [], [], [], []
        for b in range(B):
            o, n = opt.ao_off[b], nc[b]
            r, c = np.meshgrid(np.arange(n), np.arange(n), indexing='ij')
            rows.append(o + r.ravel()); cols.append(o + c.ravel())
            bid.append(np.full(n * n, b)); ri.append(r.ravel()); ci.append(c.ravel())
        cat = lambda x: torch.as_tensor(np.concatenate(x), device=dev)
        rows, cols, bid, ri, ci = cat(rows), cat(cols), cat(bid), cat(ri), cat(ci)
        N = opt.nao_cart
        torch.cuda.synchronize()
        self.timings['setup'] = time.perf_counter() - t0

        def jk(dmat):
            dcp = C @ dmat @ C.transpose(1, 2)                      # (B, ncmax, ncmax)
            big = torch.zeros((1, N, N), dtype=torch.float64, device=dev)
            big[0, rows, cols] = dcp[bid, ri, ci]
            vj, vk = opt.jk_cart(big)
            J = torch.zeros_like(dcp)
            K = torch.zeros_like(dcp)
            J[bid, ri, ci] = vj[0, rows, cols]
            K[bid, ri, ci] = vk[0, rows, cols]
            J = 2 * (J + J.transpose(1, 2))
            K = K + K.transpose(1, 2)
            Ct = C.transpose(1, 2)
            return Ct @ J @ C, Ct @ K @ C

        vj, vk = jk(D)
        if self.use_graph:
            jk = _graphed(jk, D)
        e_last = None
        done = torch.zeros(B, dtype=torch.bool, device=dev)
        focks, errs = [], []
        # orthogonal directions that do not exist (padding, dropped linear
        # dependencies) get a huge orbital energy so they are never occupied
        big_diag = 1e6 * torch.diag_embed((X.abs().sum(1) == 0).double())
        t_jk = 0.
        for cycle in range(self.max_cycle):
            F = H + vj - .5 * vk
            e = .5 * torch.einsum('bij,bij->b', D, H + F) + e_nuc
            if e_last is not None:
                done = done | ((e - e_last).abs() < self.conv_tol)
                if bool(done.all()):
                    break
            e_last = e
            err = X.transpose(1, 2) @ (F @ D @ S - S @ D @ F) @ X
            focks.append(F); errs.append(err)
            focks, errs = focks[-self.diis_space:], errs[-self.diis_space:]
            k = len(focks)
            if k > 1:
                E = torch.stack(errs, 1).reshape(B, k, -1)
                Bm = torch.zeros((B, k + 1, k + 1), dtype=torch.float64, device=dev)
                G = E @ E.transpose(1, 2)
                scale = torch.diagonal(G, dim1=1, dim2=2).amax(1).clamp_min(1e-300)
                Bm[:, :k, :k] = G + (1e-14 * scale)[:, None, None] * torch.eye(k, device=dev,
                                                                              dtype=torch.float64)
                Bm[:, k, :k] = -1
                Bm[:, :k, k] = -1
                rhs = torch.zeros((B, k + 1), dtype=torch.float64, device=dev)
                rhs[:, k] = -1
                cvec = torch.linalg.solve(Bm, rhs)[:, :k]
                Fd = torch.einsum('bk,kbij->bij', cvec, torch.stack(focks))
            else:
                Fd = F
            # converged molecules keep their density: only the others are
            # diagonalised
            act_np = np.flatnonzero(~done.cpu().numpy())
            act = torch.as_tensor(act_np, device=dev)
            Xa = X[act]
            Fo = Xa.transpose(1, 2) @ Fd[act] @ Xa + big_diag[act]
            # density from the occupied projector of the orthogonalised Fock
            # matrix (purification: batched GEMMs; an eigensolve where it
            # does not converge), D = 2 X P X^T
            Po = _occupied_projector(Fo, n0[act_np], nocc_np[act_np])
            Dn = D.clone()
            Dn[act] = 2 * Xa @ Po @ Xa.transpose(1, 2)
            tj = time.perf_counter()
            dvj, dvk = jk(Dn - D)
            torch.cuda.synchronize()
            t_jk += time.perf_counter() - tj
            vj, vk = vj + dvj, vk + dvk
            D = Dn
        self.cycles = cycle + 1
        self.converged = bool(done.all())
        self.e_tot = e.cpu().numpy()
        self.timings['jk'] = t_jk
        self.timings['total'] = time.perf_counter() - t0
        return self.e_tot


def _graphed(fn, example):
    """fn(x) -> (J, K) captured once as a CUDA graph over a static input
    shaped like example; the returned function copies its argument in,
    replays the graph and returns copies of the outputs.  The library's
    launches all go to torch's current stream, which is the capture stream
    inside torch.cuda.graph."""
    static_in = example.clone()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        fn(static_in)                      # warm-up outside the capture
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        static_out = fn(static_in)

    def replay(x):
        static_in.copy_(x)
        graph.replay()
        return static_out[0].clone(), static_out[1].clone()
    replay.graph = graph
    return replay


def batch_systems(nmol, kmin=1, kmax=12, seed=0):
    """Seeded (H2O)_k, k uniform in [kmin, kmax], cc-pVDZ-shaped basis."""
    from ..gto.basis import synthetic_basis
    from ..gto.geom import water_cluster
    rng = np.random.default_rng(seed)
    basis = synthetic_basis('cc-pvdz', ['O', 'H'])
    ks = rng.integers(kmin, kmax + 1, nmol)
    return [gto.Mole(water_cluster(int(k), seed=int(seed * 100000 + i)), basis)
            for i, k in enumerate(ks)]


def main(argv=None):
    """Molecules/s of one batched solve against one-by-one plain solves.

        python -m byteqc_b200.scf.batched --nmol 256 [--seq 256]
    """
    import argparse
    import json
    from . import hf
    ap = argparse.ArgumentParser()
    ap.add_argument('--nmol', type=int, default=256)
    ap.add_argument('--seq', type=int, default=None, help='sequential solves to time (default all)')
    ap.add_argument('--conv', type=float, default=1e-9)
    a = ap.parse_args(argv)
    mols = batch_systems(a.nmol)
    BatchedRHF(mols[:2]).kernel()          # warm-up (library load, SAD atoms)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mf = BatchedRHF(mols)
    mf.conv_tol = a.conv
    e = mf.kernel()
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    nseq = a.nmol if a.seq is None else a.seq
    t0 = time.perf_counter()
    es = []
    for m in mols[:nseq]:
        one = hf.RHF(m)
        one.conv_tol = a.conv
        es.append(one.kernel())
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    out = {'nmol': a.nmol, 'nao_total': int(sum(m.nao for m in mols)),
           'batched_s': t_batch, 'batched_mol_per_s': a.nmol / t_batch,
           'batched_cycles': mf.cycles, 'batched_converged': mf.converged,
           'batched_timings': mf.timings,
           'sequential_n': nseq, 'sequential_s': t_seq, 'sequential_mol_per_s': nseq / t_seq,
           'speedup': (a.nmol / t_batch) / (nseq / t_seq),
           'max_energy_diff': float(np.max(np.abs(np.asarray(es) - e[:nseq])))}
    print(json.dumps(out))


if __name__ == '__main__':
    main()
