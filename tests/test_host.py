"""Host-side logic (no GPU): molecule layout, basis shapes, geometry, the
decontraction transform, the committed Rys table and the C-ABI exports."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

from byteqc_b200.gto.mole import Mole, cart2sph, cart_powers
from byteqc_b200.gto.basis import synthetic_basis
from byteqc_b200.gto.geom import water_cluster, linear_alkane
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize('name,atoms,nao', [
    ('cc-pvdz', water_cluster(4, 0), 96),
    ('cc-pvtz', water_cluster(64, 0), 3712),
    ('6-31g**', linear_alkane(60), 1450),
])
def test_ao_counts(name, atoms, nao):
    els = sorted(set(a[0] for a in atoms))
    mol = Mole(atoms, synthetic_basis(name, els))
    assert mol.nao == nao


def test_water_geometry():
    at = water_cluster(8, seed=4)
    xyz = np.array([a[1] for a in at]).reshape(8, 3, 3)
    roh = np.linalg.norm(xyz[:, 1:] - xyz[:, :1], axis=2)
    assert np.allclose(roh, 0.9572)
    v1, v2 = xyz[:, 1] - xyz[:, 0], xyz[:, 2] - xyz[:, 0]
    ang = np.degrees(np.arccos(np.sum(v1 * v2, 1) / 0.9572 ** 2))
    assert np.allclose(ang, 104.52)
    assert water_cluster(8, seed=4) == at and water_cluster(8, seed=5) != at


def test_alkane_geometry():
    at = linear_alkane(5)
    assert sum(a[0] == 'C' for a in at) == 5 and sum(a[0] == 'H' for a in at) == 12
    xyz = np.array([a[1] for a in at])
    d = np.linalg.norm(xyz[:, None] - xyz[None], axis=2) + 9 * np.eye(len(at))
    assert abs(d.min() - 1.09) < 1e-9


@pytest.mark.parametrize('l', [2, 3])
def test_cart2sph_orthonormal(l):
    # exact angular integrals of monomials over the unit sphere
    from math import gamma
    def mono(a, b, c):
        if a % 2 or b % 2 or c % 2:
            return 0.
        return 2 * gamma((a + 1) / 2) * gamma((b + 1) / 2) * gamma((c + 1) / 2) / gamma((a + b + c + 3) / 2)
    P = cart_powers(l)
    G = np.array([[mono(p[0] + q[0], p[1] + q[1], p[2] + q[2]) for q in P] for p in P])
    C = cart2sph(l)
    assert np.abs(C.T @ G @ C - np.eye(2 * l + 1)).max() < 1e-12


def test_decontraction_transform():
    """J/K in the decontracted Cartesian basis, transformed with coeff, equal
    J/K in the original contracted spherical basis (both from the oracle)."""
    from byteqc_b200.scf.hf import basis_seg_contraction
    mol = Mole(water_cluster(1, seed=2), synthetic_basis('cc-pvdz', ['O', 'H']))
    pmol, coeff = basis_seg_contraction(mol)
    assert coeff.shape == (pmol.nao_nr(cart=True), mol.nao)
    assert (pmol._bas[:, 3] == 1).all()
    rng = np.random.default_rng(1)
    dm = rng.random((mol.nao, mol.nao))
    dm = dm + dm.T
    rj, rk = oracle.get_jk(mol, dm)
    vj, vk = oracle.jk_cart(pmol, coeff @ dm @ coeff.T)
    assert np.abs(coeff.T @ vj @ coeff - rj).max() < 1e-10
    assert np.abs(coeff.T @ vk @ coeff - rk).max() < 1e-10


def test_s_index_offsets():
    from byteqc_b200.scf.hf import _make_s_index_offsets
    lq = np.log(np.array([1., .5, 1e-3, 1e-7, 1e-11]))
    b = _make_s_index_offsets(lq, 10, 1e-12)
    assert b[0] == 0 and b[-1] == 5 and np.all(np.diff(b) >= 0) and len(b) == 11


def _table():
    src = open(os.path.join(ROOT, 'byteqc_b200', 'csrc', 'rys_tables.inc')).read()
    def arr(name, typ=float):
        m = re.search(r'%s\[\d+\] = \{(.*?)\};' % name, src, re.S)
        return np.array([typ(v) for v in m.group(1).replace('\n', ' ').split(',') if v.strip()])
    return (arr('RYS_XMAX', int), arr('RYS_TABLE_OFFSET', int), arr('RYS_TABLE'),
            arr('RYS_HERM_OFFSET', int), arr('RYS_HERM_R2'), arr('RYS_HERM_W'), arr('RYS_TABLE_LM'))


def test_committed_rys_table_against_mpmath():
    """Clenshaw evaluation of the committed table, restated in numpy, matches
    the 60-digit golden values."""
    xmax, off, tab, hoff, hr2, hw, tab_lm = _table()
    data = json.load(open(os.path.join(ROOT, 'tests', 'golden', 'rys_mpmath.json')))
    worst = 0
    for rec in data:
        n, x = rec['n'], rec['x']
        if x < xmax[n]:
            k = int(x)
            t = 2 * (x - k) - 1
            c = tab[off[n] + k * 12 * 2 * n: off[n] + (k + 1) * 12 * 2 * n].reshape(12, 2 * n)
            # the level-major copy holds the same coefficients
            lm = tab_lm[off[n]:off[n + 1]].reshape(12, n, xmax[n], 2)[:, :, k, :].reshape(12, 2 * n)
            assert np.array_equal(c, lm)
            b1 = c[11].copy()
            b2 = np.zeros(2 * n)
            for kk in range(10, 0, -1):
                b1, b2 = 2 * t * b1 - b2 + c[kk], b1
            v = t * b1 - b2 + c[0]
            r, w = v[:n], v[n:]
        else:
            r = hr2[hoff[n]:hoff[n] + n] / x
            w = hw[hoff[n]:hoff[n] + n] / np.sqrt(x)
        worst = max(worst, np.max(np.abs(r / rec['r'] - 1)), np.max(np.abs(w / rec['w'] - 1)))
    assert worst < 2e-15


def test_library_exports_header_symbols():
    lib_path = os.path.join(ROOT, 'byteqc_b200', 'libbyteqc_b200.so')
    if not os.path.exists(lib_path):
        pytest.skip('library not built')
    hdr = open(os.path.join(ROOT, 'include', 'byteqc_b200.h')).read()
    names = set(re.findall(r'\b((?:GINT|BQC)\w+)\s*\(', hdr))
    assert {'GINTbuild_jk', 'BQCbuild_jk'} <= names
    lib = ctypes.CDLL(lib_path)
    for n in names:
        assert hasattr(lib, n), n
    from byteqc_b200 import lib as L
    assert set(L.SYMBOLS) <= names


@pytest.mark.parametrize('layout', ['q', 'shell', 'hybrid'])
def test_tile_order_invariants(layout):
    """Every pair once, padding with q = 0, q descending inside a tile and
    along the tiles' first entries (what the host tile pruning relies on)."""
    from byteqc_b200.scf.hf import _tile_order, PAIR_TILE
    rng = np.random.default_rng(7)
    for n in [0, 1, 5, 16, 17, 100, 1000]:
        b = rng.integers(0, 20, n)
        k = rng.integers(0, 50, n)
        q = rng.random(n) ** 8
        B, K, Q, D = _tile_order(b, k, q, layout)
        assert len(B) % PAIR_TILE == 0
        assert sorted(zip(B[~D], K[~D], Q[~D])) == sorted(zip(b, k, q))
        assert np.all(Q[D] == 0)
        T = Q.reshape(-1, PAIR_TILE)
        assert np.all(np.diff(T, axis=1) <= 0)
        assert np.all(np.diff(T[:, 0]) <= 0)
        if layout == 'shell' and n:
            Bt, Dt = B.reshape(-1, PAIR_TILE), D.reshape(-1, PAIR_TILE)
            assert np.all((Bt == Bt[:, :1]) | Dt)


def test_autotune_variant_rule():
    """The Python copy of the kernel-choice rule matches the classes that
    have a ket-split variant (jk_kernels.cuh launch_class)."""
    from byteqc_b200 import autotune
    both = sorted({autotune.canonical(*c) for c in
                   [(a, b, c, d) for a in range(4) for b in range(4) for c in range(4) for d in range(4)]
                   if autotune.has_variants(*c)})
    assert both == [(1, 1, 1, 1), (2, 1, 1, 1), (2, 1, 2, 0), (2, 2, 1, 0),
                    (3, 0, 1, 1), (3, 0, 2, 0), (3, 0, 3, 0), (3, 1, 1, 0), (3, 2, 0, 0),
                    (3, 3, 0, 0)]
    assert autotune.canonical(0, 1, 2, 2) == (2, 2, 1, 0)


def test_basis_prod_ownership_reference_sequence():
    """The reference's call sequence (cuobc/scf/hf.py:410-442): init_cpu,
    init_gpu on device copies, then GINTdel_basis_prod on the device copy
    only.  The device copy shares and frees the host blocks of the cpu
    cache, so repeating the sequence does not grow the heap (the few bytes
    of the cpu struct itself are left, as in the reference)."""
    from byteqc_b200 import lib as L
    from byteqc_b200.scf.hf import basis_seg_contraction
    lib = L.load_library()
    libc = ctypes.CDLL('libc.so.6')

    class MallInfo2(ctypes.Structure):
        _fields_ = [(n, ctypes.c_size_t) for n in
                    ('arena', 'ordblks', 'smblks', 'hblks', 'hblkhd', 'usmblks', 'fsmblks',
                     'uordblks', 'fordblks', 'keepcost')]
    libc.mallinfo2.restype = MallInfo2
    mol = Mole(water_cluster(4, seed=1), synthetic_basis('cc-pvtz', ['O', 'H']))
    pmol, _ = basis_seg_contraction(mol)
    n = pmol.nbas
    # one class: all pairs of the shells of one (l, nprim) kind (the class
    # table takes l and nprim from its first pair)
    kind = pmol._bas[:, 1] * 100 + pmol._bas[:, 2]
    sel = np.flatnonzero(kind == np.bincount(kind).argmax())
    ii, jj = np.tril_indices(len(sel))
    i, j = sel[ii], sel[jj]
    p2s = np.ascontiguousarray(np.vstack([i, j]), dtype=np.int32)
    locs = np.array([0, len(i)], dtype=np.int32)
    atm = np.ascontiguousarray(pmol._atm, dtype=np.int32)
    bas = np.ascontiguousarray(pmol._bas, dtype=np.int32)
    env = np.ascontiguousarray(pmol._env)
    coords = np.empty(3 * n)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)

    def sequence():
        bp = ctypes.POINTER(L.BasisProdCache)()
        lib.GINTinit_basis_prod_cpu(ctypes.byref(bp), ctypes.c_double(.5), vp(coords), vp(p2s),
                                    vp(locs), ctypes.c_int(1), vp(atm), ctypes.c_int(pmol.natm),
                                    vp(bas), ctypes.c_int(n), vp(env))
        assert bp.contents.aexyz    # the host block the cpu cache fills
        bpg = ctypes.POINTER(L.BasisProdCache)()
        # device pointers are only stored, never dereferenced on the host
        lib.GINTinit_basis_prod_gpu(ctypes.byref(bp), ctypes.byref(bpg), None, None, None, None)
        assert ctypes.cast(bpg.contents.aexyz, ctypes.c_void_p).value == \
            ctypes.cast(bp.contents.aexyz, ctypes.c_void_p).value
        lib.GINTdel_basis_prod(ctypes.byref(bpg))
        assert not bpg

    for _ in range(5):
        sequence()
    used0 = libc.mallinfo2().uordblks + libc.mallinfo2().hblkhd
    for _ in range(50):
        sequence()
    used1 = libc.mallinfo2().uordblks + libc.mallinfo2().hblkhd
    block = 5 * 8 * len(i)       # the aexyz block of one cache
    assert used1 - used0 < block, (used1 - used0, block)


def test_reference_decontraction_matches_engine():
    """The reference-side restatement (oracle/ref_gpu.py seg_contraction of
    cuobc/scf/hf.py:481-564) and the engine's basis_seg_contraction give the
    same primitive basis and contraction matrix."""
    from byteqc_b200.scf.hf import basis_seg_contraction
    from oracle.ref_gpu import seg_contraction
    for kind in ('cc-pvdz', 'cc-pvtz'):
        mol = Mole(water_cluster(2, seed=4), synthetic_basis(kind, ['O', 'H']))
        p1, c1 = basis_seg_contraction(mol)
        p2, c2 = seg_contraction(mol)
        assert (p1._bas == p2._bas).all()
        assert np.allclose(p1._env, p2._env, rtol=1e-15, atol=0)
        assert np.allclose(c1, c2, rtol=1e-14, atol=1e-15)


def test_reference_pair_lists():
    """RefVHFOpt (cuobc/scf/hf.py:288-397 restated): per class the pairs
    above the cutoff in descending q, ish >= jsh on diagonal blocks, every
    pair listed exactly once, log q clipped at 0."""
    from oracle.ref_gpu import RefVHFOpt
    mol = Mole(water_cluster(3, seed=6), synthetic_basis('cc-pvdz', ['O', 'H']))
    opt = RefVHFOpt(mol).build(1e-13)
    q = oracle.q_cond(opt.mol)
    offs = opt.l_ctr_offsets
    seen = set()
    c = 0
    for p in range(len(opt.uniq_l_ctr)):
        for r in range(p + 1):
            sl = slice(opt.bas_pairs_locs[c], opt.bas_pairs_locs[c + 1])
            bra, ket = opt.bas_pair2shls[0, sl], opt.bas_pair2shls[1, sl]
            assert ((bra >= offs[p]) & (bra < offs[p + 1])).all()
            assert ((ket >= offs[r]) & (ket < offs[r + 1])).all()
            qs = q[bra, ket]
            assert (np.diff(qs) <= 0).all() and (qs > 1e-13).all()
            if p == r:
                assert (bra >= ket).all()
            assert np.allclose(opt.log_qs[c], np.minimum(np.log(qs), 0))
            seen.update(zip(bra.tolist(), ket.tolist()))
            c += 1
    n = opt.mol.nbas
    expect = {(i, j) if opt_i_ge(i, j, offs) else (j, i) for i in range(n) for j in range(n)
              if q[i, j] > 1e-13}
    assert seen == expect


def opt_i_ge(i, j, offs):
    """Orientation of a pair in the reference lists: the bra shell comes from
    the later (l, nprim) group, or is the larger index within one group."""
    gi = np.searchsorted(offs, i, side='right')
    gj = np.searchsorted(offs, j, side='right')
    return gi > gj or (gi == gj and i >= j)


def test_host_diis_matches_full_solve():
    """HostDIIS (incremental Gram matrix, in-place extrapolation) gives the
    Fock matrix of a full Pulay solve over the last `space` stored pairs."""
    from byteqc_b200.scf.hf import HostDIIS
    rng = np.random.default_rng(5)
    n, space = 12, 4
    diis = HostDIIS(space)
    focks, errs = [], []
    for it in range(9):
        F = rng.normal(size=(n, n))
        F = F + F.T
        X = F @ rng.normal(size=(n, n))
        err = X - X.T
        got = diis.update(F, err)
        focks.append(F)
        errs.append(err.ravel())
        fs, es = focks[-space:], np.array(errs[-space:])
        m = len(fs)
        if m < 2:
            assert got is F
            continue
        B = -np.ones((m + 1, m + 1))
        B[m, m] = 0
        B[:m, :m] = es @ es.T
        rhs = np.zeros(m + 1)
        rhs[m] = -1
        c = np.linalg.solve(B, rhs)[:m]
        ref = np.einsum('i,ijk->jk', c, np.array(fs))
        assert np.abs(got - ref).max() < 1e-10 * max(1., np.abs(ref).max())
        assert np.abs(diis.gram - es @ es.T).max() < 1e-10 * np.abs(es @ es.T).max()


def test_batched_intra_pairs_match_masked_product():
    """The per-molecule pair generation of the batched basis gives the same
    pairs, in the same order, as the full cross product masked to pairs of
    one molecule."""
    from byteqc_b200.scf import batched
    from byteqc_b200.gto import mole as gto
    mols = batched.batch_systems(24, seed=3)
    o = batched.BatchedVHFOpt(mols)
    key = o.mol._bas[:, gto.ANG_OF] * 1000 + o.mol._bas[:, gto.NPRIM_OF]
    gid = np.searchsorted(np.unique(key), key)
    shells_of = [np.flatnonzero(gid == g) for g in range(gid.max() + 1)]
    for p in range(len(shells_of)):
        for q in range(p + 1):
            i = np.repeat(shells_of[p], len(shells_of[q]))
            j = np.tile(shells_of[q], len(shells_of[p]))
            m = o.shell_mol[i] == o.shell_mol[j]
            if p == q:
                m &= i >= j
            gi, gj = batched._intra_pairs(shells_of[p], shells_of[q], o.shell_mol, len(mols), p == q)
            assert np.array_equal(gi, i[m]) and np.array_equal(gj, j[m])


def test_batched_eigh_by_size_matches_padded_solve():
    """Densities from the size-by-size eigensolve of a padded stack equal
    those of the padded solve with a large diagonal on the padding."""
    import torch
    from byteqc_b200.scf.batched import _eigh_by_size
    rng = np.random.default_rng(2)
    sizes = np.array([5, 9, 5, 12, 9])
    B, n = len(sizes), 12
    A = torch.zeros((B, n, n), dtype=torch.float64)
    for b, s in enumerate(sizes):
        m = rng.normal(size=(s, s))
        A[b, :s, :s] = torch.as_tensor(m + m.T)
    pad = torch.arange(n)[None, :] >= torch.as_tensor(sizes)[:, None]
    w0, v0 = torch.linalg.eigh(A + 1e6 * torch.diag_embed(pad.double()))
    w1, v1 = _eigh_by_size(A, sizes)
    for b, s in enumerate(sizes):
        assert torch.allclose(w1[b, :s], w0[b, :s], atol=1e-10)
        nocc = s // 2
        d0 = v0[b, :, :nocc] @ v0[b, :, :nocc].T
        d1 = v1[b, :, :nocc] @ v1[b, :, :nocc].T
        assert torch.allclose(d0, d1, atol=1e-10)


def test_batched_occupied_projector():
    """Canonical purification gives the projector onto the nocc lowest
    eigenvectors (against eigh) for gapped spectra of several sizes, one with
    a far-out eigenvalue like the one given to dropped directions; a spectrum
    without a gap at the Fermi level falls back to the eigensolver and still
    returns an idempotent projector of trace nocc."""
    import torch
    from byteqc_b200.scf.batched import _occupied_projector
    rng = np.random.default_rng(7)
    sizes = np.array([10, 30, 30, 18])
    n = 30
    A = torch.zeros((len(sizes), n, n), dtype=torch.float64)
    nocc = []
    for b, s in enumerate(sizes):
        no = s // 3
        ev = np.r_[-np.sort(rng.uniform(0.3, 20., no))[::-1], rng.uniform(0.1, 8., s - no)]
        if b == 2:
            ev[-1] = 1e6
        if b == 3:
            ev[no] = ev[no - 1]      # degenerate HOMO/LUMO
        Q, _ = np.linalg.qr(rng.normal(size=(s, s)))
        A[b, :s, :s] = torch.as_tensor(Q @ np.diag(ev) @ Q.T)
        nocc.append(no)
    P = _occupied_projector(A, sizes, nocc)
    for b, s in enumerate(sizes):
        Pb = P[b, :s, :s]
        assert float((Pb @ Pb - Pb).abs().max()) < 1e-10
        assert abs(float(Pb.trace()) - nocc[b]) < 1e-8
        outside = P[b].clone()
        outside[:s, :s] = 0
        assert float(outside.abs().max()) == 0.
        if b < 3:
            w, V = torch.linalg.eigh(A[b, :s, :s])
            Pe = V[:, :nocc[b]] @ V[:, :nocc[b]].T
            assert float((Pb - Pe).abs().max()) < 1e-10


def test_batched_tile_order_matches_per_molecule_loop():
    """The all-molecule tile ordering of the batched lists equals the 'q'
    layout of _tile_order applied molecule by molecule (ties in q included)."""
    from byteqc_b200.scf import batched
    from byteqc_b200.scf.hf import _tile_order
    rng = np.random.default_rng(11)
    nmol, n = 9, 700
    mol = np.sort(rng.integers(0, nmol, n)).astype(np.int32)
    mol[rng.permutation(n)[:50]] = mol[rng.permutation(n)[:50]]   # not sorted by molecule
    bra = rng.integers(0, 10 ** 5, n).astype(np.int32)
    ket = rng.integers(0, 10 ** 5, n).astype(np.int32)
    q = np.round(rng.random(n) * 20) / 20 + 1e-3                    # many ties
    parts = [[], [], [], [], []]
    for m in np.unique(mol):
        s = mol == m
        tb, tk, tq, td = _tile_order(bra[s], ket[s], q[s])
        for lst, v in zip(parts, (tb, tk, tq, td, np.full(len(tb), m, np.int32))):
            lst.append(v)
    ref = [np.hstack(x) for x in parts]
    got = batched._tile_order_mols(bra, ket, q, mol)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
