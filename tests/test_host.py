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
                    (3, 0, 1, 1), (3, 0, 2, 0), (3, 0, 3, 0), (3, 1, 1, 0)]
    assert autotune.canonical(0, 1, 2, 2) == (2, 2, 1, 0)
