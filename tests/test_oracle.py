"""The CPU oracle against mathematically exact golden vectors (no GPU)."""
import json
import os

import numpy as np
import pytest

from byteqc_b200.gto.mole import Mole, gto_norm, common_fac_sp, cart_powers
from byteqc_b200.gto.basis import synthetic_basis, sto3g_like
from byteqc_b200.gto.geom import water_cluster
from oracle import oracle

GOLD = os.path.join(os.path.dirname(__file__), 'golden')


def test_rys_against_mpmath():
    data = json.load(open(os.path.join(GOLD, 'rys_mpmath.json')))
    worst = 0
    for rec in data:
        r, w = oracle.rys(rec['n'], rec['x'])
        worst = max(worst, np.max(np.abs(r / rec['r'] - 1)), np.max(np.abs(w / rec['w'] - 1)))
    assert worst < 5e-14


def _prim_mol(ls, exps, cents):
    env = [0.] * 20
    atm, bas = [], []
    for ia, (c, l, e) in enumerate(zip(cents, ls, exps)):
        p = len(env)
        env += list(c) + [0.]
        atm.append([1, p, 1, p + 3, 0, 0])
        pe = len(env)
        env.append(e)
        pc = len(env)
        env.append(float(gto_norm(l, e)))
        bas.append([ia, l, 1, 1, 0, pe, pc, 0])
    m = object.__new__(Mole)
    m._atm = np.array(atm, np.int32)
    m._bas = np.array(bas, np.int32)
    m._env = np.array(env)
    m.cart = True
    return m


def test_eri_against_closed_form():
    gold = json.load(open(os.path.join(GOLD, 'eri_mpmath.json')))
    exps, cents = gold['exps'], gold['centres_bohr']
    worst = 0
    for cls in gold['classes']:
        ls = cls['ls']
        m = _prim_mol(ls, exps, cents)
        blk = oracle.eri_shells(m, 0, 1, 2, 3)
        norm = np.prod([common_fac_sp(l) * gto_norm(l, e) for l, e in zip(ls, exps)])
        for c in cls['comps']:
            ref = c['value'] * norm
            v = blk[tuple(c['f'])]
            worst = max(worst, abs(v - ref) / max(abs(ref), 1e-3))
    assert worst < 1e-13


def test_jk_digestion_against_full_tensor():
    mol = Mole(water_cluster(1, seed=3), sto3g_like(['O', 'H']))
    eri = oracle.eri_full_cart(mol)
    assert np.abs(eri - eri.transpose(1, 0, 2, 3)).max() < 1e-13
    assert np.abs(eri - eri.transpose(2, 3, 0, 1)).max() < 1e-13
    rng = np.random.default_rng(2341)
    n = eri.shape[0]
    dm = rng.random((n, n))
    dm = dm + dm.T
    vj, vk = oracle.jk_cart(mol, dm)
    assert np.abs(vj - np.einsum('ijkl,kl->ij', eri, dm)).max() < 1e-12
    assert np.abs(vk - np.einsum('ijkl,jl->ik', eri, dm)).max() < 1e-12


def test_int1e_normalisation_and_hydrogenic():
    import scipy.linalg
    mol = Mole([('O', (0, 0, 0))], synthetic_basis('cc-pvtz', ['O']))
    S, T, V = oracle.int1e(mol)
    assert np.abs(np.diag(S) - 1).max() < 1e-13
    # one electron in the field of Z = 8: E -> -Z^2/2 as the basis allows
    e = scipy.linalg.eigh(T + V, S, eigvals_only=True)
    assert -32.0 < e[0] < -31.5


def test_rhf_water_is_variational():
    mol = Mole(water_cluster(1, seed=3), synthetic_basis('cc-pvdz', ['O', 'H']))
    e, dm, it = oracle.rhf(mol, conv_tol=1e-10)
    S, _, _ = oracle.int1e(mol)
    assert abs(np.sum(dm * S) - 10) < 1e-8
    assert -76.5 < e < -74.5


def test_oracle_three_centre_closed_form():
    """The constant s shell of the density-fitting path (exponent 0, the
    s-function factor cancelled) turns the oracle's four-centre quartet
    (a b | c 1) into the three-centre Coulomb integral, whose closed form for
    normalised s Gaussians is
    Na Nb Nc exp(-ab/p |AB|^2) 2 pi^(5/2) / (p c sqrt(p + c)) F0(pc/(p+c) |PC|^2)."""
    import math
    from byteqc_b200.gto.mole import Mole
    from byteqc_b200.df.int3c import make_fake_mol, conc_mol
    from oracle import oracle
    atoms = [('H', (0., 0., 0.)), ('H', (0.3, -0.4, 1.1)), ('H', (-0.7, 0.2, 0.5))]
    exps = [1.3, 0.45, 2.2]
    mol = Mole(atoms, {'H': [[0, [1., 1.]]]}, unit='Bohr')
    env = list(mol._env)
    for ish, a in enumerate(exps):     # one primitive s shell per atom, own exponent
        mol._bas[ish, 5] = len(env)
        mol._bas[ish, 6] = len(env) + 1
        env += [a, (2 * a / math.pi) ** .75 / 0.282094791773878143]
    mol._env = np.asarray(env)
    tot = conc_mol(mol, make_fake_mol())
    R = mol.atom_coords()
    a, b, c = exps
    p = a + b
    P = (a * R[0] + b * R[1]) / p
    T = p * c / (p + c) * float(np.sum((P - R[2]) ** 2))
    F0 = math.sqrt(math.pi / (4 * T)) * math.erf(math.sqrt(T))
    Ns = [(2 * e / math.pi) ** .75 for e in exps]
    ref = Ns[0] * Ns[1] * Ns[2] * math.exp(-a * b / p * float(np.sum((R[0] - R[1]) ** 2))) * \
        2 * math.pi ** 2.5 / (p * c * math.sqrt(p + c)) * F0
    got = oracle.eri_shells(tot, 0, 1, 2, 3).ravel()[0]
    assert abs(got - ref) < 1e-14 * abs(ref), (got, ref)
