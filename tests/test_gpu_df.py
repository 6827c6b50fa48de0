"""Density-fitting integrals (byteqc_b200.df.int3c, the path of
cuobc/lib/int3c.py:177-373) against the CPU oracle (needs a B200).

The 3-centre integrals (ij|k) come from GINTfill_int2e with the auxiliary
shells paired with a constant s function; the oracle evaluates the same
(i j | k 1) quartets on the concatenated molecule.  Bar: 1e-10 absolute.
"""
import numpy as np
import pytest

from byteqc_b200.gto.mole import Mole
from byteqc_b200.gto.basis import synthetic_basis, synthetic_aux_basis
from byteqc_b200.gto.geom import water_cluster
from oracle import oracle

pytestmark = pytest.mark.gpu


def _opt(nw=1, kind='cc-pvdz', seed=3):
    from byteqc_b200.df import int3c
    atoms = water_cluster(nw, seed=seed)
    mol = Mole(atoms, synthetic_basis(kind, ['O', 'H']))
    aux = Mole(atoms, synthetic_aux_basis(['O', 'H']))
    return mol, aux, int3c.VHFOpt3c(mol, aux).build()


@pytest.mark.parametrize('kind', ['cc-pvdz', 'cc-pvtz'])
def test_int3c_against_oracle(cuda, kind):
    from byteqc_b200.df import int3c
    mol, aux, opt = _opt(kind=kind)
    full = int3c.int3c_cart(opt).cpu().numpy()
    tot = opt.tot_mol
    nbas = len(opt.ao_loc) - 1
    fake = nbas                       # the constant shell follows the orbital shells
    ao = tot.ao_loc_nr(cart=True)
    ref = np.zeros_like(full)
    for i in range(nbas):
        for j in range(nbas):
            for k in range(fake + 1, tot.nbas):
                blk = oracle.eri_shells(tot, i, j, k, fake)[..., 0]
                ref[ao[i]:ao[i + 1], ao[j]:ao[j + 1], ao[k] - opt.nao - 1:ao[k + 1] - opt.nao - 1] = blk
    err = abs(full - ref).max()
    print('int3c %s: max|(ij|k)| %.3g max err %.3e' % (kind, abs(ref).max(), err))
    assert err < 1e-10
    # the caller's bases
    ao3 = int3c.int3c_ao(opt).cpu().numpy()
    C, Ca = opt.coeff, opt.auxcoeff
    assert abs(ao3 - np.einsum('pqr,pi,qj,rk->ijk', ref, C, C, Ca)).max() < 1e-10


def test_int2c_metric_factor(cuda):
    from byteqc_b200.df import int3c
    mol, aux, opt = _opt()
    tot = opt.tot_mol
    nbas = len(opt.ao_loc) - 1
    fake = nbas
    ao = tot.ao_loc_nr(cart=True)
    n = opt.naux
    M = np.zeros((n, n))
    for k in range(fake + 1, tot.nbas):
        for l in range(fake + 1, tot.nbas):
            blk = oracle.eri_shells(tot, k, fake, l, fake)[:, 0, :, 0]
            M[ao[k] - opt.nao - 1:ao[k + 1] - opt.nao - 1, ao[l] - opt.nao - 1:ao[l + 1] - opt.nao - 1] = blk
    Ca = opt.auxcoeff
    M = Ca.T @ M @ Ca
    L = int3c.get_int2c(opt).cpu().numpy()
    assert np.allclose(L, np.tril(L))
    err = abs(L @ L.T - M).max()
    print('int2c: max|(k|l)| %.3g max err %.3e' % (abs(M).max(), err))
    assert err < 1e-10 * max(1., abs(M).max())
    # the eigenvector form spans the same metric: V^T M V = 1
    V = int3c.get_int2c(opt, j2c_eig_always=True).cpu().numpy()
    assert abs(V.T @ M @ V - np.eye(V.shape[1])).max() < 1e-8


def test_int3c_screened_pairs(cuda):
    """Two waters: pairs below the 1e-11 Schwarz cutoff are left out, so the
    tensor agrees with the oracle to the size of what was dropped."""
    from byteqc_b200.df import int3c
    mol, aux, opt = _opt(nw=2, seed=6)
    full = int3c.int3c_cart(opt).cpu().numpy()
    tot = opt.tot_mol
    nbas = len(opt.ao_loc) - 1
    fake = nbas
    ao = tot.ao_loc_nr(cart=True)
    rng = np.random.default_rng(0)
    worst = 0.
    for _ in range(300):
        i, j = rng.integers(0, nbas, 2)
        k = rng.integers(fake + 1, tot.nbas)
        blk = oracle.eri_shells(tot, i, j, k, fake)[..., 0]
        got = full[ao[i]:ao[i + 1], ao[j]:ao[j + 1], ao[k] - opt.nao - 1:ao[k + 1] - opt.nao - 1]
        worst = max(worst, abs(got - blk).max())
    print('int3c two waters: max err %.3e over 300 shell triples' % worst)
    assert worst < 1e-10
