"""Learned-guess host logic (no GPU): local frames make the pair blocks
rotation invariant, and assembly inverts the local-frame transform."""
import numpy as np

from byteqc_b200.gto.mole import Mole
from byteqc_b200.gto.basis import synthetic_basis
from byteqc_b200.gto.geom import water_cluster
from byteqc_b200.learned import dataset, features
from oracle import oracle


def _rotate(atoms, Q, shift):
    return [(s, tuple(Q @ np.array(x) + shift)) for s, x in atoms]


def test_shell_rotation_orthogonal():
    rng = np.random.default_rng(1)
    Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    for l in range(4):
        U = features.shell_rotation(l, Q)
        assert np.abs(U @ U.T - np.eye(2 * l + 1)).max() < 1e-10
    assert np.abs(features.shell_rotation(1, Q) - Q).max() < 1e-10


def test_local_blocks_are_rotation_invariant():
    atoms = water_cluster(2, seed=6)
    basis = synthetic_basis('cc-pvdz', ['O', 'H'])
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(Q) < 0:
        Q[:, 0] *= -1
    m1 = Mole(atoms, basis)
    m2 = Mole(_rotate(atoms, Q, np.array([0.3, -1.0, 2.0])), basis)
    e1, d1, _ = oracle.rhf(m1, conv_tol=1e-11)
    e2, d2, _ = oracle.rhf(m2, conv_tol=1e-11)
    assert abs(e1 - e2) < 1e-8
    z1 = np.zeros_like(d1)
    f1, t1, k1 = dataset.samples(m1, d1, z1)
    f2, t2, k2 = dataset.samples(m2, d2, z1)
    assert np.abs(f1 - f2).max() < 1e-8
    assert np.abs(t1 - t2).max() < 1e-5


def test_assemble_inverts_samples():
    atoms = water_cluster(2, seed=8)
    mol = Mole(atoms, synthetic_basis('cc-pvdz', ['O', 'H']))
    rng = np.random.default_rng(0)
    d = rng.normal(size=(mol.nao, mol.nao))
    d = d + d.T
    # keep only blocks of pairs inside the cutoff (the rest is not modelled)
    sl = mol.aoslice_by_atom()
    pairs = features.canonical_pairs(mol)
    keep = np.zeros_like(d)
    for a, b in pairs:
        keep[sl[a, 2]:sl[a, 3], sl[b, 2]:sl[b, 3]] = 1
        keep[sl[b, 2]:sl[b, 3], sl[a, 2]:sl[a, 3]] = 1
    d *= keep
    sad = np.zeros_like(d)
    f, t, k = dataset.samples(mol, d, sad)
    back = dataset.assemble(mol, dataset.pair_frames(mol), t, sad)
    assert np.abs(back - d).max() < 1e-10


def test_device_assembly_matches_host():
    """assemble_device (torch, here on the CPU) adds the same blocks as the
    numpy assembly, for both basis shapes."""
    import torch
    for kind, width in (('cc-pvdz', 208), ('cc-pvtz', 912)):
        mol = Mole(water_cluster(3, seed=2), synthetic_basis(kind, ['O', 'H']))
        pf = dataset.pair_frames(mol)
        rng = np.random.default_rng(1)
        pred = rng.normal(size=(len(pf.pairs), width))
        sad = rng.normal(size=(mol.nao, mol.nao))
        ref = dataset.assemble(mol, pf, pred, sad)
        got = dataset.assemble_device(mol, pf, torch.as_tensor(pred), torch.as_tensor(sad)).numpy()
        assert np.abs(got - ref).max() < 1e-12
        assert np.abs(got - got.T).max() < 1e-12 + np.abs(sad - sad.T).max()
