"""What the learned initial density gains over the method without it (needs a
B200 and the trained weights in byteqc_b200/learned/).

On held-out systems (the training set is seeded (H2O)_k with k in [2, 16]
and CnH(2n+2) with n in [4, 20]): the plain FP64 RHF from the learned guess
and from SAD converge to the same energy (within 1e-9 Eh: the converged FP64
SCF fixes the energy, only the iteration count may change), and the learned
guess needs fewer SCF cycles in total.  Cycles and wall times are printed.
"""
import time

import pytest

from byteqc_b200.gto.geom import water_cluster, linear_alkane

pytestmark = pytest.mark.gpu


def _solve(mol, guess, weights):
    import torch
    from byteqc_b200.scf import hf, guess as G
    G._SAD_CACHE.clear()
    mf = hf.RHF(mol)
    mf.conv_tol = 1e-9
    mf.init_guess = guess
    if weights:
        mf.mlp_weights = weights
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e = mf.kernel()
    torch.cuda.synchronize()
    return e, mf.cycles, time.perf_counter() - t0, mf


@pytest.mark.parametrize('basis', ['cc-pvdz', 'cc-pvtz'])
def test_learned_guess_gains_over_sad(cuda, basis):
    from byteqc_b200.learned import infer, train
    systems = [('(H2O)32', water_cluster(32, seed=7)), ('C40H82', linear_alkane(40))]
    if basis == 'cc-pvtz':
        systems = [('(H2O)24', water_cluster(24, seed=7)), ('C24H50', linear_alkane(24))]
    probe = train.make_mol(systems[0][1], basis)
    weights = infer.weights_for(probe)
    if weights is None:
        pytest.skip('no trained model for the %s shape' % basis)
    gained = 0
    for name, atoms in systems:
        mol = train.make_mol(atoms, basis)
        _solve(mol, 'sad', None)                       # warm-up: library, atomic densities
        e_sad, c_sad, t_sad, _ = _solve(mol, 'sad', None)
        e_mlp, c_mlp, t_mlp, mf = _solve(mol, 'mlp', weights)
        print('%s %s: SAD %d cycles %.3f s, learned %d cycles %.3f s%s, |dE| %.1e' % (
            name, basis, c_sad, t_sad, c_mlp, t_mlp,
            ' (fell back to SAD)' if mf.guess_fallback else '', abs(e_mlp - e_sad)))
        assert abs(e_mlp - e_sad) < 1e-9
        gained += c_sad - c_mlp
    assert gained > 0
