"""Batched RHF of molecules of uneven size against one-by-one RHF (B200)."""
import numpy as np
import pytest

from byteqc_b200.gto.mole import Mole
from byteqc_b200.gto.basis import synthetic_basis
from byteqc_b200.gto.geom import water_cluster

pytestmark = pytest.mark.gpu


def test_batched_rhf_matches_single(cuda):
    from byteqc_b200.scf import hf
    from byteqc_b200.scf.batched import BatchedRHF
    basis = synthetic_basis('cc-pvdz', ['O', 'H'])
    mols = [Mole(water_cluster(k, seed=20 + k), basis) for k in (1, 3, 2, 1)]
    mf = BatchedRHF(mols)
    mf.conv_tol = 1e-10
    e = mf.kernel()
    assert mf.converged
    for m, eb in zip(mols, e):
        one = hf.RHF(m)
        one.conv_tol = 1e-10
        e1 = one.kernel()
        assert abs(eb - e1) < 1e-8, (eb, e1)


def test_batched_jk_has_no_cross_molecule_terms(cuda):
    """J/K of the block-diagonal density equal the per-molecule J/K."""
    import torch
    from byteqc_b200.scf import hf
    from byteqc_b200.scf.batched import BatchedVHFOpt
    basis = synthetic_basis('cc-pvdz', ['O', 'H'])
    mols = [Mole(water_cluster(k, seed=30 + k), basis) for k in (2, 1)]
    opt = BatchedVHFOpt(mols).build()
    rng = np.random.default_rng(5)
    N = opt.nao_cart
    big = torch.zeros((1, N, N), dtype=torch.float64, device=cuda)
    refs = []
    for b, m in enumerate(mols):
        d = rng.random((m.nao, m.nao))
        d = d + d.T
        C = torch.as_tensor(opt.coeffs[b], device=cuda)
        o0, o1 = opt.ao_off[b], opt.ao_off[b + 1]
        big[0, o0:o1, o0:o1] = C @ torch.as_tensor(d, device=cuda) @ C.T
        refs.append(hf.get_jk(m, d))
    vj, vk = opt.jk_cart(big)
    J = 2 * (vj + vj.transpose(-1, -2))
    K = vk + vk.transpose(-1, -2)
    for b, (rj, rk) in enumerate(refs):
        C = torch.as_tensor(opt.coeffs[b], device=cuda)
        o0, o1 = opt.ao_off[b], opt.ao_off[b + 1]
        jb = (C.T @ J[0, o0:o1, o0:o1] @ C).cpu().numpy()
        kb = (C.T @ K[0, o0:o1, o0:o1] @ C).cpu().numpy()
        assert abs(jb - rj).max() < 1e-9
        assert abs(kb - rk).max() < 1e-9
    # nothing lands outside the diagonal blocks
    mask = torch.ones_like(J[0], dtype=torch.bool)
    for b in range(len(mols)):
        o0, o1 = opt.ao_off[b], opt.ao_off[b + 1]
        mask[o0:o1, o0:o1] = False
    assert float(J[0][mask].abs().max()) == 0.0
    assert float(K[0][mask].abs().max()) == 0.0


def test_batched_jk_graph_replay_matches_eager(cuda):
    """The batched J/K build captured as a CUDA graph (device-scheduled
    tiles, no host round trip) replays to the eager result for new
    densities, twice in a row."""
    import torch
    from byteqc_b200.scf.batched import BatchedVHFOpt, _graphed
    basis = synthetic_basis('cc-pvdz', ['O', 'H'])
    mols = [Mole(water_cluster(k, seed=40 + k), basis) for k in (3, 1, 2)]
    opt = BatchedVHFOpt(mols).build()
    N = opt.nao_cart
    rng = np.random.default_rng(9)

    def dens():
        d = torch.zeros((1, N, N), dtype=torch.float64, device=cuda)
        for b in range(len(mols)):
            o0, o1 = opt.ao_off[b], opt.ao_off[b + 1]
            x = torch.as_tensor(rng.random((o1 - o0, o1 - o0)), device=cuda)
            d[0, o0:o1, o0:o1] = x + x.T
        return d

    fn = lambda d: opt.jk_cart(d)
    g = _graphed(fn, dens())
    for _ in range(2):
        d = dens()
        vj0, vk0 = opt.jk_cart(d)
        vj1, vk1 = g(d)
        assert float((vj1 - vj0).abs().max()) < 1e-12 * max(1., float(vj0.abs().max()))
        assert float((vk1 - vk0).abs().max()) < 1e-12 * max(1., float(vk0.abs().max()))
    opt.clear()
