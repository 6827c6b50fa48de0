"""Parity on the benchmark configurations and on the reference's calling
sequences (needs a B200).

* C1: (H2O)_4 in the cc-pVDZ shape (96 AO): SCF to 1e-10 against the CPU
  oracle's RHF (energy within 1e-9 Eh) and J/K on the density of the
  reference's timing script (cuobc/test/jk.py) against the oracle.
* C3: all-trans C60H122 in the 6-31G** shape (1450 AO): the FP32 band below
  1e-6 against the plain FP64 build on the converged density and on a
  difference density of the SCF, and the mixed-precision SCF energy.
* The drop-in as cuobc drives it: the reference's host logic (Schwarz pair
  lists sorted by q, log-q bins, nbins > 1, class-level density screen,
  cuobc/scf/hf.py:91-180) calling this library's GINTbuild_jk, against the
  oracle.
* get_veff (pyscf's direct-SCF potential) and an open-shell UHF against the
  oracle's UHF.
* The reference's SCF path of the benchmark's reference arm (its kernels from
  oracle/_ref) against this engine's RHF.
"""
import numpy as np
import pytest

from byteqc_b200.gto.mole import Mole
from byteqc_b200.gto.basis import synthetic_basis
from byteqc_b200.gto.geom import water_cluster, linear_alkane
from oracle import oracle

pytestmark = pytest.mark.gpu

TOL_JK = 1e-10


def _jkpy_dm(nao, seed=2341, scale=0.1):
    rng = np.random.default_rng(seed)
    dm = rng.random((nao, nao))
    return scale * (dm + dm.T)


def test_c1_water4_dz_scf_and_jk(cuda):
    from byteqc_b200.scf import hf
    mol = Mole(water_cluster(4, seed=0), synthetic_basis('cc-pvdz', ['O', 'H']))
    assert mol.nao == 96
    mf = hf.RHF(mol)
    mf.conv_tol = 1e-10
    e = mf.kernel()
    assert mf.converged
    e_ref, _, _ = oracle.rhf(mol, conv_tol=1e-11)
    print('C1 SCF: E %.12f oracle %.12f |dE| %.2e' % (e, e_ref, abs(e - e_ref)))
    assert abs(e - e_ref) < 1e-9
    dm = _jkpy_dm(mol.nao)
    vj, vk = hf.get_jk(mol, dm, vhfopt=mf.opt)
    rj, rk = oracle.get_jk(mol, dm)
    ej, ek = abs(vj - rj).max(), abs(vk - rk).max()
    print('C1 J/K: max|J| %.3g max|dJ| %.3e max|dK| %.3e' % (abs(rj).max(), ej, ek))
    assert ej < TOL_JK and ek < TOL_JK


def test_c3_alkane_mixed_precision(cuda):
    """FP32 for quartets whose bound q_ij q_kl max|D| < 1e-6, FP64 above:
    J/K max-abs error against the plain FP64 build <= 1e-10 on the converged
    density (|J| ~ 40) and on the SCF's second-cycle difference density."""
    import torch
    from byteqc_b200.scf import hf, guess
    mol = Mole(linear_alkane(60), synthetic_basis('6-31g**', ['C', 'H']))
    assert mol.nao == 1450
    guess._SAD_CACHE.clear()
    mf0 = hf.RHF(mol)
    mf0.conv_tol = 1e-9
    ddm = []
    mf0.jk_hook = lambda d, f: ddm.append(d.clone()) if len(ddm) < 2 else None
    e0 = mf0.kernel()
    assert mf0.converged
    opt = mf0.opt
    for label, d in (('converged', mf0.dm), ('cycle-2 difference', ddm[1])):
        d = d[None]
        vj0, vk0 = opt.jk_ao(d)
        vj1, vk1 = opt.jk_ao(d, fp32_below=1e-6)
        ej = float((vj1 - vj0).abs().max())
        ek = float((vk1 - vk0).abs().max())
        print('C3 %s: max|J| %.3g max|dJ| %.3e max|dK| %.3e' % (label, float(vj0.abs().max()), ej, ek))
        assert ej < TOL_JK and ek < TOL_JK
    guess._SAD_CACHE.clear()
    mf1 = hf.RHF(mol)
    mf1.conv_tol = 1e-9
    mf1.fp32_threshold = 1e-6
    e1 = mf1.kernel()
    assert mf1.converged
    print('C3 SCF: plain %.10f mixed %.10f |dE| %.2e' % (e0, e1, abs(e1 - e0)))
    assert abs(e1 - e0) < 1e-9
    assert any(rec[1] > 0 for rec in mf1.build_log)


def test_dropin_multibin_gint_build_jk(cuda):
    """cuobc's get_jk host logic (RefVHFOpt pair lists in the reference's
    order, nbins = 10 log-q bins, class-level density screen) driving this
    library's GINTinit_basis_prod_* / GINTbuild_jk, as a drop-in for
    libgint/libgvhf; J/K against the oracle."""
    import torch
    from byteqc_b200 import lib as L
    from oracle import ref_gpu
    lib = L.load_library()
    mol = Mole(water_cluster(3, seed=8), synthetic_basis('cc-pvtz', ['O', 'H']))
    opt = ref_gpu.RefVHFOpt(mol).build(1e-13)
    jk = ref_gpu.RefJK(opt, libs=(lib, lib))
    assert jk.nbins >= 10
    C = torch.as_tensor(opt.coeff, device=cuda)
    dm = _jkpy_dm(mol.nao, seed=5)
    dmc = (C @ torch.as_tensor(dm, device=cuda) @ C.T)[None].contiguous()
    tasks = jk.tasks(dmc)
    assert any(len(np.unique(bi)) > 2 for _, _, bi, _ in tasks)   # several non-empty bins
    J, K = jk.jk_cart(dmc, tasks=tasks)
    J = (C.T @ J[0] @ C).cpu().numpy()
    K = (C.T @ K[0] @ C).cpu().numpy()
    jk.close()
    rj, rk = oracle.get_jk(mol, dm)
    ej, ek = abs(J - rj).max(), abs(K - rk).max()
    print('drop-in multi-bin: max|J| %.3g max|dJ| %.3e max|dK| %.3e' % (abs(rj).max(), ej, ek))
    # the bins drop quartets below 1e-13 / max|D_class| only
    assert ej < TOL_JK and ek < TOL_JK


def test_get_veff_direct_scf(cuda):
    """RHF.get_veff: J - K/2 for a density, and the incremental form
    vhf_last + veff(dm - dm_last) equals the full potential."""
    from byteqc_b200.scf import hf
    mol = Mole(water_cluster(2, seed=3), synthetic_basis('cc-pvdz', ['O', 'H']))
    mf = hf.RHF(mol)
    d0 = _jkpy_dm(mol.nao, seed=1, scale=0.05)
    d1 = d0 + _jkpy_dm(mol.nao, seed=2, scale=0.005)
    v0 = mf.get_veff(mol, d0)
    rj, rk = oracle.get_jk(mol, d0)
    assert abs(v0 - (rj - .5 * rk)).max() < TOL_JK
    v1 = mf.get_veff(mol, d1, dm_last=d0, vhf_last=v0)
    rj, rk = oracle.get_jk(mol, d1)
    assert abs(v1 - (rj - .5 * rk)).max() < TOL_JK


def test_uhf_open_shell_against_oracle(cuda):
    """Doublet water cation: the engine's UHF and the oracle's UHF from the
    same initial densities converge to the same energy; UHF.get_veff at the
    converged densities equals the oracle's potentials."""
    import torch
    from byteqc_b200.scf import hf
    mol = Mole(water_cluster(1, seed=2), synthetic_basis('cc-pvdz', ['O', 'H']), charge=1, spin=1)
    na, nb = mol.nelec
    assert (na, nb) == (5, 4)
    S, T, V = oracle.int1e(mol)
    h = T + V
    seig, U = np.linalg.eigh(S)
    X = U / np.sqrt(seig)
    e, c = np.linalg.eigh(X.T @ h @ X)
    c = X @ c
    dm0 = np.stack([c[:, :na] @ c[:, :na].T, c[:, :nb] @ c[:, :nb].T])
    mf = hf.UHF(mol)
    mf.conv_tol = 1e-10
    mf.max_cycle = 200
    e_gpu = mf.kernel(dm0)
    assert mf.converged
    e_ref, dm_ref, _ = oracle.uhf(mol, conv_tol=1e-10, dm0=dm0)
    print('UHF doublet: E %.12f oracle %.12f |dE| %.2e' % (e_gpu, e_ref, abs(e_gpu - e_ref)))
    assert abs(e_gpu - e_ref) < 1e-9
    dm = mf.dm.cpu().numpy()
    v = mf.get_veff(mol, dm)
    rj, rk = oracle.get_jk(mol, dm)
    ref_v = np.stack([rj[0] + rj[1] - rk[0], rj[0] + rj[1] - rk[1]])
    assert v.shape == (2, mol.nao, mol.nao)
    assert abs(v - ref_v).max() < TOL_JK
    with pytest.raises(ValueError):
        mf.get_veff(mol, dm[0])


def test_reference_scf_path_matches_engine(cuda):
    """The benchmark's reference arm (the reference's kernels and host logic,
    oracle/ref_scf.py) converges to the engine's RHF energy."""
    from byteqc_b200.scf import hf
    from oracle import ref_gpu
    from oracle.ref_scf import RefSCF
    if not ref_gpu.available():
        pytest.skip('reference libraries not built (oracle/build_ref.sh)')
    mol = Mole(water_cluster(2, seed=1), synthetic_basis('cc-pvdz', ['O', 'H']))
    ref = RefSCF(mol, conv_tol=1e-10)
    e_ref = ref.kernel()
    ref.close()
    assert ref.converged
    mf = hf.RHF(mol)
    mf.conv_tol = 1e-10
    e = mf.kernel()
    print('reference SCF path: E %.12f engine %.12f (%d / %d cycles)' % (e_ref, e, ref.cycles, mf.cycles))
    assert abs(e - e_ref) < 1e-9
