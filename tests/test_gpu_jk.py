"""Parity of the device J/K engine with the CPU oracle (needs a B200).

Tolerances: J and K max-abs error <= 1e-10 in plain FP64 (the bar of the
drop-in), SCF total energy within 1e-9 Eh.
"""
import numpy as np
import pytest

from byteqc_b200.gto.mole import Mole
from byteqc_b200.gto.basis import synthetic_basis, sto3g_like
from byteqc_b200.gto.geom import water_cluster, linear_alkane
from oracle import oracle

pytestmark = pytest.mark.gpu

TOL_JK = 1e-10


def _rand_dm(nao, seed=2341):
    # the density recipe of the reference's timing script: rand + rand^T
    rng = np.random.default_rng(seed)
    dm = rng.random((nao, nao))
    return dm + dm.T


def _mol(kind, nw=1, seed=3):
    atoms = water_cluster(nw, seed=seed)
    return Mole(atoms, synthetic_basis(kind, ['O', 'H']))


@pytest.mark.parametrize('kind', ['cc-pvdz', 'cc-pvtz'])
def test_jk_water(cuda, kind):
    from byteqc_b200.scf import hf
    mol = _mol(kind)
    dm = _rand_dm(mol.nao)
    vj, vk = hf.get_jk(mol, dm)
    rj, rk = oracle.get_jk(mol, dm)
    ej, ek = abs(vj - rj).max(), abs(vk - rk).max()
    print('water %s: max|J| %.3g max|dJ| %.3e max|dK| %.3e' % (kind, abs(rj).max(), ej, ek))
    assert ej < TOL_JK and ek < TOL_JK


@pytest.mark.parametrize('variant', [1, 2])
def test_jk_class_variants(cuda, variant):
    """Every class in the group kernel (1) or, where it splits, in ket-split
    tile launches (2): the same J/K as the oracle."""
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    lib = L.load_library()
    shapes = [(a, b, c, d) for a in range(4) for b in range(a + 1)
              for c in range(4) for d in range(c + 1)]
    try:
        for sh in shapes:
            assert lib.BQCset_class_variant(*sh, variant) == 0
        mol = _mol('cc-pvtz', nw=2, seed=4)
        dm = _rand_dm(mol.nao) * 0.1
        vj, vk = hf.get_jk(mol, dm)
    finally:
        for sh in shapes:
            lib.BQCset_class_variant(*sh, 0)
    rj, rk = oracle.get_jk(mol, dm)
    print('variant %d: max|dJ| %.3e max|dK| %.3e' % (variant, abs(vj - rj).max(), abs(vk - rk).max()))
    assert abs(vj - rj).max() < TOL_JK
    assert abs(vk - rk).max() < TOL_JK
    assert lib.BQCset_class_variant(0, 0, 0, 0, 7) == 3
    assert lib.BQCset_class_variant(4, 0, 0, 0, 1) == 2


def test_jk_batch_and_flags(cuda):
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvdz')
    dms = np.stack([_rand_dm(mol.nao, s) for s in (1, 2)])
    opt = hf._VHFOpt(mol).build()
    vj, vk = hf.get_jk(mol, dms, vhfopt=opt)
    assert vj.shape == dms.shape and vk.shape == dms.shape
    for i in range(2):
        rj, rk = oracle.get_jk(mol, dms[i])
        assert abs(vj[i] - rj).max() < TOL_JK
        assert abs(vk[i] - rk).max() < TOL_JK
    vj_only, vk_none = hf.get_jk(mol, dms[0], vhfopt=opt, with_k=False)
    assert vk_none is None and abs(vj_only - vj[0]).max() < 1e-12
    vj_none, vk_only = hf.get_jk(mol, dms[0], vhfopt=opt, with_j=False)
    assert vj_none is None and abs(vk_only - vk[0]).max() < 1e-12
    with pytest.raises(NotImplementedError):
        hf.get_jk(mol, dms[0], hermi=0, vhfopt=opt)
    with pytest.raises(NotImplementedError):
        hf.get_jk(mol, dms[0], vhfopt=opt, omega=0.3)


def test_jk_two_waters_tz(cuda):
    """Every s-f class pair of the TZ-shaped basis, inter-molecular pairs included."""
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvtz', nw=2, seed=5)
    dm = _rand_dm(mol.nao, 7)
    vj, vk = hf.get_jk(mol, dm)
    rj, rk = oracle.get_jk(mol, dm)
    ej, ek = abs(vj - rj).max(), abs(vk - rk).max()
    print('TZ dimer: max|J| %.3g max|dJ| %.3e max|dK| %.3e' % (abs(rj).max(), ej, ek))
    assert ej < TOL_JK and ek < TOL_JK


def test_schwarz_and_int1e(cuda):
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvtz')
    opt = hf._VHFOpt(mol).build()
    S, T, V = [x.cpu().numpy() for x in opt.int1e()]
    rS, rT, rV = oracle.int1e(mol)
    assert abs(S - rS).max() < 1e-12
    assert abs(T - rT).max() < 1e-10
    assert abs(V - rV).max() < 1e-10
    # Schwarz factors of the kept pairs against the oracle's (ij|ij)
    q = oracle.q_cond(opt.mol)
    real = ~opt.pair_dummy          # padding pairs of the tile layout carry q = 0
    p2s = opt.bas_pair2shls[:, real]
    dev_q = opt.pair_q.cpu().numpy()[real]
    ref = q[p2s[0], p2s[1]]
    assert np.allclose(dev_q, ref, rtol=1e-10, atol=1e-14)
    assert (opt.pair_q.cpu().numpy()[~real] == 0).all()


def test_gint_abi_matches_native(cuda):
    """The reference-ABI entry point GINTbuild_jk, driven the way
    cuobc/scf/hf.py drives it (class pairs x bins), equals the native build."""
    import ctypes
    import torch
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvdz', nw=2, seed=11)
    opt = hf._VHFOpt(mol).build()
    lib = L.load_library()
    dm = _rand_dm(mol.nao, 3)
    C = opt.coeff_dev
    dmc = (C @ torch.as_tensor(dm, device=cuda) @ C.T)[None].contiguous()
    nao = dmc.shape[-1]
    vj = torch.zeros_like(dmc)
    vk = torch.zeros_like(dmc)
    # the native pair lists are laid out in shell-grouped tiles (q is not
    # globally sorted, padding pairs are interleaved), so drive GINTbuild_jk
    # with one bin that spans each whole class
    nbins = 1
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for cij in range(opt.ncptype):
        for ckl in range(cij + 1):
            if len(opt.log_qs[cij]) == 0 or len(opt.log_qs[ckl]) == 0:
                continue
            bi = np.array([0, len(opt.log_qs[cij])], dtype=np.int32)
            bk = np.array([0, len(opt.log_qs[ckl])], dtype=np.int32)
            err = lib.GINTbuild_jk(opt.bpcache, ctypes.c_void_p(vj.data_ptr()),
                                   ctypes.c_void_p(vk.data_ptr()), ctypes.c_void_p(dmc.data_ptr()),
                                   ctypes.c_int(nao), ctypes.c_int(1),
                                   bi.ctypes.data_as(ctypes.c_void_p),
                                   bk.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(nbins),
                                   ctypes.c_int(cij), ctypes.c_int(ckl), stream)
            assert err == 0
    J = 2 * (vj + vj.transpose(-1, -2))
    K = vk + vk.transpose(-1, -2)
    J = (C.T @ J[0] @ C).cpu().numpy()
    K = (C.T @ K[0] @ C).cpu().numpy()
    rj, rk = oracle.get_jk(mol, dm)
    print('GINT ABI: max|J| %.3g max|dJ| %.3e max|dK| %.3e' % (abs(rj).max(), abs(J - rj).max(),
                                                             abs(K - rk).max()))
    assert abs(J - rj).max() < TOL_JK
    assert abs(K - rk).max() < TOL_JK


def test_rhf_energy(cuda):
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvdz', nw=2, seed=1)
    mf = hf.RHF(mol)
    mf.conv_tol = 1e-10
    e = mf.kernel()
    assert mf.converged
    e_ref, _, _ = oracle.rhf(mol, conv_tol=1e-11)
    assert abs(e - e_ref) < 1e-9


def test_host_loop_matches_device_loop(cuda):
    """The drop-in arrangement (host numpy SCF loop, get_jk with host
    densities, host DIIS) converges to the device loop's energy, in plain
    FP64 and in the fast form."""
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvdz', nw=2, seed=1)
    for fast in (False, True):
        ms = []
        for host in (False, True):
            mf = hf.RHF(mol)
            mf.conv_tol = 1e-10
            if fast:
                mf.fp32_threshold = 1e-4
                mf.early_tol = 1e-10
            e = mf.kernel_hostloop() if host else mf.kernel()
            assert mf.converged
            ms.append(e)
        assert abs(ms[0] - ms[1]) < 1e-9, (fast, ms)


def test_uhf_closed_shell_equals_rhf(cuda):
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvdz', nw=1, seed=2)
    e_r = hf.RHF(mol).kernel()
    mf = hf.UHF(mol)
    e_u = mf.kernel()
    assert abs(e_r - e_u) < 1e-8


def test_alkane_631gss(cuda):
    from byteqc_b200.scf import hf
    mol = Mole(linear_alkane(2), synthetic_basis('6-31g**', ['C', 'H']))
    dm = _rand_dm(mol.nao, 5) * 0.1
    vj, vk = hf.get_jk(mol, dm)
    rj, rk = oracle.get_jk(mol, dm)
    print('ethane: max|J| %.3g max|dJ| %.3e max|dK| %.3e' % (abs(rj).max(), abs(vj - rj).max(),
                                                           abs(vk - rk).max()))
    assert abs(vj - rj).max() < TOL_JK
    assert abs(vk - rk).max() < TOL_JK


def test_mixed_precision_jk_error(cuda):
    """FP32 band below 1e-6: J/K error against the FP64 build stays small."""
    import torch
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvtz', nw=2, seed=5)
    opt = hf._VHFOpt(mol).build()
    rng = np.random.default_rng(8)
    dm = rng.random((mol.nao, mol.nao)) * 1e-3
    dm = torch.as_tensor(dm + dm.T, device=cuda)[None]
    vj0, vk0 = opt.jk_ao(dm)
    vj1, vk1 = opt.jk_ao(dm, fp32_below=1e-6)
    ej = float((vj1 - vj0).abs().max())
    ek = float((vk1 - vk0).abs().max())
    assert ej < 1e-9 and ek < 1e-9, (ej, ek)
    # every quartet is in the FP32 band: still within FP32 accuracy of FP64
    vj2, vk2 = opt.jk_ao(dm, fp32_below=1e30)
    assert float((vj2 - vj0).abs().max()) < 1e-5 * float(vj0.abs().max())
    assert float((vk2 - vk0).abs().max()) < 1e-5 * float(vk0.abs().max())


def test_mixed_precision_scf_energy(cuda):
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvdz', nw=3, seed=4)
    mf0 = hf.RHF(mol)
    mf0.conv_tol = 1e-10
    e0 = mf0.kernel()
    mf1 = hf.RHF(mol)
    mf1.conv_tol = 1e-10
    mf1.fp32_threshold = 1e-6
    e1 = mf1.kernel()
    mf2 = hf.RHF(mol)
    mf2.conv_tol = 1e-10
    mf2.fp32_threshold = 1e-6
    mf2.early_tol = 1e-10
    e2 = mf2.kernel()
    assert mf0.converged and mf1.converged and mf2.converged
    assert abs(e1 - e0) < 1e-9
    assert abs(e2 - e0) < 1e-9
    assert any(rec[1] > 0 for rec in mf1.build_log)


def test_autotune_keeps_results(cuda):
    """The autotuner picks kernels per class; J/K stay the same."""
    import torch
    from byteqc_b200 import autotune
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvtz', nw=2, seed=6)
    opt = hf._VHFOpt(mol).build()
    dm = torch.as_tensor(_rand_dm(mol.nao) * 0.1, device=cuda)[None]
    vj0, vk0 = opt.jk_ao(dm)
    try:
        choice = autotune.tune(opt, reps=1)
        assert choice and set(choice.values()) <= {1, 2}
        vj1, vk1 = opt.jk_ao(dm)
    finally:
        lib = L.load_library()
        for key in choice:
            lib.BQCset_class_variant(*key, 0)
    assert float((vj1 - vj0).abs().max()) < 1e-11
    assert float((vk1 - vk0).abs().max()) < 1e-11


@pytest.mark.parametrize('kind', ['cc-pvdz', 'cc-pvtz'])
def test_fill_int2e_matches_oracle(cuda, kind):
    """GINTfill_int2e (the ERI writer) over every ordered class pair writes
    the Cartesian (ij|kl) blocks of the listed pairs; they equal the oracle's
    integrals of the same decontracted, sorted basis."""
    import ctypes
    import torch
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    from byteqc_b200.scf.hf import _stream
    lib = L.load_library()
    mol = _mol(kind)
    opt = hf._VHFOpt(mol).build(diag_block_with_triu=True)
    pmol = opt.mol
    n = int(pmol.ao_loc_nr(cart=True)[-1])
    eri = torch.zeros((n, n, n, n), dtype=torch.float64, device=cuda)
    strides = np.array([n ** 3, n ** 2, n, 1], dtype=np.int32)
    offs = np.zeros(4, dtype=np.int32)
    locs = opt.bas_pairs_locs
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    for cij in range(opt.ncptype):
        for ckl in range(opt.ncptype):
            nij, nkl = locs[cij + 1] - locs[cij], locs[ckl + 1] - locs[ckl]
            if nij == 0 or nkl == 0:
                continue
            bi = np.array([0, nij], dtype=np.int32)
            bk = np.array([0, nkl], dtype=np.int32)
            err = lib.GINTfill_int2e(ctypes.cast(opt.bpcache, ctypes.c_void_p),
                                     ctypes.c_void_p(eri.data_ptr()), n, vp(strides), vp(offs),
                                     vp(bi), vp(bk), 1, cij, ckl, _stream())
            assert err == 0
    torch.cuda.synchronize()
    got = eri.cpu().numpy()
    ref = oracle.eri_full_cart(pmol)
    ao = pmol.ao_loc_nr(cart=True)
    keep = ~opt.pair_dummy
    pairs = [(int(i), int(j)) for i, j, kp in zip(*opt.bas_pair2shls, keep) if kp]
    mask = np.zeros((n, n), bool)
    for i, j in pairs:
        mask[ao[i]:ao[i + 1], ao[j]:ao[j + 1]] = True
    sel = mask[:, :, None, None] & mask[None, None, :, :]
    assert sel.sum() > 0
    err = abs(got[sel] - ref[sel]).max()
    assert err < 1e-10 * max(1., abs(ref).max()), err
    # nothing is written outside the listed pairs
    assert abs(got[~sel]).max() == 0
    # a missing output buffer is an argument error
    assert lib.GINTfill_int2e(ctypes.cast(opt.bpcache, ctypes.c_void_p), None, n, vp(strides),
                              vp(offs), vp(bi), vp(bk), 1, 0, 0, _stream()) == 3


@pytest.mark.parametrize('fp32_below', [0., 1e-6])
def test_device_schedule_matches_host_pruning(cuda, fp32_below):
    """BQCbuild_jk_plan (tiles pruned and counted on the device, persistent
    launches) gives the J/K of BQCbuild_jk (tiles pruned on the host) for
    two densities at once, with and without the FP32 band."""
    import ctypes
    import torch
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    from byteqc_b200.scf.hf import _ptr, _stream
    lib = L.load_library()
    mol = _mol('cc-pvtz', nw=3, seed=12)
    opt = hf._VHFOpt(mol).build()
    rng = np.random.default_rng(3)
    d = rng.random((2, mol.nao, mol.nao)) * 1e-2
    C = opt.coeff_dev
    dmc = (C @ torch.as_tensor(d + d.transpose(0, 2, 1), device=cuda) @ C.T).contiguous()
    nao = dmc.shape[-1]
    dm_cond = torch.empty((opt.mol.nbas, opt.mol.nbas), dtype=torch.float64, device=cuda)
    assert lib.BQCdm_cond(_ptr(dmc), 2, nao, _ptr(opt._mem['ao_loc']), opt.mol.nbas, _ptr(dm_cond),
                          _stream()) == 0
    out = []
    for plan in (False, True):
        vj = torch.zeros_like(dmc)
        vk = torch.zeros_like(dmc)
        if plan:
            err = lib.BQCbuild_jk_plan(opt._plan, _ptr(opt.pair_q), _ptr(dm_cond), _ptr(vj), _ptr(vk),
                                       _ptr(dmc), nao, 2, opt.direct_scf_tol, fp32_below, _stream())
        else:
            err = lib.BQCbuild_jk(ctypes.cast(opt.bpcache, ctypes.c_void_p), _ptr(opt.pair_q),
                                  opt.pair_q_host.ctypes.data_as(ctypes.c_void_p), _ptr(dm_cond),
                                  float(dm_cond.max()), _ptr(vj), _ptr(vk), _ptr(dmc), nao, 2,
                                  opt.direct_scf_tol, fp32_below, None, _stream())
        assert err == 0
        out.append((vj, vk))
    torch.cuda.synchronize()
    (j0, k0), (j1, k1) = out
    assert float((j1 - j0).abs().max()) < 1e-12 * max(1., float(j0.abs().max()))
    assert float((k1 - k0).abs().max()) < 1e-12 * max(1., float(k0.abs().max()))
    assert float(j0.abs().max()) > 0


def test_repeated_builds_agree(cuda):
    """Two builds of the same density differ only by the order of the FP64
    atomic additions: at most a few units in the last place of the largest
    element (bound 1e-13 relative)."""
    import torch
    from byteqc_b200.scf import hf
    mol = _mol('cc-pvtz', nw=3, seed=13)
    opt = hf._VHFOpt(mol).build()
    dm = torch.as_tensor(_rand_dm(mol.nao, 17) * 0.1, device=cuda)[None]
    vj0, vk0 = opt.jk_ao(dm)
    vj1, vk1 = opt.jk_ao(dm)
    dj = float((vj1 - vj0).abs().max()) / float(vj0.abs().max())
    dk = float((vk1 - vk0).abs().max()) / float(vk0.abs().max())
    print('repeat: relative max|dJ| %.2e max|dK| %.2e' % (dj, dk))
    assert dj < 1e-13 and dk < 1e-13
