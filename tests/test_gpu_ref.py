"""The reference's own GPU J/K kernels as a second checker (needs a B200 and
oracle/_ref/, built from the reference sources by oracle/build_ref.sh).

The reference libraries are driven through the same C ABI as this package's:
its GINTinit_basis_prod_cpu/_gpu build its own basis-product cache from the
engine's pair lists (padding pairs removed), and its GINTbuild_jk runs every
class pair with one bin (no density screening).  J and K must agree with the
CPU oracle and with this engine to 1e-10.  With the reference's own host
screening (oracle/ref_gpu.py: log q bins, class-level density bound) the two
builds differ only by what each screen drops.
"""
import ctypes
import os

import numpy as np
import pytest

from byteqc_b200.gto.mole import Mole
from byteqc_b200.gto.basis import synthetic_basis
from byteqc_b200.gto.geom import water_cluster
from oracle import oracle

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle', '_ref')


def _ref_libs():
    gint = os.path.join(REF, 'libgint.so')
    gvhf = os.path.join(REF, 'libgvhf.so')
    if not (os.path.exists(gint) and os.path.exists(gvhf)):
        pytest.skip('reference libraries not built (oracle/build_ref.sh)')
    lg = ctypes.CDLL(gint, mode=ctypes.RTLD_GLOBAL)
    lv = ctypes.CDLL(gvhf)
    return lg, lv


@pytest.mark.parametrize('kind', ['cc-pvdz', 'cc-pvtz'])
def test_reference_kernels_agree(cuda, kind):
    import torch
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    lg, lv = _ref_libs()
    mol = Mole(water_cluster(2, seed=5), synthetic_basis(kind, ['O', 'H']))
    opt = hf._VHFOpt(mol).build()
    pmol = opt.mol
    # engine pair lists without the padding pairs of the tile layout
    keep = ~opt.pair_dummy
    locs = opt.bas_pairs_locs
    p2s, new_locs = [], [0]
    for c in range(opt.ncptype):
        k = keep[locs[c]:locs[c + 1]]
        p2s.append(opt.bas_pair2shls[:, locs[c]:locs[c + 1]][:, k])
        new_locs.append(new_locs[-1] + int(k.sum()))
    p2s = np.ascontiguousarray(np.hstack(p2s), dtype=np.int32)
    new_locs = np.asarray(new_locs, dtype=np.int32)
    ncp = opt.ncptype
    atm = np.ascontiguousarray(pmol._atm, dtype=np.int32)
    bas = np.ascontiguousarray(pmol._bas, dtype=np.int32)
    env = np.ascontiguousarray(pmol._env)
    bas_coords = np.empty(pmol.nbas * 3)
    bp = ctypes.POINTER(L.BasisProdCache)()
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lg.GINTinit_basis_prod_cpu(ctypes.byref(bp), ctypes.c_double(0.5), vp(bas_coords), vp(p2s),
                               vp(new_locs), ctypes.c_int(ncp), vp(atm), ctypes.c_int(pmol.natm),
                               vp(bas), ctypes.c_int(pmol.nbas), vp(env))
    nprim = bp.contents.primitive_pairs_locs[ncp]
    aexyz = np.ctypeslib.as_array(bp.contents.aexyz, (nprim * 5,)).copy()
    dev = cuda
    d_ao = torch.as_tensor(pmol.ao_loc_nr(cart=True), dtype=torch.int32, device=dev)
    d_xyz = torch.as_tensor(bas_coords, device=dev)
    d_ae = torch.as_tensor(aexyz, device=dev)
    d_p2s = torch.as_tensor(p2s.ravel(), device=dev)
    bpg = ctypes.POINTER(L.BasisProdCache)()
    tp = lambda t: ctypes.c_void_p(t.data_ptr())
    lg.GINTinit_basis_prod_gpu(ctypes.byref(bp), ctypes.byref(bpg), tp(d_ao), tp(d_xyz), tp(d_ae),
                               tp(d_p2s))
    rng = np.random.default_rng(2341)
    dm = rng.random((mol.nao, mol.nao))
    dm = dm + dm.T
    C = opt.coeff_dev
    dmc = (C @ torch.as_tensor(dm, device=dev) @ C.T)[None].contiguous()
    nao = dmc.shape[-1]
    vj = torch.zeros_like(dmc)
    vk = torch.zeros_like(dmc)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for cij in range(ncp):
        for ckl in range(cij + 1):
            nij = new_locs[cij + 1] - new_locs[cij]
            nkl = new_locs[ckl + 1] - new_locs[ckl]
            if nij == 0 or nkl == 0:
                continue
            bi = np.array([0, nij], dtype=np.int32)
            bk = np.array([0, nkl], dtype=np.int32)
            err = lv.GINTbuild_jk(bpg, tp(vj), tp(vk), tp(dmc), ctypes.c_int(nao), ctypes.c_int(1),
                                  vp(bi), vp(bk), ctypes.c_int(1), ctypes.c_int(cij),
                                  ctypes.c_int(ckl), stream)
            assert err == 0
    torch.cuda.synchronize()
    J = 2 * (vj + vj.transpose(-1, -2))
    K = vk + vk.transpose(-1, -2)
    J = (C.T @ J[0] @ C).cpu().numpy()
    K = (C.T @ K[0] @ C).cpu().numpy()
    rj, rk = oracle.get_jk(mol, dm)
    assert abs(J - rj).max() < 1e-9, abs(J - rj).max()
    assert abs(K - rk).max() < 1e-9, abs(K - rk).max()
    ej, ek = hf.get_jk(mol, dm, vhfopt=opt)
    assert abs(ej - J).max() < 1e-9
    assert abs(ek - K).max() < 1e-9
    # as cuobc/scf/hf.py does, release through the device copy only (it owns
    # the class table and pair block it shares with the host cache)
    lg.GINTdel_basis_prod(ctypes.byref(bpg))


def test_reference_screened_build_agrees(cuda):
    import torch
    from byteqc_b200.scf import hf
    from oracle import ref_gpu
    if not ref_gpu.available():
        pytest.skip('reference libraries not built (oracle/build_ref.sh)')
    mol = Mole(water_cluster(3, seed=2), synthetic_basis('cc-pvdz', ['O', 'H']))
    mf = hf.RHF(mol)
    mf.kernel()
    opt = mf.opt
    ref = ref_gpu.RefJK(opt)
    C = opt.coeff_dev
    dmc = (C @ mf.dm @ C.T)[None].contiguous()
    J1, K1 = opt.jk_cart(dmc)
    J2, K2 = ref.jk_cart(dmc)
    ref.close()
    # both screens drop quartets below 1e-13 only
    assert float((J1 - J2).abs().max()) < 1e-10
    assert float((K1 - K2).abs().max()) < 1e-10
    rj, rk = oracle.get_jk(mol, mf.dm.cpu().numpy())
    J = (C.T @ J2[0] @ C).cpu().numpy()
    K = (C.T @ K2[0] @ C).cpu().numpy()
    assert abs(J - rj).max() < 1e-9
    assert abs(K - rk).max() < 1e-9
