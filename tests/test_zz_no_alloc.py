"""The J/K entry point that allocates nothing (BQCbuild_jk_noalloc).

It serves callers that hand the library only their own input and output
buffers and forbid it any device allocation (a host program that carves all
device memory from a fixed arena at start-up).  The test drives it through
the C ABI and checks it against the allocating entry point BQCbuild_jk on the
same inputs, twice in a row (the shared scratch keeps the previous call's
contents, which must not leak into the next result), and checks that a basis
beyond the stated 512-shell limit is refused.  This file is collected last so
that a failure here stops a -x run only after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from byteqc_b200.gto.mole import Mole
from byteqc_b200.gto.basis import synthetic_basis
from byteqc_b200.gto.geom import water_cluster

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _vp(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def _build(lib, opt, dmc, noalloc):
    import torch
    vj = torch.zeros_like(dmc)
    vk = torch.zeros_like(dmc)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    bp = ctypes.cast(opt.bpcache, ctypes.c_void_p)
    nao, n_dm = dmc.shape[-1], dmc.shape[0]
    if noalloc:
        err = lib.BQCbuild_jk_noalloc(bp, _vp(opt.pair_q), _vp(vj), _vp(vk), _vp(dmc),
                                      ctypes.c_int(nao), ctypes.c_int(n_dm),
                                      ctypes.c_double(opt.direct_scf_tol), stream)
    else:
        dm_cond = torch.empty((opt.mol.nbas, opt.mol.nbas), dtype=torch.float64, device=dmc.device)
        assert lib.BQCdm_cond(_vp(dmc), ctypes.c_int(n_dm), ctypes.c_int(nao),
                              _vp(opt._mem['ao_loc']), ctypes.c_int(opt.mol.nbas), _vp(dm_cond),
                              stream) == 0
        err = lib.BQCbuild_jk(bp, _vp(opt.pair_q), opt.pair_q_host.ctypes.data_as(ctypes.c_void_p),
                              _vp(dm_cond), float(dm_cond.max()), _vp(vj), _vp(vk), _vp(dmc),
                              nao, n_dm, opt.direct_scf_tol, 0., None, stream)
    torch.cuda.synchronize()
    return err, vj, vk


def test_noalloc_matches_allocating_entry_point():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    lib = L.load_library()
    mol = Mole(water_cluster(2, seed=9), synthetic_basis('cc-pvtz', ['O', 'H']))
    opt = hf._VHFOpt(mol).build()
    assert opt.mol.nbas <= 512
    rng = np.random.default_rng(4)
    for call in range(2):
        dm = rng.random((2, mol.nao, mol.nao))
        dm = dm + dm.transpose(0, 2, 1)
        C = opt.coeff_dev
        dmc = (C @ torch.as_tensor(dm, device='cuda') @ C.T).contiguous()
        err0, vj0, vk0 = _build(lib, opt, dmc, noalloc=False)
        err1, vj1, vk1 = _build(lib, opt, dmc, noalloc=True)
        assert err0 == 0 and err1 == 0
        assert float((vj1 - vj0).abs().max()) < TOL * max(1., float(vj0.abs().max()))
        assert float((vk1 - vk0).abs().max()) < TOL * max(1., float(vk0.abs().max()))


def test_noalloc_rejects_basis_beyond_limit():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    lib = L.load_library()
    mol = Mole(water_cluster(30, seed=1), synthetic_basis('cc-pvdz', ['O', 'H']))
    opt = hf._VHFOpt(mol).build()
    assert opt.mol.nbas > 512
    dmc = torch.zeros((1, opt.nao_cart, opt.nao_cart), dtype=torch.float64, device='cuda')
    err, vj, vk = _build(lib, opt, dmc, noalloc=True)
    assert err == 3
    assert float(vj.abs().max()) == 0.0
