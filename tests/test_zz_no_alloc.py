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


def _driver_pool_high(dev=0):
    """Used-memory high watermark of the device's default stream-ordered
    memory pool (driver API), which cudaMallocAsync draws from."""
    import ctypes
    cu = ctypes.CDLL('libcuda.so.1')
    pool = ctypes.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), ctypes.c_int(dev)) == 0
    val = ctypes.c_uint64(0)
    CU_MEMPOOL_ATTR_USED_MEM_HIGH = 8
    assert cu.cuMemPoolGetAttribute(pool, ctypes.c_int(CU_MEMPOOL_ATTR_USED_MEM_HIGH),
                                    ctypes.byref(val)) == 0
    return cu, pool, val.value


def _reset_pool_high(cu, pool):
    import ctypes
    zero = ctypes.c_uint64(0)
    assert cu.cuMemPoolSetAttribute(pool, ctypes.c_int(8), ctypes.byref(zero)) == 0


def test_noalloc_allocates_nothing():
    """After a warm-up call, two more calls leave the device's free memory
    and the default memory pool's high watermark unchanged, while the
    allocating entry point does raise that watermark (so the probe sees
    stream-ordered allocations); a NULL pair_q is refused."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from byteqc_b200 import lib as L
    from byteqc_b200.scf import hf
    lib = L.load_library()
    mol = Mole(water_cluster(2, seed=9), synthetic_basis('cc-pvdz', ['O', 'H']))
    opt = hf._VHFOpt(mol).build()
    rng = np.random.default_rng(6)
    dm = rng.random((mol.nao, mol.nao))
    C = opt.coeff_dev
    dmc = (C @ torch.as_tensor(dm + dm.T, device='cuda') @ C.T)[None].contiguous()
    vj = torch.zeros_like(dmc)
    vk = torch.zeros_like(dmc)
    bp = ctypes.cast(opt.bpcache, ctypes.c_void_p)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        vj.zero_()
        vk.zero_()
        err = lib.BQCbuild_jk_noalloc(bp, _vp(opt.pair_q), _vp(vj), _vp(vk), _vp(dmc),
                                      ctypes.c_int(dmc.shape[-1]), ctypes.c_int(1),
                                      ctypes.c_double(opt.direct_scf_tol), stream)
        torch.cuda.synchronize()
        return err

    assert call() == 0   # warm-up: the device address look-up
    cu, pool, _ = _driver_pool_high()
    _reset_pool_high(cu, pool)
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        assert call() == 0
    free1 = torch.cuda.mem_get_info()[0]
    _, _, high = _driver_pool_high()
    assert high == 0, high
    assert free1 == free0
    err, _, _ = _build(lib, opt, dmc, noalloc=False)      # positive control
    assert err == 0
    _, _, high = _driver_pool_high()
    assert high > 0
    # no Schwarz factors: refused
    assert lib.BQCbuild_jk_noalloc(bp, None, _vp(vj), _vp(vk), _vp(dmc), ctypes.c_int(dmc.shape[-1]),
                                   ctypes.c_int(1), ctypes.c_double(1e-13), stream) == 3
