"""Initial densities: superposition of atomic densities (SAD) and core guess.

SAD: one spherically averaged atomic Hartree-Fock per element (fractional
occupation of degenerate shells, DIIS), run through the same device J/K
engine; the atomic densities are placed on the diagonal blocks of the
molecular density.  Core: the density of the lowest eigenvectors of the
core Hamiltonian.
"""
import numpy as np
import torch

from ..gto.mole import Mole

_SAD_CACHE = {}


def _aufbau_fractional(mo_e, nelec, tol=1e-4):
    """Occupations in [0, 2] filling degenerate groups with equal fractions."""
    order = torch.argsort(mo_e)
    e = mo_e[order].cpu().numpy()
    occ = np.zeros(len(e))
    left = float(nelec)
    i = 0
    while left > 1e-12 and i < len(e):
        j = i + 1
        while j < len(e) and abs(e[j] - e[i]) < tol:
            j += 1
        cap = 2. * (j - i)
        put = min(cap, left)
        occ[i:j] = put / (j - i)
        left -= put
        i = j
    out = torch.zeros_like(mo_e)
    out[order] = torch.as_tensor(occ, dtype=mo_e.dtype, device=mo_e.device)
    return out


def atomic_density(symbol, basis, max_cycle=60, conv_tol=1e-9):
    """Spherically averaged atomic density of one element in the AO basis."""
    from .hf import RHF
    key = (symbol, repr(basis.get(symbol)))
    if key in _SAD_CACHE:
        return _SAD_CACHE[key]
    mol = Mole([(symbol, (0., 0., 0.))], {symbol: basis[symbol]}, unit='Bohr')
    mf = RHF(mol)
    S = mf.get_ovlp()
    h = mf.get_hcore()
    ne = mol.nelectron
    mo_e, mo_c = mf._eigh(h, S)
    occ = _aufbau_fractional(mo_e, ne)
    dm = (mo_c * occ) @ mo_c.T
    mf._diis_reset()
    e_last = None
    for _ in range(max_cycle):
        vj, vk = mf.opt.jk_ao(dm[None])
        F = h + vj[0] - .5 * vk[0]
        e = float(.5 * torch.sum(dm * (h + F)))
        if e_last is not None and abs(e - e_last) < conv_tol:
            break
        e_last = e
        Fd = mf._diis(F, F @ dm @ S - S @ dm @ F)
        mo_e, mo_c = mf._eigh(Fd, S)
        occ = _aufbau_fractional(mo_e, ne)
        dm = (mo_c * occ) @ mo_c.T
    _SAD_CACHE[key] = dm
    return dm


def init_guess(mf, kind='sad'):
    mol = mf.mol
    if kind in ('1e', 'hcore', 'core'):
        e, c = mf._eigh(mf.get_hcore(), mf.get_ovlp())
        nocc = mol.nelectron // 2
        c = c[:, torch.argsort(e)[:nocc]]
        return 2. * c @ c.T
    if kind == 'mlp':
        from ..learned.infer import mlp_density, weights_for
        path = getattr(mf, 'mlp_weights', None) or weights_for(mol)
        if path is None:
            raise FileNotFoundError('no trained density model for the basis shape %r'
                                    % getattr(mol, 'basis_name', 'cc-pvdz'))
        return mlp_density(mf, init_guess(mf, 'sad'), path)
    if kind not in ('sad', 'minao', 'atom'):
        raise ValueError('unknown init_guess %r' % kind)
    nao = mol.nao
    dm = torch.zeros((nao, nao), dtype=torch.float64, device=mf.get_ovlp().device)
    slices = mol.aoslice_by_atom()
    for ia, (sym, _) in enumerate(mol.atom):
        d = atomic_density(sym, mol.basis)
        p0, p1 = slices[ia, 2], slices[ia, 3]
        dm[p0:p1, p0:p1] = d
    # renormalise to the molecular electron count
    ne = float(torch.sum(dm * mf.get_ovlp()))
    if ne > 0:
        dm *= mol.nelectron / ne
    return dm
