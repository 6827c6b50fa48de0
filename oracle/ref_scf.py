"""The reference's SCF path, run with the reference's own GPU J/K kernels.

Test and measurement infrastructure only (the reference arm of bench.py and
the tests); it loads oracle/_ref (libgint, libgvhf compiled from the
reference's cuobc/lib sources) and the CPU oracle, and nothing of the engine
library.

What runs, following cuobc/scf/hf.py and the pyscf 2.5 SCF loop it plugs into:

* set-up: RefVHFOpt (decontraction, shell sort, Schwarz pair lists; the
  Schwarz factors from the CPU oracle in place of libcint) and the
  reference's basis-product cache (hf.py:288-437);
* get_jk (hf.py:53-227): host density to the device, D' = C D C^T, copy back
  to the host for the class-level density screen, one GINTbuild_jk per class
  pair over log-q bins, J = C^T 2(V + V^T) C, K = C^T (V + V^T) C, results
  back to host arrays;
* the SCF loop on the host as pyscf runs it: one-electron integrals (CPU
  oracle, pyscf computes them with libcint on the CPU), incremental Fock
  builds from difference densities (pyscf's direct SCF), DIIS on
  FDS - SDF, the generalized eigenproblem on the GPU (the reference's eig,
  hf.py:253-265, cupy/cuSOLVER; here torch/cuSOLVER), convergence on
  |Delta E|.
* initial guess: superposition of spherically averaged atomic densities
  from fractional-occupation atomic Hartree-Fock with the CPU oracle (pyscf's
  default would be minao; the engine starts from the same kind of guess).
"""
import time

import numpy as np

from . import oracle
from .ref_gpu import RefJK, RefVHFOpt


def _aufbau_fractional(e, nelec, tol=1e-4):
    order = np.argsort(e)
    es = e[order]
    occ = np.zeros(len(e))
    left = float(nelec)
    i = 0
    while left > 1e-12 and i < len(es):
        j = i + 1
        while j < len(es) and abs(es[j] - es[i]) < tol:
            j += 1
        put = min(2. * (j - i), left)
        occ[i:j] = put / (j - i)
        left -= put
        i = j
    out = np.zeros(len(e))
    out[order] = occ
    return out


_ATOM_CACHE = {}


def atomic_density(symbol, basis, max_cycle=60, conv_tol=1e-9):
    """Spherically averaged atomic RHF density (fractional occupation of
    degenerate levels, DIIS) with the CPU oracle's integrals."""
    from byteqc_b200.gto.mole import Mole
    key = (symbol, repr(basis.get(symbol)))
    if key in _ATOM_CACHE:
        return _ATOM_CACHE[key]
    mol = Mole([(symbol, (0., 0., 0.))], {symbol: basis[symbol]}, unit='Bohr')
    S, T, V = oracle.int1e(mol)
    h = T + V
    seig, U = np.linalg.eigh(S)
    X = U[:, seig > 1e-15] / np.sqrt(seig[seig > 1e-15])
    ne = mol.nelectron

    def density(F):
        e, c = np.linalg.eigh(X.T @ F @ X)
        c = X @ c
        occ = _aufbau_fractional(e, ne)
        return (c * occ) @ c.T

    dm = density(h)
    e_last = None
    focks, errs = [], []
    for _ in range(max_cycle):
        vj, vk = oracle.get_jk(mol, dm)
        F = h + vj - .5 * vk
        e = .5 * np.sum(dm * (h + F))
        if e_last is not None and abs(e - e_last) < conv_tol:
            break
        e_last = e
        focks.append(F)
        errs.append((F @ dm @ S - S @ dm @ F).ravel())
        focks, errs = focks[-8:], errs[-8:]
        n = len(focks)
        if n > 1:
            B = -np.ones((n + 1, n + 1))
            B[n, n] = 0
            E = np.array(errs)
            B[:n, :n] = E @ E.T
            rhs = np.zeros(n + 1)
            rhs[n] = -1
            c = np.linalg.solve(B, rhs)[:n]
            F = np.einsum('i,ijk->jk', c, np.array(focks))
        dm = density(F)
    _ATOM_CACHE[key] = dm
    return dm


def sad_guess(mol, S):
    nao = mol.nao
    dm = np.zeros((nao, nao))
    sl = mol.aoslice_by_atom()
    for ia, (sym, _) in enumerate(mol.atom):
        p0, p1 = sl[ia, 2], sl[ia, 3]
        dm[p0:p1, p0:p1] = atomic_density(sym, mol.basis)
    ne = float(np.sum(dm * S))
    if ne > 0:
        dm *= mol.nelectron / ne
    return dm


def eig(h, s):
    """cuobc/scf/hf.py:253-265 on the GPU (torch's cuSOLVER eigh), host in/out."""
    import torch
    s = torch.as_tensor(s, device='cuda')
    h = torch.as_tensor(h, device='cuda')
    seig, t = torch.linalg.eigh(s)
    inv = 1. / torch.sqrt(seig)
    inv[seig < 1e-15] = 0
    t = t * inv
    e, c = torch.linalg.eigh(t.T @ h @ t)
    return e.cpu().numpy(), (t @ c).cpu().numpy()


class RefSCF:
    """One restricted SCF along the reference's path (see the module doc).

    get_jk(dm_host) is the reference's get_jk; kernel() runs the host loop
    and returns the energy; timings holds the set-up and per-cycle seconds.
    """

    def __init__(self, mol, direct_scf_tol=1e-13, conv_tol=1e-8, max_cycle=60, diis_space=8):
        self.mol = mol
        self.direct_scf_tol = direct_scf_tol
        self.conv_tol = conv_tol
        self.max_cycle = max_cycle
        self.diis_space = diis_space
        self.timings = {}
        self.opt = None
        self.jk = None

    def build(self):
        t0 = time.perf_counter()
        self.opt = RefVHFOpt(self.mol).build(self.direct_scf_tol)
        self.jk = RefJK(self.opt)
        import torch
        self.coeff = torch.as_tensor(self.opt.coeff, device='cuda')
        self.timings['vhfopt'] = time.perf_counter() - t0
        return self

    def get_jk(self, dm):
        """cuobc/scf/hf.py:53-227 for one host density (nao0 x nao0)."""
        import torch
        C = self.coeff
        d = torch.as_tensor(np.asarray(dm), device='cuda')
        dmc = (C @ d @ C.T)[None].contiguous()
        J, K = self.jk.jk_cart(dmc, tol=self.direct_scf_tol)
        vj = (C.T @ J[0] @ C).cpu().numpy()
        vk = (C.T @ K[0] @ C).cpu().numpy()
        return vj, vk

    def kernel(self, dm0=None, cycle_hook=None):
        """Host SCF loop to |Delta E| < conv_tol.  cycle_hook(cycle, seconds)
        is called after every cycle.  Keeps the last difference density
        (last_ddm) and the matrices of the last cycle for repeat_cycle()."""
        t0 = time.perf_counter()
        if self.opt is None:
            self.build()
        mol = self.mol
        S, T, V = oracle.int1e(mol)
        h = T + V
        e_nuc = mol.energy_nuc()
        dm = sad_guess(mol, S) if dm0 is None else np.asarray(dm0)
        nocc = mol.nelectron // 2
        self.timings['setup'] = time.perf_counter() - t0
        focks, errs = [], []
        vhf = None
        dm_last = None
        e_last = None
        self.converged = False
        self.cycle_s = []
        for cycle in range(self.max_cycle):
            tc = time.perf_counter()
            if dm_last is None:
                vj, vk = self.get_jk(dm)
                vhf = vj - .5 * vk
                self.last_ddm = dm
            else:
                self.last_ddm = dm - dm_last
                vj, vk = self.get_jk(self.last_ddm)
                vhf = vhf + vj - .5 * vk
            F = h + vhf
            e = float(.5 * np.sum(dm * (h + F))) + e_nuc
            self.cycles = cycle + 1
            done = e_last is not None and abs(e - e_last) < self.conv_tol
            if not done:
                e_last = e
                focks.append(F)
                errs.append((F @ dm @ S - S @ dm @ F).ravel())
                focks, errs = focks[-self.diis_space:], errs[-self.diis_space:]
                n = len(focks)
                Fd = F
                if n > 1:
                    B = -np.ones((n + 1, n + 1))
                    B[n, n] = 0
                    E = np.array(errs)
                    B[:n, :n] = E @ E.T
                    rhs = np.zeros(n + 1)
                    rhs[n] = -1
                    c = np.linalg.solve(B, rhs)[:n]
                    Fd = np.einsum('i,ijk->jk', c, np.array(focks))
                mo_e, mo_c = eig(Fd, S)
                idx = np.argsort(mo_e)[:nocc]
                dm_last = dm
                dm = 2. * mo_c[:, idx] @ mo_c[:, idx].T
            self.cycle_s.append(time.perf_counter() - tc)
            if cycle_hook is not None:
                cycle_hook(cycle, self.cycle_s[-1])
            if done:
                self.converged = True
                break
        self.e_tot = e
        self.dm = dm
        self._last = (h, S, vhf, nocc)
        self.timings['total'] = time.perf_counter() - t0
        return e

    def repeat_cycle(self):
        """One more SCF cycle's work at the end point: the incremental J/K of
        the last difference density, the Fock matrix, the energy and the
        eigenproblem (the density is kept).  Returns the seconds taken."""
        t = time.perf_counter()
        h, S, vhf, nocc = self._last
        vj, vk = self.get_jk(self.last_ddm)
        F = h + vhf + vj - .5 * vk
        float(.5 * np.sum(self.dm * (h + F)))
        eig(F, S)
        return time.perf_counter() - t

    def close(self):
        if self.jk is not None:
            self.jk.close()
            self.jk = None
