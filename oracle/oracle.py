"""ctypes front end of the CPU FP64 oracle (test infrastructure only).

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module; the engine never does.  It wraps ``libjk_oracle.so`` (built from
``jk_oracle.c`` by ``make -C oracle``) and adds the numpy pieces of the
reference's get_jk that sit around the integral loop:

* the AO transform D' = C D C^T into the Cartesian basis and J = C^T J' C back
  (cuobc/scf/hf.py:67-74, 171-181), here with C the Cartesian-to-spherical
  matrix of the basis as given;
* a restricted Hartree-Fock loop (core guess, DIIS on FDS - SDF, canonical
  orthogonalisation as in cuobc/scf/hf.py:253-265) used to pin SCF energies.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, 'libjk_oracle.so')

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            subprocess.check_call(['make', '-s', '-C', HERE])
        _lib = ctypes.CDLL(LIBPATH)
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _basis_args(mol):
    atm = np.ascontiguousarray(mol._atm, dtype=np.int32)
    bas = np.ascontiguousarray(mol._bas, dtype=np.int32)
    env = np.ascontiguousarray(mol._env, dtype=np.float64)
    return atm, bas, env


def rys(n, x):
    lib = load()
    r = np.zeros(n)
    w = np.zeros(n)
    err = lib.oracle_rys(ctypes.c_int(n), ctypes.c_double(x), _ptr(r), _ptr(w))
    if err:
        raise RuntimeError('oracle_rys failed')
    return r, w


def eri_shells(mol, ish, jsh, ksh, lsh):
    """Cartesian block (ij|kl) over the AOs of four shells."""
    lib = load()
    atm, bas, env = _basis_args(mol)
    dims = []
    for s in (ish, jsh, ksh, lsh):
        l = mol.bas_angular(s)
        dims.append((l + 1) * (l + 2) // 2 * mol.bas_nctr(s))
    out = np.zeros(dims)
    lib.oracle_eri_shells(_ptr(atm), ctypes.c_int(mol.natm), _ptr(bas), ctypes.c_int(mol.nbas),
                          _ptr(env), ctypes.c_int(ish), ctypes.c_int(jsh), ctypes.c_int(ksh),
                          ctypes.c_int(lsh), _ptr(out))
    return out


def eri_full_cart(mol):
    """Full (ij|kl) tensor over Cartesian AOs (small molecules only)."""
    ao_loc = mol.ao_loc_nr(cart=True)
    n = ao_loc[-1]
    out = np.zeros((n, n, n, n))
    for i in range(mol.nbas):
        for j in range(mol.nbas):
            for k in range(mol.nbas):
                for l in range(mol.nbas):
                    out[ao_loc[i]:ao_loc[i + 1], ao_loc[j]:ao_loc[j + 1],
                        ao_loc[k]:ao_loc[k + 1], ao_loc[l]:ao_loc[l + 1]] = \
                        eri_shells(mol, i, j, k, l)
    return out


def jk_cart(mol, dm_cart, nthreads=0):
    """J and K over Cartesian AOs of the basis as given."""
    lib = load()
    atm, bas, env = _basis_args(mol)
    dm = np.ascontiguousarray(dm_cart, dtype=np.float64)
    shape = dm.shape
    dm = dm.reshape(-1, shape[-1], shape[-1])
    vj = np.zeros_like(dm)
    vk = np.zeros_like(dm)
    err = lib.oracle_jk(_ptr(atm), ctypes.c_int(mol.natm), _ptr(bas), ctypes.c_int(mol.nbas),
                        _ptr(env), _ptr(dm), ctypes.c_int(dm.shape[0]), _ptr(vj), _ptr(vk),
                        ctypes.c_int(nthreads))
    if err:
        raise RuntimeError('oracle_jk failed')
    return vj.reshape(shape), vk.reshape(shape)


def c2s(mol):
    """Cartesian-to-AO matrix (identity for a Cartesian molecule)."""
    if mol.cart:
        return np.eye(mol.nao_nr(cart=True))
    return mol.cart2sph_coeff()


def get_jk(mol, dm, nthreads=0):
    """J, K in the molecule's AO basis for a symmetric density (n_dm, nao, nao)."""
    C = c2s(mol)
    dm = np.asarray(dm, dtype=np.float64)
    shape = dm.shape
    dms = dm.reshape(-1, shape[-1], shape[-1])
    dmc = np.einsum('pi,nij,qj->npq', C, dms, C)
    vj, vk = jk_cart(mol, dmc, nthreads)
    vj = np.einsum('pi,npq,qj->nij', C, vj, C)
    vk = np.einsum('pi,npq,qj->nij', C, vk, C)
    return vj.reshape(shape), vk.reshape(shape)


def q_cond(mol):
    lib = load()
    atm, bas, env = _basis_args(mol)
    q = np.zeros((mol.nbas, mol.nbas))
    lib.oracle_q_cond(_ptr(atm), ctypes.c_int(mol.natm), _ptr(bas), ctypes.c_int(mol.nbas),
                      _ptr(env), _ptr(q))
    return q


def int1e(mol):
    """Overlap, kinetic and nuclear-attraction matrices in the AO basis."""
    lib = load()
    atm, bas, env = _basis_args(mol)
    n = mol.nao_nr(cart=True)
    S = np.zeros((n, n))
    T = np.zeros((n, n))
    V = np.zeros((n, n))
    lib.oracle_int1e(_ptr(atm), ctypes.c_int(mol.natm), _ptr(bas), ctypes.c_int(mol.nbas),
                     _ptr(env), _ptr(S), _ptr(T), _ptr(V))
    C = c2s(mol)
    return C.T @ S @ C, C.T @ T @ C, C.T @ V @ C


def rhf(mol, conv_tol=1e-10, max_cycle=100, dm0=None, nthreads=0):
    """Restricted HF with DIIS.  Returns (energy, density, n_iterations)."""
    S, T, V = int1e(mol)
    h = T + V
    e_nuc = mol.energy_nuc()
    seig, U = np.linalg.eigh(S)
    keep = seig > 1e-15
    X = U[:, keep] / np.sqrt(seig[keep])
    nocc = mol.nelectron // 2

    def new_dm(F):
        e, c = np.linalg.eigh(X.T @ F @ X)
        c = X @ c
        return 2 * c[:, :nocc] @ c[:, :nocc].T

    dm = new_dm(h) if dm0 is None else dm0
    e_last = 0.
    focks, errs = [], []
    for it in range(max_cycle):
        vj, vk = get_jk(mol, dm, nthreads)
        F = h + vj - .5 * vk
        e = .5 * np.sum(dm * (h + F)) + e_nuc
        err = F @ dm @ S - S @ dm @ F
        focks.append(F)
        errs.append(X.T @ err @ X)
        focks, errs = focks[-8:], errs[-8:]
        if abs(e - e_last) < conv_tol and it > 0:
            return e, dm, it + 1
        e_last = e
        nd = len(focks)
        B = -np.ones((nd + 1, nd + 1))
        B[nd, nd] = 0
        for a in range(nd):
            for b in range(nd):
                B[a, b] = np.sum(errs[a] * errs[b])
        rhs = np.zeros(nd + 1)
        rhs[nd] = -1
        c = np.linalg.solve(B, rhs)[:nd]
        Fd = sum(ci * fi for ci, fi in zip(c, focks))
        dm = new_dm(Fd)
    raise RuntimeError('oracle RHF did not converge')


def uhf(mol, conv_tol=1e-10, max_cycle=200, dm0=None, nthreads=0):
    """Unrestricted HF with DIIS on the stacked alpha/beta commutators.
    Returns (energy, (dm_alpha, dm_beta), n_iterations).  dm0: initial
    (2, nao, nao) densities (default: core-Hamiltonian orbitals filled with
    nalpha / nbeta electrons).  The potentials follow pyscf's UHF:
    F_s = h + J(dm_a + dm_b) - K(dm_s)."""
    S, T, V = int1e(mol)
    h = T + V
    e_nuc = mol.energy_nuc()
    seig, U = np.linalg.eigh(S)
    keep = seig > 1e-15
    X = U[:, keep] / np.sqrt(seig[keep])
    na, nb = mol.nelec

    def new_dm(F, n):
        e, c = np.linalg.eigh(X.T @ F @ X)
        c = X @ c
        return c[:, :n] @ c[:, :n].T

    if dm0 is None:
        dm = np.stack([new_dm(h, na), new_dm(h, nb)])
    else:
        dm = np.asarray(dm0, dtype=np.float64)
    e_last = 0.
    focks, errs = [], []
    for it in range(max_cycle):
        vj, vk = get_jk(mol, dm, nthreads)
        F = np.stack([h + vj[0] + vj[1] - vk[s] for s in range(2)])
        e = .5 * sum(np.sum(dm[s] * (h + F[s])) for s in range(2)) + e_nuc
        if abs(e - e_last) < conv_tol and it > 0:
            return e, dm, it + 1
        e_last = e
        err = np.concatenate([(X.T @ (F[s] @ dm[s] @ S - S @ dm[s] @ F[s]) @ X).ravel()
                              for s in range(2)])
        focks.append(F)
        errs.append(err)
        focks, errs = focks[-8:], errs[-8:]
        nd = len(focks)
        B = -np.ones((nd + 1, nd + 1))
        B[nd, nd] = 0
        E = np.array(errs)
        B[:nd, :nd] = E @ E.T
        rhs = np.zeros(nd + 1)
        rhs[nd] = -1
        c = np.linalg.solve(B, rhs)[:nd]
        Fd = sum(ci * fi for ci, fi in zip(c, focks))
        dm = np.stack([new_dm(Fd[0], na), new_dm(Fd[1], nb)])
    raise RuntimeError('oracle UHF did not converge')
