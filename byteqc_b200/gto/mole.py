"""Molecule and basis container in the pyscf ``Mole`` layout.

The J/K engine is a drop-in behind cuobc's ``get_jk(mol, dm, ...)``
(cuobc/scf/hf.py:53-227), which reads a pyscf 2.5 ``Mole``: the integer tables
``_atm`` (natm x 6) and ``_bas`` (nbas x 8) and the float array ``_env``.
pyscf is not a dependency of this package, so this module provides a ``Mole``
with the same fields, slot numbers, normalisation and AO ordering:

* ``_atm`` slots: CHARGE_OF, PTR_COORD, NUC_MOD_OF, PTR_ZETA, PTR_FRAC_CHARGE,
  RESERVE (cuobc/lib/gint/gint.h:28-33);
* ``_bas`` slots: ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, KAPPA_OF, PTR_EXP,
  PTR_COEFF, RESERVE (gint.h:36-43);
* contraction coefficients in ``_env`` carry the radial normalisation of each
  primitive and of each contracted radial function, contraction-major
  (``coeff[ictr * nprim + iprim]``);
* Cartesian components are ordered x^a y^b z^c with a descending, then b
  descending; spherical components m = -l..l, except p which is (x, y, z);
* a Cartesian s or p function carries the factor 1/sqrt(4 pi) or
  sqrt(3/(4 pi)) (the constant ``CINTcommon_fac_sp`` of
  cuobc/lib/gint/pair_data.c:27-28); for l >= 2 that normalisation sits in
  the Cartesian-to-spherical matrix (real solid harmonics, no Condon-Shortley
  phase).
"""
import math

import numpy as np

# slots of _atm
CHARGE_OF, PTR_COORD, NUC_MOD_OF, PTR_ZETA, PTR_FRAC_CHARGE, ATM_SLOTS = 0, 1, 2, 3, 4, 6
# slots of _bas
ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, KAPPA_OF, PTR_EXP, PTR_COEFF, BAS_SLOTS = 0, 1, 2, 3, 4, 5, 6, 8
PTR_ENV_START = 20

BOHR = 0.52917721092  # Angstrom per Bohr

ELEMENTS = {'H': 1, 'He': 2, 'Li': 3, 'Be': 4, 'B': 5, 'C': 6, 'N': 7, 'O': 8, 'F': 9, 'Ne': 10}


def gaussian_int(n, alpha):
    """int_0^inf x^n exp(-alpha x^2) dx."""
    n1 = (n + 1) * .5
    return math.gamma(n1) / (2. * alpha ** n1)


def gto_norm(l, expnt):
    """Normalisation of the radial function r^l exp(-a r^2)."""
    expnt = np.asarray(expnt, dtype=float)
    return 1. / np.sqrt(np.array([gaussian_int(l * 2 + 2, 2 * a) for a in expnt.ravel()])
                        ).reshape(expnt.shape)


def normalize_shell(l, exps, cs):
    """Primitive and contracted radial normalisation (pyscf make_bas_env)."""
    exps = np.asarray(exps, dtype=float)
    cs = np.asarray(cs, dtype=float).reshape(len(exps), -1)
    cs = cs * gto_norm(l, exps)[:, None]
    ee = exps[:, None] + exps[None, :]
    ee = np.vectorize(lambda a: gaussian_int(l * 2 + 2, a))(ee)
    s1 = 1. / np.sqrt(np.einsum('pi,pq,qi->i', cs, ee, cs))
    return cs * s1


def ncart(l):
    return (l + 1) * (l + 2) // 2


def nsph(l):
    return 2 * l + 1


def cart_powers(l):
    """Cartesian exponents (a, b, c) of x^a y^b z^c in the AO order."""
    out = []
    for a in range(l, -1, -1):
        for b in range(l - a, -1, -1):
            out.append((a, b, l - a - b))
    return out


def common_fac_sp(l):
    if l == 0:
        return 0.282094791773878143
    if l == 1:
        return 0.488602511902919921
    return 1.


def _poly_mul(p, q):
    out = {}
    for ka, va in p.items():
        for kb, vb in q.items():
            k = (ka[0] + kb[0], ka[1] + kb[1], ka[2] + kb[2])
            out[k] = out.get(k, 0) + va * vb
    return out


def _real_solid_harmonic(l, m):
    """Coefficients of r^l Y_lm (real, normalised over the sphere, no
    Condon-Shortley phase) over the monomials x^a y^b z^c.

    Uses r^l P_l^|m|(cos t) e^{i|m|p} = (x + i y)^|m| r^(l-|m|) P_l^(|m|)(z/r),
    with P_l^(|m|) the |m|-th derivative of the Legendre polynomial.
    """
    am = abs(m)
    # Legendre P_l(u) = sum_k (-1)^k (2l-2k)! / (2^l k! (l-k)! (l-2k)!) u^(l-2k)
    leg = {}
    for k in range(l // 2 + 1):
        leg[l - 2 * k] = (-1) ** k * math.factorial(2 * l - 2 * k) / (
            2 ** l * math.factorial(k) * math.factorial(l - k) * math.factorial(l - 2 * k))
    # |m|-th derivative
    der = {}
    for p, c in leg.items():
        if p >= am:
            der[p - am] = der.get(p - am, 0) + c * math.factorial(p) / math.factorial(p - am)
    # r^(l-|m|) * sum_p d_p (z/r)^p = sum_p d_p z^p (r^2)^((l-|m|-p)/2)
    r2 = {(2, 0, 0): 1., (0, 2, 0): 1., (0, 0, 2): 1.}
    zpart = {}
    for p, c in der.items():
        e = l - am - p
        assert e % 2 == 0
        term = {(0, 0, p): c}
        for _ in range(e // 2):
            term = _poly_mul(term, r2)
        for k, v in term.items():
            zpart[k] = zpart.get(k, 0) + v
    # (x + i y)^|m| split into real and imaginary parts
    re_part, im_part = {}, {}
    for k in range(am + 1):
        c = math.comb(am, k)
        # i^k
        ik = [(1, 0), (0, 1), (-1, 0), (0, -1)][k % 4]
        key = (am - k, k, 0)
        if ik[0]:
            re_part[key] = re_part.get(key, 0) + c * ik[0]
        if ik[1]:
            im_part[key] = im_part.get(key, 0) + c * ik[1]
    ang = re_part if m >= 0 else im_part
    poly = _poly_mul(ang, zpart)
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    if m != 0:
        norm *= math.sqrt(2.)
    return {k: v * norm for k, v in poly.items() if abs(v) > 0}


_C2S_CACHE = {}


def cart2sph(l):
    """(ncart(l), nsph(l)) matrix: spherical AO = cart AOs @ column.

    For l <= 1 it is the identity (the Cartesian s/p functions already carry
    the spherical normalisation); for l >= 2 it holds the real solid harmonic
    coefficients.
    """
    if l in _C2S_CACHE:
        return _C2S_CACHE[l]
    if l < 2:
        c = np.eye(ncart(l))
    else:
        powers = cart_powers(l)
        c = np.zeros((ncart(l), nsph(l)))
        for im, m in enumerate(range(-l, l + 1)):
            poly = _real_solid_harmonic(l, m)
            for k, v in poly.items():
                c[powers.index(k), im] = v
    _C2S_CACHE[l] = c
    return c


class Mole:
    """Minimal pyscf-layout molecule: atoms, basis, charge, spin.

    ``atom`` is a list of (symbol, (x, y, z)) in ``unit`` (Angstrom or Bohr);
    ``basis`` maps element symbols to pyscf internal basis lists
    ``[[l, [exp, c_1, ..., c_nctr], ...], ...]``.
    """

    def __init__(self, atom, basis, unit='Angstrom', charge=0, spin=0, cart=False,
                 verbose=0):
        self.atom = [(s, tuple(float(v) for v in xyz)) for s, xyz in atom]
        self.basis = basis
        self.unit = unit
        self.charge = charge
        self.spin = spin
        self.cart = cart
        self.verbose = verbose
        self.build()

    def build(self):
        scale = 1. / BOHR if self.unit.lower().startswith('a') else 1.
        env = [0.] * PTR_ENV_START
        atm = []
        bas = []
        basis_ptrs = {}
        for ia, (sym, xyz) in enumerate(self.atom):
            ptr = len(env)
            env.extend([xyz[0] * scale, xyz[1] * scale, xyz[2] * scale, 0.])
            atm.append([ELEMENTS[sym], ptr, 1, ptr + 3, 0, 0])
        for ia, (sym, xyz) in enumerate(self.atom):
            if sym not in basis_ptrs:
                shells = []
                for shell in self.basis[sym]:
                    l = shell[0]
                    prims = np.asarray(shell[1:], dtype=float)
                    exps = prims[:, 0]
                    cs = normalize_shell(l, exps, prims[:, 1:])
                    pexp = len(env)
                    env.extend(exps.tolist())
                    pcoeff = len(env)
                    env.extend(cs.T.ravel().tolist())
                    shells.append((l, len(exps), cs.shape[1], pexp, pcoeff))
                basis_ptrs[sym] = shells
            for (l, nprim, nctr, pexp, pcoeff) in basis_ptrs[sym]:
                bas.append([ia, l, nprim, nctr, 0, pexp, pcoeff, 0])
        self._atm = np.asarray(atm, dtype=np.int32).reshape(-1, ATM_SLOTS)
        self._bas = np.asarray(bas, dtype=np.int32).reshape(-1, BAS_SLOTS)
        self._env = np.asarray(env, dtype=np.float64)
        return self

    # ---- pyscf-style accessors -------------------------------------------------
    @property
    def natm(self):
        return len(self._atm)

    @property
    def nbas(self):
        return len(self._bas)

    def atom_charges(self):
        return self._atm[:, CHARGE_OF].copy()

    def atom_coords(self):
        ptr = self._atm[:, PTR_COORD]
        return np.stack([self._env[ptr], self._env[ptr + 1], self._env[ptr + 2]], axis=1)

    @property
    def nelectron(self):
        return int(self.atom_charges().sum()) - self.charge

    @property
    def nelec(self):
        ne = self.nelectron
        na = (ne + self.spin) // 2
        return na, ne - na

    def bas_angular(self, i):
        return int(self._bas[i, ANG_OF])

    def bas_nprim(self, i):
        return int(self._bas[i, NPRIM_OF])

    def bas_nctr(self, i):
        return int(self._bas[i, NCTR_OF])

    def bas_atom(self, i):
        return int(self._bas[i, ATOM_OF])

    def bas_exp(self, i):
        p = self._bas[i, PTR_EXP]
        return self._env[p:p + self._bas[i, NPRIM_OF]].copy()

    def bas_ctr_coeff(self, i):
        """(nprim, nctr) normalised contraction coefficients."""
        nprim, nctr = self._bas[i, NPRIM_OF], self._bas[i, NCTR_OF]
        p = self._bas[i, PTR_COEFF]
        return self._env[p:p + nprim * nctr].reshape(nctr, nprim).T.copy()

    def ao_loc_nr(self, cart=None):
        cart = self.cart if cart is None else cart
        l = self._bas[:, ANG_OF]
        nctr = self._bas[:, NCTR_OF]
        dims = ((l + 1) * (l + 2) // 2 if cart else 2 * l + 1) * nctr
        return np.append(0, np.cumsum(dims)).astype(np.int32)

    @property
    def ao_loc(self):
        return self.ao_loc_nr()

    def nao_nr(self, cart=None):
        return int(self.ao_loc_nr(cart)[-1])

    @property
    def nao(self):
        return self.nao_nr()

    def nao_cart(self):
        return self.nao_nr(cart=True)

    def aoslice_by_atom(self):
        """(natm, 4): shell start, shell end, AO start, AO end per atom."""
        ao_loc = self.ao_loc_nr()
        out = np.zeros((self.natm, 4), dtype=int)
        atoms = self._bas[:, ATOM_OF]
        for ia in range(self.natm):
            idx = np.where(atoms == ia)[0]
            if len(idx):
                out[ia] = [idx[0], idx[-1] + 1, ao_loc[idx[0]], ao_loc[idx[-1] + 1]]
            elif ia > 0:
                out[ia] = [out[ia - 1, 1]] * 2 + [out[ia - 1, 3]] * 2
        return out

    def cart2sph_coeff(self):
        """(nao_cart, nao_sph) block-diagonal transformation."""
        blocks = []
        for i in range(self.nbas):
            l = self.bas_angular(i)
            for _ in range(self.bas_nctr(i)):
                blocks.append(cart2sph(l))
        nc = sum(b.shape[0] for b in blocks)
        ns = sum(b.shape[1] for b in blocks)
        c = np.zeros((nc, ns))
        r0 = c0 = 0
        for b in blocks:
            c[r0:r0 + b.shape[0], c0:c0 + b.shape[1]] = b
            r0 += b.shape[0]
            c0 += b.shape[1]
        return c

    def energy_nuc(self):
        z = self.atom_charges().astype(float)
        r = self.atom_coords()
        e = 0.
        for i in range(self.natm):
            for j in range(i):
                e += z[i] * z[j] / np.linalg.norm(r[i] - r[j])
        return e

    def copy(self):
        import copy
        m = copy.copy(self)
        m._atm = self._atm.copy()
        m._bas = self._bas.copy()
        m._env = self._env.copy()
        return m


M = Mole
