"""Synthetic basis sets shaped like cc-pVDZ, cc-pVTZ and 6-31G**.

The workloads this engine is measured on name cc-pVDZ, cc-pVTZ and 6-31G**.
Those basis-set files normally ship inside pyscf, which is not installed here,
and their numbers are published data that this project does not retype.  This
module therefore builds *synthetic* basis sets with the same shell structure:
per element the same list of (l, number of primitives, number of contractions),
hence the same AO counts (H2O: 24 AO in the DZ shape, 58 in the TZ shape; CH2
unit of an alkane 14 + 2 x 5 AO in the 6-31G** shape) and the same integral
classes (s-d for DZ, s-f for TZ).  The numbers are generated, not copied:

* primitive exponents form even-tempered sequences a_k = a_max * r^-k whose
  range and ratio per element and angular momentum are chosen here;
* contraction coefficients are least-squares fits of the primitives to a
  Slater-type radial function r^(n-1) exp(-zeta r) with zeta from Slater's
  rules (the STO-nG fitting procedure of Hehre, Stewart and Pople,
  J. Chem. Phys. 51 (1969) 2657, done numerically here).

Energies computed with these sets are not comparable with literature values
for the real basis sets; integral classes, shapes, screening statistics and
costs are.
"""
import functools
import math

import numpy as np

from .mole import gaussian_int, gto_norm

# Slater exponents (Slater's rules) for the 1s and the valence shell
_SLATER = {
    'H': {'1s': 1.24, 'val': 1.24},
    'C': {'1s': 5.67, 'val': 1.625},
    'N': {'1s': 6.67, 'val': 1.95},
    'O': {'1s': 7.66, 'val': 2.275},
}


def _even_tempered(amax, ratio, n):
    return [amax / ratio ** k for k in range(n)]


def _gto_sto_overlap(l, a, n, zeta):
    """<r^l e^{-a r^2} | r^(n-1) e^{-zeta r}> over r^2 dr, numerically."""
    from scipy.integrate import quad
    f = lambda r: r ** (l + n + 1) * math.exp(-a * r * r - zeta * r)
    v, _ = quad(f, 0, np.inf, limit=400, epsabs=0, epsrel=1e-13)
    return v


@functools.lru_cache(maxsize=None)
def _fit(l, exps, n, zeta):
    """Coefficients, over normalised primitives (the pyscf basis-file
    convention), of the least-squares fit to the radial Slater function
    r^(n-1) e^{-zeta r}."""
    exps = np.asarray(exps)
    S = np.array([[gaussian_int(2 * l + 2, ai + aj) for aj in exps] for ai in exps])
    b = np.array([_gto_sto_overlap(l, a, n, zeta) for a in exps])
    c = np.linalg.solve(S, b)
    return c / gto_norm(l, exps)


def _shell(l, exps, cols):
    """pyscf internal shell entry [l, [e, c1, c2...], ...]."""
    return [l] + [[e] + [col[k] for col in cols] for k, e in enumerate(exps)]


def _heavy(sym, kind):
    z1 = _SLATER[sym]['1s']
    zv = _SLATER[sym]['val']
    Z = {'C': 6, 'N': 7, 'O': 8}[sym]
    shells = []
    if kind in ('dz', 'tz'):
        # generally contracted s block: 8 primitives, 2 contractions (1s, 2s)
        amax = 180. * Z * Z
        sexp = tuple(_even_tempered(amax, 3.6, 8))
        c1 = _fit(0, sexp, 1, z1)
        c2 = _fit(0, sexp, 2, zv)
        shells.append(_shell(0, sexp, [c1, c2]))
        if kind == 'dz':
            shells.append([0, [0.045 * Z, 1.]])
        else:
            shells.append([0, [0.30 * Z / 8 * 5.5, 1.]])
            shells.append([0, [0.030 * Z, 1.]])
        pexp = tuple(_even_tempered(2.2 * Z, 4.0, 3))
        cp = _fit(1, pexp, 2, zv)
        shells.append(_shell(1, pexp, [cp]))
        if kind == 'dz':
            shells.append([1, [0.034 * Z, 1.]])
            shells.append([2, [0.15 * Z, 1.]])
        else:
            shells.append([1, [0.10 * Z, 1.]])
            shells.append([1, [0.027 * Z, 1.]])
            shells.append([2, [0.33 * Z, 1.]])
            shells.append([2, [0.10 * Z, 1.]])
            shells.append([3, [0.18 * Z, 1.]])
    else:  # 6-31G** shape
        core = tuple(_even_tempered(500. * Z * Z / 8, 3.3, 6))
        shells.append(_shell(0, core, [_fit(0, core, 1, z1)]))
        val = tuple(_even_tempered(0.9 * Z, 3.5, 3))
        shells.append(_shell(0, val, [_fit(0, val, 2, zv)]))
        shells.append(_shell(1, val, [_fit(1, val, 2, zv)]))
        shells.append([0, [0.03 * Z, 1.]])
        shells.append([1, [0.03 * Z, 1.]])
        shells.append([2, [0.8, 1.]])
    return shells


def _hydrogen(kind):
    zh = _SLATER['H']['1s']
    sexp = tuple(_even_tempered(16.0, 6.0, 3))
    shells = [_shell(0, sexp, [_fit(0, sexp, 1, zh)])]
    if kind == 'dz':
        shells.append([0, [0.13, 1.]])
        shells.append([1, [0.75, 1.]])
    elif kind == 'tz':
        shells.append([0, [0.32, 1.]])
        shells.append([0, [0.10, 1.]])
        shells.append([1, [1.30, 1.]])
        shells.append([1, [0.40, 1.]])
        shells.append([2, [1.00, 1.]])
    else:
        shells.append([0, [0.16, 1.]])
        shells.append([1, [1.10, 1.]])
    return shells


_KINDS = {'cc-pvdz': 'dz', 'cc-pvtz': 'tz', '6-31g**': 'pople'}


def synthetic_basis(name, elements):
    """Basis dict {symbol: shells} for a named shape.

    ``name`` is one of 'cc-pvdz', 'cc-pvtz', '6-31g**' (case-insensitive); the
    result has that basis set's shell structure with synthetic numbers.
    """
    kind = _KINDS[name.lower()]
    out = {}
    for sym in elements:
        out[sym] = _hydrogen(kind) if sym == 'H' else _heavy(sym, kind)
    return out


def sto3g_like(elements):
    """A small contracted s/p basis (3 primitives per shell) for quick tests."""
    out = {}
    for sym in elements:
        if sym == 'H':
            e = tuple(_even_tempered(3.4, 5.0, 3))
            out[sym] = [_shell(0, e, [_fit(0, e, 1, 1.24)])]
        else:
            Z = {'C': 6, 'N': 7, 'O': 8}[sym]
            z1, zv = _SLATER[sym]['1s'], _SLATER[sym]['val']
            e1 = tuple(_even_tempered(2.3 * z1 * z1, 5.0, 3))
            ev = tuple(_even_tempered(2.3 * zv * zv * 0.5, 4.5, 3))
            out[sym] = [_shell(0, e1, [_fit(0, e1, 1, z1)]),
                        _shell(0, ev, [_fit(0, ev, 2, zv)]),
                        _shell(1, ev, [_fit(1, ev, 2, zv)])]
    return out


def synthetic_aux_basis(elements):
    """A synthetic auxiliary (density-fitting) basis: uncontracted
    even-tempered shells per element, s-f on heavy atoms and s-d on H, the
    kind of shell structure JK-fitting sets have.  Generated here, not
    copied from any published set; for the 3-centre integral engine and its
    tests only."""
    out = {}
    for sym in elements:
        if sym == 'H':
            spec = [(0, 12., 3.5, 4), (1, 2.0, 3.0, 2), (2, 1.2, 1., 1)]
        else:
            Z = {'C': 6, 'N': 7, 'O': 8}[sym]
            spec = [(0, 60. * Z, 3.2, 7), (1, 8. * Z, 3.0, 4), (2, 2.5 * Z, 2.8, 3),
                    (3, 0.6 * Z, 2.5, 2)]
        shells = []
        for l, amax, ratio, n in spec:
            for e in _even_tempered(amax, ratio, n):
                shells.append([l, [e, 1.]])
        out[sym] = shells
    return out
