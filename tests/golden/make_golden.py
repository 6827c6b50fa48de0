"""Generate the golden vectors that pin the CPU oracle (run once; committed).

* rys_mpmath.json: Rys nodes and weights for n = 1..7 at a spread of x, from
  60-digit mpmath (Boys moments 1F1, Chebyshev algorithm, Golub-Welsch).
* eri_mpmath.json: primitive Cartesian ERIs (ij|kl) of single-primitive
  shells on four random centres, for classes up to (dd|ss) / (pp|pp) /
  (ds|ds), from the closed form of (ss|ss) (Boys F0 via erf at 40 digits) and
  its derivatives with respect to the centres
  (x_A e^{-a r_A^2} = (1/2a) d/dA_x e^{-a r_A^2}).

Usage: python tests/golden/make_golden.py
"""
import json
import os
import sys

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from byteqc_b200.rys.gen_rys_tables import rys_exact  # noqa: E402


def cart_powers(l):
    out = []
    for a in range(l, -1, -1):
        for b in range(l - a, -1, -1):
            out.append((a, b, l - a - b))
    return out


def ssss(a, A, b, B, c, C, d, D):
    p = a + b
    q = c + d
    P = [(a * A[i] + b * B[i]) / p for i in range(3)]
    Q = [(c * C[i] + d * D[i]) / q for i in range(3)]
    AB2 = sum((A[i] - B[i]) ** 2 for i in range(3))
    CD2 = sum((C[i] - D[i]) ** 2 for i in range(3))
    PQ2 = sum((P[i] - Q[i]) ** 2 for i in range(3))
    x = p * q / (p + q) * PQ2
    F0 = mp.sqrt(mp.pi / x) / 2 * mp.erf(mp.sqrt(x)) if x > 0 else mp.mpf(1)
    return 2 * mp.pi ** mp.mpf(2.5) / (p * q * mp.sqrt(p + q)) * mp.exp(-a * b / p * AB2 - c * d / q * CD2) * F0


def eri_prim(exps, cents, pows):
    """(ij|kl) of unnormalised primitives x^a y^b z^c e^{-alpha r^2}."""
    def f(*v):
        cs = [[v[3 * i], v[3 * i + 1], v[3 * i + 2]] for i in range(4)]
        return ssss(exps[0], cs[0], exps[1], cs[1], exps[2], cs[2], exps[3], cs[3])
    x0 = [c for C in cents for c in C]
    terms = [(mp.mpf(1), [0] * 12)]
    for i, pw in enumerate(pows):
        for d, n in enumerate(pw):
            a = exps[i]
            new = []
            for coef, o in terms:
                if n == 0:
                    new.append((coef, o))
                elif n == 1:
                    o2 = o[:]
                    o2[3 * i + d] += 1
                    new.append((coef / (2 * a), o2))
                else:
                    o2 = o[:]
                    o2[3 * i + d] += 2
                    new.append((coef / (2 * a) ** 2, o2))
                    new.append((coef / (2 * a), o))
            terms = new
    tot = 0
    for coef, o in terms:
        tot += coef * (mp.diff(f, x0, tuple(o)) if any(o) else f(*x0))
    return tot


def main():
    mp.mp.dps = 60
    xs = [0.0, 1e-6, 0.05, 0.7, 2.3, 6.1, 13.7, 29.9, 44.4, 68.2, 74.9, 75.0, 90.0, 500.0]
    rys = []
    for n in range(1, 8):
        for x in xs:
            r, w = rys_exact(n, x)
            rys.append({'n': n, 'x': x, 'r': [float(v) for v in r], 'w': [float(v) for v in w]})
    with open(os.path.join(HERE, 'rys_mpmath.json'), 'w') as f:
        json.dump(rys, f)

    mp.mp.dps = 40
    rng = np.random.default_rng(5)
    exps = [1.3, 0.7, 2.1, 0.45]
    cents = [[float(v) for v in rng.normal(size=3) * 0.8] for _ in range(4)]
    eris = []
    for ls in [(0, 0, 0, 0), (1, 0, 0, 0), (1, 1, 0, 0), (1, 0, 1, 0), (2, 0, 0, 0), (1, 1, 1, 0),
               (2, 1, 0, 0), (1, 1, 1, 1), (2, 0, 2, 0)]:
        comps = []
        pw = [cart_powers(l) for l in ls]
        n = 0
        for fi in range(len(pw[0])):
            for fj in range(len(pw[1])):
                for fk in range(len(pw[2])):
                    for fl in range(len(pw[3])):
                        if n >= 6:
                            break
                        v = eri_prim([mp.mpf(e) for e in exps], [[mp.mpf(c) for c in C] for C in cents],
                                     [pw[0][fi], pw[1][fj], pw[2][fk], pw[3][fl]])
                        comps.append({'f': [fi, fj, fk, fl], 'value': float(v)})
                        n += 1
        eris.append({'ls': ls, 'comps': comps})
    with open(os.path.join(HERE, 'eri_mpmath.json'), 'w') as f:
        json.dump({'exps': exps, 'centres_bohr': cents, 'classes': eris}, f, indent=0)


if __name__ == '__main__':
    main()
