"""Generate the Rys quadrature tables used by the CUDA kernels.

The Rys quadrature of order n for the Boys function

    F_m(x) = int_0^1 t^(2m) exp(-x t^2) dt,   m = 0 .. 2n-1

has nodes s_i = t_i^2 in (0, 1) and weights w_i with sum_i w_i s_i^m = F_m(x).
The kernels need (s_i, w_i) for x >= 0 and n = 1 .. NMAX (n = L/2 + 1 for a
shell quartet of total angular momentum L; s-f quartets need n <= 7).

The reference evaluates the same quantities from libcint-derived fitted tables
(cuobc/lib/gint/rys_roots.cu:1214-2176, rys_xw.cuh, roots_for_x0.cuh).  Those
tables are not used here.  This script derives its own from the mathematics:

* exact values at a sample point come from mpmath at 60 digits: the moments
  F_m(x) = 1F1(m+1/2; m+3/2; -x)/(2m+1), Gautschi's Chebyshev algorithm for the
  three-term recurrence of the orthogonal polynomials of the weight
  exp(-x s)/(2 sqrt(s)) on [0, 1], and the Golub-Welsch eigenproblem of the
  Jacobi matrix (Golub & Welsch, Math. Comp. 23 (1969) 221);
* for 0 <= x < XMAX[n] the range is cut into unit intervals and every node and
  weight is interpolated at the 12 Chebyshev points of each interval
  (degree-11 Chebyshev series, evaluated with Clenshaw's recurrence);
* for x >= XMAX[n] the quadrature is the half-range Gauss-Hermite rule:
  s_i = h_i^2 / x, w_i = W_i / sqrt(x), where h_i > 0 are the positive roots of
  the Hermite polynomial H_2n and W_i their Gauss-Hermite weights.  XMAX[n] is
  the first integer at which this limit agrees with the exact rule to 1e-15.

Output: ``byteqc_b200/csrc/rys_tables.inc`` (C source, included by the CUDA
library) and ``rys_tables_report.json`` (fit errors measured at off-node points).

Run:  python -m byteqc_b200.rys.gen_rys_tables   (about a minute on 8 cores)
"""
import json
import multiprocessing as mproc
import os
import sys

import mpmath as mp

NMAX = 7          # s-f shell quartets: L <= 12  ->  n <= 7
DEG = 11          # Chebyshev degree per unit interval
DPS = 60

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_INC = os.path.join(HERE, '..', 'csrc', 'rys_tables.inc')
OUT_REPORT = os.path.join(HERE, 'rys_tables_report.json')


def boys(m, x):
    mp.mp.dps = DPS
    x = mp.mpf(x)
    if x == 0:
        return mp.mpf(1) / (2 * m + 1)
    return mp.hyp1f1(m + mp.mpf(1) / 2, m + mp.mpf(3) / 2, -x) / (2 * m + 1)


def rys_exact(n, x):
    """Nodes s_i (ascending) and weights w_i of the order-n Rys rule at x."""
    mp.mp.dps = DPS
    mu = [boys(m, x) for m in range(2 * n)]
    alpha = [mp.mpf(0)] * n
    beta = [mp.mpf(0)] * n
    sig_prev = [mp.mpf(0)] * (2 * n)
    sig = mu[:]
    alpha[0] = mu[1] / mu[0]
    beta[0] = mu[0]
    for k in range(1, n):
        sig_new = [mp.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            sig_new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
        alpha[k] = sig_new[k + 1] / sig_new[k] - sig[k] / sig[k - 1]
        beta[k] = sig_new[k] / sig[k - 1]
        sig_prev, sig = sig, sig_new
    J = mp.zeros(n, n)
    for i in range(n):
        J[i, i] = alpha[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mp.sqrt(beta[i + 1])
    E, Q = mp.eigsy(J)
    idx = sorted(range(n), key=lambda i: E[i])
    return [E[i] for i in idx], [mu[0] * Q[0, i] ** 2 for i in idx]


def hermite_half(n):
    """Positive roots h_i (ascending) of H_2n and their Gauss-Hermite weights."""
    mp.mp.dps = DPS
    N = 2 * n
    coeffs = mp.taylor(lambda t: mp.hermite(N, t), 0, N)[::-1]
    roots = mp.polyroots(coeffs, maxsteps=400, extraprec=400)
    roots = sorted(mp.re(r) for r in roots if mp.re(r) > 0)
    out = []
    for h in roots:
        # Newton polish
        for _ in range(5):
            h = h - mp.hermite(N, h) / (2 * N * mp.hermite(N - 1, h))
        W = 2 ** (N - 1) * mp.factorial(N) * mp.sqrt(mp.pi) / (N ** 2 * mp.hermite(N - 1, h) ** 2)
        out.append((h, W))
    return out


def find_xmax(n, herm):
    mp.mp.dps = DPS
    x = 20
    while True:
        r, w = rys_exact(n, x)
        err = 0
        for i, (h, W) in enumerate(herm):
            err = max(err, abs(h * h / x / r[i] - 1), abs(W / mp.sqrt(x) / w[i] - 1))
        if err < 1e-15:
            return x
        x += 1


def _cheb_nodes():
    N = DEG + 1
    return [mp.cos(mp.pi * (k + mp.mpf(1) / 2) / N) for k in range(N)]


def fit_interval(args):
    n, a = args
    mp.mp.dps = DPS
    N = DEG + 1
    nodes = _cheb_nodes()
    vals = [rys_exact(n, a + mp.mpf(1) / 2 + t / 2) for t in nodes]
    funcs = [[v[0][i] for v in vals] for i in range(n)] + \
            [[v[1][i] for v in vals] for i in range(n)]
    coefs = []
    for f in funcs:
        c = [2 * mp.fsum(f[k] * mp.cos(mp.pi * j * (k + mp.mpf(1) / 2) / N)
                         for k in range(N)) / N for j in range(N)]
        c[0] /= 2
        coefs.append([float(v) for v in c])
    # measure the error of the double-precision Clenshaw sum off the nodes
    err = 0.0
    for t in (-0.93, -0.41, 0.05, 0.57, 0.96):
        r, w = rys_exact(n, a + mp.mpf(1) / 2 + mp.mpf(t) / 2)
        exact = r + w
        for q, c in enumerate(coefs):
            b1 = b2 = 0.0
            for cj in reversed(c[1:]):
                b1, b2 = 2 * t * b1 - b2 + cj, b1
            val = t * b1 - b2 + c[0]
            err = max(err, abs(val / float(exact[q]) - 1))
    return n, a, coefs, err


def main():
    herm = {n: hermite_half(n) for n in range(1, NMAX + 1)}
    xmax = {n: find_xmax(n, herm[n]) for n in range(1, NMAX + 1)}
    print('XMAX', xmax, file=sys.stderr)
    jobs = [(n, a) for n in range(1, NMAX + 1) for a in range(xmax[n])]
    with mproc.get_context('spawn').Pool(os.cpu_count()) as pool:
        results = pool.map(fit_interval, jobs, chunksize=4)
    table = {}
    errs = {}
    for n, a, coefs, err in results:
        table[(n, a)] = coefs
        errs[n] = max(errs.get(n, 0.0), err)
    print('max rel fit error per n', errs, file=sys.stderr)

    lines = []
    lines.append('// Generated by byteqc_b200/rys/gen_rys_tables.py; do not edit.')
    lines.append('// Rys nodes s=t^2 and weights: degree-%d Chebyshev series on unit' % DEG)
    lines.append('// intervals of x in [0, XMAX[n]); Gauss-Hermite limit beyond.')
    lines.append('// Two layouts of the same coefficients:')
    lines.append('// RYS_TABLE, interval-major: per (n, interval a) [coef k = 0..%d][q = 0..2n-1];' % DEG)
    lines.append('//   the functions of one x are contiguous (several lanes evaluating')
    lines.append('//   different functions of one x read one line).')
    lines.append('// RYS_TABLE_LM, level-major: per n [k][pair p = 0..n-1][a = 0..XMAX[n]-1][2]')
    lines.append('//   holding functions q = 2p, 2p+1 (lanes evaluating the same functions of')
    lines.append('//   different x read neighbouring addresses).')
    lines.append('// q < n: nodes s = t^2 in ascending order, q >= n: weights.')
    lines.append('#define RYS_NMAX %d' % NMAX)
    lines.append('#define RYS_NCOEF %d' % (DEG + 1))
    lines.append('// The including file defines RYS_CONST (storage of the big table) and')
    lines.append('// RYS_CONST_SMALL (storage of the small index tables).')
    lines.append('RYS_CONST_SMALL int RYS_XMAX[%d] = {0, %s};' % (
        NMAX + 1, ', '.join(str(xmax[n]) for n in range(1, NMAX + 1))))
    lines.append('// the same list for compile-time use (strides of the level-major layout)')
    lines.append('#define RYS_XMAX_LIST 0, %s' % ', '.join(str(xmax[n]) for n in range(1, NMAX + 1)))
    offs = [0]
    for n in range(1, NMAX + 1):
        offs.append(offs[-1] + xmax[n] * (DEG + 1) * 2 * n)
    lines.append('RYS_CONST_SMALL int RYS_TABLE_OFFSET[%d] = {0, %s};' % (
        NMAX + 2, ', '.join(str(o) for o in offs)))
    lines.append('#ifndef RYS_NO_BIG_TABLE')
    lines.append('RYS_CONST double RYS_TABLE[%d] = {' % offs[-1])
    for n in range(1, NMAX + 1):
        for a in range(xmax[n]):
            coefs = table[(n, a)]
            vals = []
            for k in range(DEG + 1):
                for q in range(2 * n):
                    vals.append('%.17g' % coefs[q][k])
            lines.append('  ' + ', '.join(vals) + ',')
    lines.append('};')
    lines.append('RYS_CONST double RYS_TABLE_LM[%d] = {' % offs[-1])
    for n in range(1, NMAX + 1):
        for k in range(DEG + 1):
            for p in range(n):
                vals = []
                for a in range(xmax[n]):
                    coefs = table[(n, a)]
                    vals.append('%.17g' % coefs[2 * p][k])
                    vals.append('%.17g' % coefs[2 * p + 1][k])
                lines.append('  ' + ', '.join(vals) + ',')
    lines.append('};')
    lines.append('#endif')
    hoffs = [0]
    for n in range(1, NMAX + 1):
        hoffs.append(hoffs[-1] + n)
    lines.append('RYS_CONST_SMALL int RYS_HERM_OFFSET[%d] = {0, %s};' % (
        NMAX + 2, ', '.join(str(o) for o in hoffs)))
    lines.append('// squared positive roots h_i^2 of H_2n, ascending')
    lines.append('RYS_CONST_SMALL double RYS_HERM_R2[%d] = {%s};' % (hoffs[-1], ', '.join(
        '%.17g' % float(h * h) for n in range(1, NMAX + 1) for h, W in herm[n])))
    lines.append('// Gauss-Hermite weights of those roots')
    lines.append('RYS_CONST_SMALL double RYS_HERM_W[%d] = {%s};' % (hoffs[-1], ', '.join(
        '%.17g' % float(W) for n in range(1, NMAX + 1) for h, W in herm[n])))
    with open(OUT_INC, 'w') as f:
        f.write('\n'.join(lines) + '\n')
    with open(OUT_REPORT, 'w') as f:
        json.dump({'xmax': xmax, 'deg': DEG, 'max_rel_fit_error': errs}, f, indent=1)


if __name__ == '__main__':
    main()
