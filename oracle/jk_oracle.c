/*
 * CPU FP64 oracle for the direct-SCF J/K path.  TEST INFRASTRUCTURE ONLY:
 * the parity tests, the smoke check and the CPU-baseline leg of the benchmark
 * load this library as the checker; the product path never calls it.
 *
 * It restates, in plain C with OpenMP, the algorithm of the reference's
 * cuobc get_jk path:
 *   - primitive pair factors   a12 = ai + aj,
 *       e12 = ci cj fac_sp(li) fac_sp(lj) exp(-ai aj |AB|^2 / a12),
 *       P = (ai A + aj B) / a12                   (cuobc/lib/gint/pair_data.c:83-142)
 *   - ERI prefactor 2 pi^(5/2) / (p q sqrt(p + q))  (cuobc/lib/gint/g2e.c:41,
 *                                                    cuobc/lib/gvhf/g2e.cu:38-46)
 *   - Rys 2D integrals: VRR along (i+j) and (k+l), then HRR to j and l
 *                                                  (cuobc/lib/gvhf/g2e.cu:32-490)
 *   - J/K digestion of each unique quartet (ish>=jsh, ksh>=lsh, ij>=kl) with
 *     the 1/2 factors on ish==jsh, ksh==lsh and ij==kl, into
 *       vj[i,j] += (ij|kl) D[k,l],  vj[k,l] += (ij|kl) D[i,j],
 *       vk[i,k] += D[j,l], vk[i,l] += D[j,k], vk[j,k] += D[i,l], vk[j,l] += D[i,k]
 *                                                  (cuobc/lib/gvhf/contract_jk.cu:225-312)
 *   - J = 2 (V + V^T), K = V + V^T                 (cuobc/scf/hf.py:171-181)
 * It differs from the reference in two deliberate ways: it works on the
 * generally contracted basis as given (the reference first decontracts it,
 * cuobc/scf/hf.py:481-564) and it evaluates every quartet (no screening), so
 * it is exact where the engine screens.
 *
 * Rys roots and weights are computed here independently of the engine's
 * fitted tables: the recurrence coefficients of the weight exp(-x t^2) on
 * t in [0,1] come from the Stieltjes procedure on a 128-point Gauss-Legendre
 * discretisation, the nodes and weights from the Golub-Welsch eigenproblem of
 * the Jacobi matrix (implicit-shift QL).  For x >= 80 the half-range
 * Gauss-Hermite limit is used, its nodes also from Golub-Welsch.
 *
 * One-electron integrals (overlap, kinetic, nuclear attraction) for the SCF
 * energy check use the Obara-Saika overlap recursion and a one-centre Rys
 * quadrature.
 *
 * Basis layout: pyscf _atm/_bas/_env (slots as in cuobc/lib/gint/gint.h:28-43),
 * Cartesian components, contraction-major within a shell.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ATM_SLOTS 6
#define BAS_SLOTS 8
#define CHARGE_OF 0
#define PTR_COORD 1
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define NCTR_OF 3
#define PTR_EXP 5
#define PTR_COEFF 6

#define LMAX 4
#define NROOT_MAX 9
#define NGL 128
#define XSWITCH 80.0

static double gl_t[NGL], gl_w[NGL];
static int gl_ready = 0;

/* Gauss-Legendre nodes on [0,1] by Newton iteration on P_N */
static void gl_init(void) {
    if (gl_ready) return;
    for (int i = 0; i < NGL; i++) {
        double z = cos(M_PI * (i + 0.75) / (NGL + 0.5));
        double pp = 0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1, p2 = 0;
            for (int j = 1; j <= NGL; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = NGL * (z * p1 - p2) / (z * z - 1);
            double dz = p1 / pp;
            z -= dz;
            if (fabs(dz) < 1e-17) break;
        }
        gl_t[i] = 0.5 * (1 - z);
        gl_w[i] = 1.0 / ((1 - z * z) * pp * pp);  /* 2/((1-z^2)P'^2) * 1/2 */
    }
    gl_ready = 1;
}

/* Eigenvalues d[] and first eigenvector components z[] of the symmetric
 * tridiagonal matrix (diag d, off-diagonal e[1..n-1]) by implicit QL. */
static int tql(int n, double *d, double *e, double *z) {
    for (int i = 0; i < n; i++) z[i] = (i == 0) ? 1.0 : 0.0;
    /* z holds the first row of the accumulated eigenvector matrix */
    double Z[NROOT_MAX][NROOT_MAX];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) Z[i][j] = (i == j);
    for (int i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0;
    for (int l = 0; l < n; l++) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; m++) {
                double dd = fabs(d[m]) + fabs(d[m + 1]);
                if (fabs(e[m]) + dd == dd) break;
            }
            if (m != l) {
                if (iter++ == 60) return 1;
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = hypot(g, 1.0);
                g = d[m] - d[l] + e[l] / (g + (g >= 0 ? fabs(r) : -fabs(r)));
                double s = 1, c = 1, p = 0;
                int i;
                for (i = m - 1; i >= l; i--) {
                    double f = s * e[i], b = c * e[i];
                    r = hypot(f, g);
                    e[i + 1] = r;
                    if (r == 0) {
                        d[i + 1] -= p;
                        e[m] = 0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    for (int k = 0; k < n; k++) {
                        f = Z[k][i + 1];
                        Z[k][i + 1] = s * Z[k][i] + c * f;
                        Z[k][i] = c * Z[k][i] - s * f;
                    }
                }
                if (r == 0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0;
            }
        } while (m != l);
    }
    for (int i = 0; i < n; i++) z[i] = Z[0][i];
    return 0;
}

static void sort_pairs(int n, double *r, double *w) {
    for (int i = 1; i < n; i++)
        for (int j = i; j > 0 && r[j] < r[j - 1]; j--) {
            double t = r[j]; r[j] = r[j - 1]; r[j - 1] = t;
            t = w[j]; w[j] = w[j - 1]; w[j - 1] = t;
        }
}

/* Rys nodes s_i = t_i^2 and weights of order n at x. */
int oracle_rys(int n, double x, double *r, double *w) {
    double d[NROOT_MAX], e[NROOT_MAX], z[NROOT_MAX];
    if (n < 1 || n > NROOT_MAX) return 1;
    if (x >= XSWITCH) {
        /* Gauss-Hermite with 2n nodes: Jacobi matrix alpha=0, beta_k=k/2 */
        double dd[NROOT_MAX], ee[NROOT_MAX], zz[NROOT_MAX];
        /* the 2n-point rule: use the n-point rule of the even part instead:
         * positive Hermite nodes h with weights W equal the Gauss rule of
         * the weight exp(-u) u^(-1/2) on u = h^2 (generalised Laguerre,
         * alpha = -1/2): alpha_k = 2k + 1/2, beta_k = k (k - 1/2). */
        for (int k = 0; k < n; k++) {
            dd[k] = 2.0 * k + 0.5;
            ee[k] = (k == 0) ? 0 : sqrt(k * (k - 0.5));
        }
        if (tql(n, dd, ee, zz)) return 2;
        double mu0 = sqrt(M_PI) / 2;   /* int_0^inf exp(-h^2) dh */
        for (int i = 0; i < n; i++) {
            r[i] = dd[i] / x;
            w[i] = mu0 * zz[i] * zz[i] / sqrt(x);
        }
        sort_pairs(n, r, w);
        return 0;
    }
    gl_init();
    /* discretised measure: nodes s_k = t_k^2, weights gl_w exp(-x t_k^2) */
    double s[NGL], lam[NGL], p0[NGL], p1[NGL];
    double mu0 = 0;
    for (int k = 0; k < NGL; k++) {
        s[k] = gl_t[k] * gl_t[k];
        lam[k] = gl_w[k] * exp(-x * s[k]);
        mu0 += lam[k];
        p0[k] = 0;
        p1[k] = 1;
    }
    double nrm_prev = 1, nrm = mu0;
    for (int j = 0; j < n; j++) {
        double num = 0;
        for (int k = 0; k < NGL; k++) num += lam[k] * s[k] * p1[k] * p1[k];
        d[j] = num / nrm;
        double b = (j == 0) ? 0 : nrm / nrm_prev;
        e[j] = (j == 0) ? 0 : sqrt(b);
        if (j == n - 1) break;
        double nn = 0;
        for (int k = 0; k < NGL; k++) {
            double p2 = (s[k] - d[j]) * p1[k] - b * p0[k];
            p0[k] = p1[k];
            p1[k] = p2;
            nn += lam[k] * p2 * p2;
        }
        nrm_prev = nrm;
        nrm = nn;
    }
    if (tql(n, d, e, z)) return 2;
    for (int i = 0; i < n; i++) {
        r[i] = d[i];
        w[i] = mu0 * z[i] * z[i];
    }
    sort_pairs(n, r, w);
    return 0;
}

/* ------------------------------------------------------------------------ */
static double fac_sp(int l) {
    return l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0);
}

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart_pow(int l, int *px, int *py, int *pz) {
    int n = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--, n++) {
            px[n] = a;
            py[n] = b;
            pz[n] = l - a - b;
        }
}

typedef struct {
    const int *atm, *bas;
    const double *env;
    int nbas;
    int *ao_loc;
} Basis;

static void shell_info(const Basis *B, int ish, int *l, int *np, int *nc,
                       const double **ex, const double **cf, const double **R) {
    const int *b = B->bas + ish * BAS_SLOTS;
    *l = b[ANG_OF];
    *np = b[NPRIM_OF];
    *nc = b[NCTR_OF];
    *ex = B->env + b[PTR_EXP];
    *cf = B->env + b[PTR_COEFF];
    *R = B->env + B->atm[b[ATOM_OF] * ATM_SLOTS + PTR_COORD];
}

/* Contracted Cartesian block (ish jsh | ksh lsh), layout
 * out[((((ci*ncj + cj)*nck + ck)*ncl + cl)*nfi + fi)*nfj + fj)*nfk + fk)*nfl + fl]
 * where ci.. are contraction columns and fi.. Cartesian components. */
static void eri_block(const Basis *B, int ish, int jsh, int ksh, int lsh, double *out) {
    int li, lj, lk, ll, npi, npj, npk, npl, nci, ncj, nck, ncl;
    const double *ei, *ej, *ek, *el, *ci, *cj, *ck, *cl, *Ri, *Rj, *Rk, *Rl;
    shell_info(B, ish, &li, &npi, &nci, &ei, &ci, &Ri);
    shell_info(B, jsh, &lj, &npj, &ncj, &ej, &cj, &Rj);
    shell_info(B, ksh, &lk, &npk, &nck, &ek, &ck, &Rk);
    shell_info(B, lsh, &ll, &npl, &ncl, &el, &cl, &Rl);
    int nfi = ncart(li), nfj = ncart(lj), nfk = ncart(lk), nfl = ncart(ll);
    int nf = nfi * nfj * nfk * nfl;
    int nctr = nci * ncj * nck * ncl;
    memset(out, 0, sizeof(double) * nf * nctr);
    int pxi[15], pyi[15], pzi[15], pxj[15], pyj[15], pzj[15];
    int pxk[15], pyk[15], pzk[15], pxl[15], pyl[15], pzl[15];
    cart_pow(li, pxi, pyi, pzi);
    cart_pow(lj, pxj, pyj, pzj);
    cart_pow(lk, pxk, pyk, pzk);
    cart_pow(ll, pxl, pyl, pzl);
    int lij = li + lj, lkl = lk + ll;
    int nroots = (lij + lkl) / 2 + 1;
    double AB[3], CD[3], rab2 = 0, rcd2 = 0;
    for (int d = 0; d < 3; d++) {
        AB[d] = Ri[d] - Rj[d];
        CD[d] = Rk[d] - Rl[d];
        rab2 += AB[d] * AB[d];
        rcd2 += CD[d] * CD[d];
    }
    double norm = fac_sp(li) * fac_sp(lj) * fac_sp(lk) * fac_sp(ll);
    double *prim = malloc(sizeof(double) * nf);
    /* 2D tables: g[d][root][n][m] then I[d][root][i][j][k][l] */
    int gn = lij + 1, gm = lkl + 1;
    double g[3][NROOT_MAX][2 * LMAX + 1][2 * LMAX + 1];
    double I[3][nroots][li + 1][lj + 1][lk + 1][ll + 1];
    double h[2 * LMAX + 2][LMAX + 1][2 * LMAX + 1];
    for (int ip = 0; ip < npi; ip++)
    for (int jp = 0; jp < npj; jp++) {
        double ai = ei[ip], aj = ej[jp], p = ai + aj;
        double Eab = exp(-ai * aj / p * rab2);
        double P[3];
        for (int d = 0; d < 3; d++) P[d] = (ai * Ri[d] + aj * Rj[d]) / p;
        for (int kp = 0; kp < npk; kp++)
        for (int lp = 0; lp < npl; lp++) {
            double ak = ek[kp], al = el[lp], q = ak + al;
            double Ecd = exp(-ak * al / q * rcd2);
            double Q[3], PQ2 = 0;
            for (int d = 0; d < 3; d++) {
                Q[d] = (ak * Rk[d] + al * Rl[d]) / q;
                PQ2 += (P[d] - Q[d]) * (P[d] - Q[d]);
            }
            double rho = p * q / (p + q);
            double x = rho * PQ2;
            double rt[NROOT_MAX], wt[NROOT_MAX];
            oracle_rys(nroots, x, rt, wt);
            double pref = 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q)) * Eab * Ecd * norm;
            for (int r = 0; r < nroots; r++) {
                double s = rt[r];
                double B00 = 0.5 * s / (p + q);
                double B10 = (1 - q * s / (p + q)) / (2 * p);
                double B01 = (1 - p * s / (p + q)) / (2 * q);
                for (int d = 0; d < 3; d++) {
                    double C00 = (P[d] - Ri[d]) - q * s / (p + q) * (P[d] - Q[d]);
                    double C0p = (Q[d] - Rk[d]) + p * s / (p + q) * (P[d] - Q[d]);
                    double (*G)[2 * LMAX + 1] = g[d][r];
                    G[0][0] = (d == 2) ? wt[r] * pref : 1.0;
                    for (int n = 0; n < gn - 1; n++)
                        G[n + 1][0] = C00 * G[n][0] + (n ? n * B10 * G[n - 1][0] : 0);
                    for (int m = 0; m < gm - 1; m++) {
                        for (int n = 0; n < gn; n++) {
                            double v = C0p * G[n][m];
                            if (m) v += m * B01 * G[n][m - 1];
                            if (n) v += n * B00 * G[n - 1][m];
                            G[n][m + 1] = v;
                        }
                    }
                    /* HRR on the bra: h(i, j, m) */
                    for (int m = 0; m < gm; m++) {
                        double t[2 * LMAX + 2][LMAX + 1];
                        for (int n = 0; n < gn; n++) t[n][0] = G[n][m];
                        for (int j = 1; j <= lj; j++)
                            for (int i = 0; i <= lij - j; i++)
                                t[i][j] = t[i + 1][j - 1] + AB[d] * t[i][j - 1];
                        for (int i = 0; i <= li; i++)
                            for (int j = 0; j <= lj; j++) h[i][j][m] = t[i][j];
                    }
                    /* HRR on the ket */
                    for (int i = 0; i <= li; i++)
                    for (int j = 0; j <= lj; j++) {
                        double t[2 * LMAX + 2][LMAX + 1];
                        for (int m = 0; m < gm; m++) t[m][0] = h[i][j][m];
                        for (int l = 1; l <= ll; l++)
                            for (int k = 0; k <= lkl - l; k++)
                                t[k][l] = t[k + 1][l - 1] + CD[d] * t[k][l - 1];
                        for (int k = 0; k <= lk; k++)
                            for (int l = 0; l <= ll; l++) I[d][r][i][j][k][l] = t[k][l];
                    }
                }
            }
            /* primitive Cartesian block */
            int n = 0;
            for (int fi = 0; fi < nfi; fi++)
            for (int fj = 0; fj < nfj; fj++)
            for (int fk = 0; fk < nfk; fk++)
            for (int fl = 0; fl < nfl; fl++, n++) {
                double v = 0;
                for (int r = 0; r < nroots; r++)
                    v += I[0][r][pxi[fi]][pxj[fj]][pxk[fk]][pxl[fl]]
                       * I[1][r][pyi[fi]][pyj[fj]][pyk[fk]][pyl[fl]]
                       * I[2][r][pzi[fi]][pzj[fj]][pzk[fk]][pzl[fl]];
                prim[n] = v;
            }
            /* contract into every column combination */
            int c = 0;
            for (int a = 0; a < nci; a++)
            for (int b = 0; b < ncj; b++)
            for (int e = 0; e < nck; e++)
            for (int f = 0; f < ncl; f++, c++) {
                double cc = ci[a * npi + ip] * cj[b * npj + jp] * ck[e * npk + kp] * cl[f * npl + lp];
                double *o = out + (size_t)c * nf;
                for (int k = 0; k < nf; k++) o[k] += cc * prim[k];
            }
        }
    }
    free(prim);
}

static int *make_ao_loc(const int *bas, int nbas) {
    int *ao_loc = malloc(sizeof(int) * (nbas + 1));
    ao_loc[0] = 0;
    for (int i = 0; i < nbas; i++) {
        const int *b = bas + i * BAS_SLOTS;
        ao_loc[i + 1] = ao_loc[i] + ncart(b[ANG_OF]) * b[NCTR_OF];
    }
    return ao_loc;
}

/* Block of shells (ish jsh|ksh lsh) in AO layout: out[i][j][k][l] over the
 * AOs of the four shells (contraction-major inside each shell). */
int oracle_eri_shells(const int *atm, int natm, const int *bas, int nbas, const double *env,
                      int ish, int jsh, int ksh, int lsh, double *out) {
    Basis B = {atm, bas, env, nbas, NULL};
    int sh[4] = {ish, jsh, ksh, lsh};
    int l[4], nc[4], nf[4], dim[4];
    for (int a = 0; a < 4; a++) {
        const int *b = bas + sh[a] * BAS_SLOTS;
        l[a] = b[ANG_OF];
        nc[a] = b[NCTR_OF];
        nf[a] = ncart(l[a]);
        dim[a] = nf[a] * nc[a];
    }
    int nft = nf[0] * nf[1] * nf[2] * nf[3];
    int nct = nc[0] * nc[1] * nc[2] * nc[3];
    double *blk = malloc(sizeof(double) * nft * nct);
    eri_block(&B, ish, jsh, ksh, lsh, blk);
    for (int a = 0; a < nc[0]; a++) for (int b = 0; b < nc[1]; b++)
    for (int c = 0; c < nc[2]; c++) for (int d = 0; d < nc[3]; d++) {
        double *src = blk + (size_t)(((a * nc[1] + b) * nc[2] + c) * nc[3] + d) * nft;
        int n = 0;
        for (int i = 0; i < nf[0]; i++) for (int j = 0; j < nf[1]; j++)
        for (int k = 0; k < nf[2]; k++) for (int m = 0; m < nf[3]; m++, n++) {
            int I = a * nf[0] + i, J = b * nf[1] + j, K = c * nf[2] + k, L = d * nf[3] + m;
            out[((size_t)(I * dim[1] + J) * dim[2] + K) * dim[3] + L] = src[n];
        }
    }
    free(blk);
    return 0;
}

/* Full J/K over all unique shell quartets.  dm: n_dm x nao x nao (Cartesian,
 * symmetric).  vj, vk: outputs (may be NULL), same shape, overwritten. */
int oracle_jk(const int *atm, int natm, const int *bas, int nbas, const double *env,
              const double *dm, int n_dm, double *vj, double *vk, int nthreads) {
    gl_init();
    int *ao_loc = make_ao_loc(bas, nbas);
    int nao = ao_loc[nbas];
    size_t nn = (size_t)nao * nao;
    int npair = nbas * (nbas + 1) / 2;
    int *pi = malloc(sizeof(int) * npair), *pj = malloc(sizeof(int) * npair);
    for (int i = 0, n = 0; i < nbas; i++)
        for (int j = 0; j <= i; j++, n++) { pi[n] = i; pj[n] = j; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    double *VJ = calloc((size_t)nthr * n_dm * nn, sizeof(double));
    double *VK = calloc((size_t)nthr * n_dm * nn, sizeof(double));
    #pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *vjt = VJ + (size_t)tid * n_dm * nn;
        double *vkt = VK + (size_t)tid * n_dm * nn;
        size_t maxblk = 0;
        for (int i = 0; i < nbas; i++) {
            size_t d = ao_loc[i + 1] - ao_loc[i];
            if (d > maxblk) maxblk = d;
        }
        double *blk = malloc(sizeof(double) * maxblk * maxblk * maxblk * maxblk);
        #pragma omp for schedule(dynamic, 1)
        for (int ij = 0; ij < npair; ij++) {
            int ish = pi[ij], jsh = pj[ij];
            for (int kl = 0; kl <= ij; kl++) {
                int ksh = pi[kl], lsh = pj[kl];
                oracle_eri_shells(atm, natm, bas, nbas, env, ish, jsh, ksh, lsh, blk);
                double fac = 1.0;
                if (ish == jsh) fac *= 0.5;
                if (ksh == lsh) fac *= 0.5;
                if (ij == kl) fac *= 0.5;
                int i0 = ao_loc[ish], i1 = ao_loc[ish + 1];
                int j0 = ao_loc[jsh], j1 = ao_loc[jsh + 1];
                int k0 = ao_loc[ksh], k1 = ao_loc[ksh + 1];
                int l0 = ao_loc[lsh], l1 = ao_loc[lsh + 1];
                int dj = j1 - j0, dk = k1 - k0, dl = l1 - l0;
                for (int id = 0; id < n_dm; id++) {
                    const double *D = dm + id * nn;
                    double *vJ = vjt + id * nn, *vK = vkt + id * nn;
                    for (int i = i0; i < i1; i++) for (int j = j0; j < j1; j++)
                    for (int k = k0; k < k1; k++) for (int l = l0; l < l1; l++) {
                        double s = fac * blk[(((size_t)(i - i0) * dj + (j - j0)) * dk + (k - k0)) * dl + (l - l0)];
                        vJ[(size_t)i * nao + j] += s * D[(size_t)k * nao + l];
                        vJ[(size_t)k * nao + l] += s * D[(size_t)i * nao + j];
                        vK[(size_t)i * nao + k] += s * D[(size_t)j * nao + l];
                        vK[(size_t)i * nao + l] += s * D[(size_t)j * nao + k];
                        vK[(size_t)j * nao + k] += s * D[(size_t)i * nao + l];
                        vK[(size_t)j * nao + l] += s * D[(size_t)i * nao + k];
                    }
                }
            }
        }
        free(blk);
    }
    for (int id = 0; id < n_dm; id++) {
        for (size_t a = 0; a < (size_t)nao; a++)
        for (size_t b = 0; b < (size_t)nao; b++) {
            double sj = 0, sk = 0;
            for (int t = 0; t < nthr; t++) {
                const double *vjt = VJ + ((size_t)t * n_dm + id) * nn;
                const double *vkt = VK + ((size_t)t * n_dm + id) * nn;
                sj += vjt[a * nao + b] + vjt[b * nao + a];
                sk += vkt[a * nao + b] + vkt[b * nao + a];
            }
            if (vj) vj[id * nn + a * nao + b] = 2.0 * sj;
            if (vk) vk[id * nn + a * nao + b] = sk;
        }
    }
    free(VJ);
    free(VK);
    free(pi);
    free(pj);
    free(ao_loc);
    return 0;
}

/* Schwarz factors q[ish*nbas + jsh] = sqrt(max |(ij|ij)|). */
int oracle_q_cond(const int *atm, int natm, const int *bas, int nbas, const double *env,
                  double *q) {
    gl_init();
    int *ao_loc = make_ao_loc(bas, nbas);
    #pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < nbas; i++) {
        for (int j = 0; j <= i; j++) {
            int di = ao_loc[i + 1] - ao_loc[i], dj = ao_loc[j + 1] - ao_loc[j];
            double *blk = malloc(sizeof(double) * di * dj * di * dj);
            oracle_eri_shells(atm, natm, bas, nbas, env, i, j, i, j, blk);
            double m = 0;
            for (int a = 0; a < di; a++) for (int b = 0; b < dj; b++) {
                double v = fabs(blk[((size_t)(a * dj + b) * di + a) * dj + b]);
                if (v > m) m = v;
            }
            q[i * nbas + j] = q[j * nbas + i] = sqrt(m);
            free(blk);
        }
    }
    free(ao_loc);
    return 0;
}

/* ---------------- one-electron integrals -------------------------------- */
/* 1D overlap table S[i][j] (i <= li+2, j <= lj+2) of x_A^i x_B^j e^{-..} */
static void overlap_1d(double p, double PA, double PB, int imax, int jmax, double S[8][8]) {
    S[0][0] = 1.0;   /* the sqrt(pi/p) exp(..) factor is applied outside */
    for (int i = 0; i <= imax; i++) {
        for (int j = 0; j <= jmax; j++) {
            if (i == 0 && j == 0) continue;
            double v;
            if (j == 0) {
                v = PA * S[i - 1][0] + (i > 1 ? (i - 1) / (2 * p) * S[i - 2][0] : 0);
            } else {
                v = PB * S[i][j - 1] + (j > 1 ? (j - 1) / (2 * p) * S[i][j - 2] : 0)
                  + (i > 0 ? i / (2 * p) * S[i - 1][j - 1] : 0);
            }
            S[i][j] = v;
        }
    }
}

/* S, T, V over Cartesian contracted AOs (nao x nao each; any may be NULL). */
int oracle_int1e(const int *atm, int natm, const int *bas, int nbas, const double *env,
                 double *S, double *T, double *V) {
    gl_init();
    Basis B = {atm, bas, env, nbas, NULL};
    int *ao_loc = make_ao_loc(bas, nbas);
    int nao = ao_loc[nbas];
    #pragma omp parallel for schedule(dynamic, 2)
    for (int ish = 0; ish < nbas; ish++) {
        for (int jsh = 0; jsh < nbas; jsh++) {
            int li, lj, npi, npj, nci, ncj;
            const double *ei, *ej, *ci, *cj, *Ri, *Rj;
            shell_info(&B, ish, &li, &npi, &nci, &ei, &ci, &Ri);
            shell_info(&B, jsh, &lj, &npj, &ncj, &ej, &cj, &Rj);
            int nfi = ncart(li), nfj = ncart(lj);
            int pxi[15], pyi[15], pzi[15], pxj[15], pyj[15], pzj[15];
            cart_pow(li, pxi, pyi, pzi);
            cart_pow(lj, pxj, pyj, pzj);
            double norm = fac_sp(li) * fac_sp(lj);
            double AB[3], rab2 = 0;
            for (int d = 0; d < 3; d++) { AB[d] = Ri[d] - Rj[d]; rab2 += AB[d] * AB[d]; }
            int nroots = (li + lj) / 2 + 1;
            double sblk[15][15], tblk[15][15], vblk[15][15];
            for (int a = 0; a < nci; a++)
            for (int b = 0; b < ncj; b++) {
                memset(sblk, 0, sizeof sblk);
                memset(tblk, 0, sizeof tblk);
                memset(vblk, 0, sizeof vblk);
                for (int ip = 0; ip < npi; ip++)
                for (int jp = 0; jp < npj; jp++) {
                    double ai = ei[ip], aj = ej[jp], p = ai + aj;
                    double cc = ci[a * npi + ip] * cj[b * npj + jp] * norm;
                    double Eab = exp(-ai * aj / p * rab2);
                    double P[3];
                    for (int d = 0; d < 3; d++) P[d] = (ai * Ri[d] + aj * Rj[d]) / p;
                    double S1[3][8][8];
                    for (int d = 0; d < 3; d++)
                        overlap_1d(p, P[d] - Ri[d], P[d] - Rj[d], li + 2, lj + 2, S1[d]);
                    double s0 = pow(M_PI / p, 1.5) * Eab * cc;
                    for (int fi = 0; fi < nfi; fi++)
                    for (int fj = 0; fj < nfj; fj++) {
                        int e1[3] = {pxi[fi], pyi[fi], pzi[fi]};
                        int e2[3] = {pxj[fj], pyj[fj], pzj[fj]};
                        double sx = S1[0][e1[0]][e2[0]], sy = S1[1][e1[1]][e2[1]], sz = S1[2][e1[2]][e2[2]];
                        sblk[fi][fj] += s0 * sx * sy * sz;
                        double k1[3];
                        for (int d = 0; d < 3; d++) {
                            int i = e1[d], j = e2[d];
                            double v = -2 * aj * (2 * j + 1) * S1[d][i][j] + 4 * aj * aj * S1[d][i][j + 2];
                            if (j >= 2) v += j * (j - 1) * S1[d][i][j - 2];
                            k1[d] = v;
                        }
                        tblk[fi][fj] += -0.5 * s0 * (k1[0] * sy * sz + sx * k1[1] * sz + sx * sy * k1[2]);
                    }
                    /* nuclear attraction: sum over nuclei, one-centre Rys */
                    for (int ia = 0; ia < natm; ia++) {
                        double Z = atm[ia * ATM_SLOTS + CHARGE_OF];
                        const double *C = env + atm[ia * ATM_SLOTS + PTR_COORD];
                        double PC2 = 0;
                        for (int d = 0; d < 3; d++) PC2 += (P[d] - C[d]) * (P[d] - C[d]);
                        double rt[NROOT_MAX], wt[NROOT_MAX];
                        oracle_rys(nroots, p * PC2, rt, wt);
                        double pref = -Z * 2 * M_PI / p * Eab * cc;
                        double I1[3][NROOT_MAX][LMAX + 1][LMAX + 1];
                        for (int r = 0; r < nroots; r++) {
                            double s = rt[r];
                            double B10 = (1 - s) / (2 * p);
                            for (int d = 0; d < 3; d++) {
                                double C00 = (P[d] - Ri[d]) - s * (P[d] - C[d]);
                                double t[2 * LMAX + 2][LMAX + 1];
                                t[0][0] = (d == 2) ? wt[r] * pref : 1.0;
                                for (int n = 0; n < li + lj; n++)
                                    t[n + 1][0] = C00 * t[n][0] + (n ? n * B10 * t[n - 1][0] : 0);
                                for (int j = 1; j <= lj; j++)
                                    for (int i = 0; i <= li + lj - j; i++)
                                        t[i][j] = t[i + 1][j - 1] + AB[d] * t[i][j - 1];
                                for (int i = 0; i <= li; i++)
                                    for (int j = 0; j <= lj; j++) I1[d][r][i][j] = t[i][j];
                            }
                        }
                        for (int fi = 0; fi < nfi; fi++)
                        for (int fj = 0; fj < nfj; fj++) {
                            double v = 0;
                            for (int r = 0; r < nroots; r++)
                                v += I1[0][r][pxi[fi]][pxj[fj]] * I1[1][r][pyi[fi]][pyj[fj]]
                                   * I1[2][r][pzi[fi]][pzj[fj]];
                            vblk[fi][fj] += v;
                        }
                    }
                }
                int i0 = ao_loc[ish] + a * nfi, j0 = ao_loc[jsh] + b * nfj;
                for (int fi = 0; fi < nfi; fi++)
                for (int fj = 0; fj < nfj; fj++) {
                    size_t o = (size_t)(i0 + fi) * nao + j0 + fj;
                    if (S) S[o] = sblk[fi][fj];
                    if (T) T[o] = tblk[fi][fj];
                    if (V) V[o] = vblk[fi][fj];
                }
            }
        }
    }
    free(ao_loc);
    return 0;
}

int oracle_nao_cart(const int *bas, int nbas) {
    int *ao_loc = make_ao_loc(bas, nbas);
    int n = ao_loc[nbas];
    free(ao_loc);
    return n;
}
