// Device building blocks of the J/K kernels: Rys roots and weights, the
// per-root 2D integral tables (VRR + HRR), Cartesian component tables.
#pragma once
#include "bqc.h"

// The big coefficient table lives in one translation unit (rys_table.cu) and
// reaches the kernels as a pointer (JKArgs::rys); the small index tables are
// compiled into every unit.  RYS_TABLE itself is not defined here.
#define RYS_CONST_SMALL static __constant__ const
#define RYS_NO_BIG_TABLE
#include "rys_tables.inc"
#undef RYS_NO_BIG_TABLE
#undef RYS_CONST_SMALL

namespace bqc {

// number of unit intervals of the order-n table (compile-time copy of RYS_XMAX)
constexpr int kRysXmax[RYS_NMAX + 1] = {RYS_XMAX_LIST};

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// Power of x (d = 0), y (d = 1) or z (d = 2) of Cartesian component c of
// angular momentum l, components ordered x^a y^b z^c with a descending, then
// b descending (the pyscf / libcint order).
__host__ __device__ constexpr int cart_pow(int l, int c, int d) {
    int n = 0;
    for (int a = l; a >= 0; a--) {
        for (int b = l - a; b >= 0; b--) {
            if (n == c) return d == 0 ? a : (d == 1 ? b : l - a - b);
            n++;
        }
    }
    return 0;
}

// Rys nodes s = t^2 and weights of order N at x, FP64, from the fitted tables
// (Chebyshev series on unit intervals, Gauss-Hermite limit beyond XMAX).
// table is the level-major copy (RYS_TABLE_LM): the lanes of a warp hold
// different x and read neighbouring addresses.
template <int N>
__device__ __forceinline__ void rys_roots(const double *__restrict__ table, double x,
                                          double *__restrict__ r, double *__restrict__ w) {
    constexpr int nint = kRysXmax[N];
    if (x < (double)nint) {
        int k = (int)x;
        double t = 2.0 * (x - k) - 1.0;
        double t2 = t + t;
        // level-major layout: (level kk, pair q) rows of XMAX[N] intervals
        const double2 *c = reinterpret_cast<const double2 *>(table + RYS_TABLE_OFFSET[N]) + k;
        double b1[2 * N], b2[2 * N];
#pragma unroll
        for (int q = 0; q < N; q++) {
            double2 v = __ldg(c + ((RYS_NCOEF - 1) * N + q) * nint);
            b1[2 * q] = v.x;
            b1[2 * q + 1] = v.y;
            b2[2 * q] = 0.0;
            b2[2 * q + 1] = 0.0;
        }
#pragma unroll
        for (int kk = RYS_NCOEF - 2; kk >= 1; kk--) {
#pragma unroll
            for (int q = 0; q < N; q++) {
                double2 v = __ldg(c + (kk * N + q) * nint);
                double n0 = fma(t2, b1[2 * q], v.x - b2[2 * q]);
                double n1 = fma(t2, b1[2 * q + 1], v.y - b2[2 * q + 1]);
                b2[2 * q] = b1[2 * q];
                b2[2 * q + 1] = b1[2 * q + 1];
                b1[2 * q] = n0;
                b1[2 * q + 1] = n1;
            }
        }
#pragma unroll
        for (int q = 0; q < N; q++) {
            double2 v = __ldg(c + q * nint);
            double f0 = fma(t, b1[2 * q], v.x - b2[2 * q]);
            double f1 = fma(t, b1[2 * q + 1], v.y - b2[2 * q + 1]);
            // function index 2q and 2q+1: nodes are 0..N-1, weights N..2N-1
            if (2 * q < N) r[2 * q] = f0; else w[2 * q - N] = f0;
            if (2 * q + 1 < N) r[2 * q + 1] = f1; else w[2 * q + 1 - N] = f1;
        }
    } else {
        double ix = 1.0 / x;
        double isx = sqrt(ix);
#pragma unroll
        for (int i = 0; i < N; i++) {
            r[i] = RYS_HERM_R2[RYS_HERM_OFFSET[N] + i] * ix;
            w[i] = RYS_HERM_W[RYS_HERM_OFFSET[N] + i] * isx;
        }
    }
}

// One function of the order-N rule (q < N: node q, q >= N: weight q - N),
// from the interval-major table (the lanes that call it for one x read the
// same interval).
template <int N>
__device__ __forceinline__ double rys_one(const double *__restrict__ table, double x, int q) {
    constexpr int nint = kRysXmax[N];
    if (x < (double)nint) {
        int k = (int)x;
        double t = 2.0 * (x - k) - 1.0;
        double t2 = t + t;
        const double *c = table + RYS_TABLE_OFFSET[N] + k * (RYS_NCOEF * 2 * N) + q;
        double b1 = __ldg(c + (RYS_NCOEF - 1) * 2 * N), b2 = 0.0;
#pragma unroll
        for (int kk = RYS_NCOEF - 2; kk >= 1; kk--) {
            double n0 = fma(t2, b1, __ldg(c + kk * 2 * N) - b2);
            b2 = b1;
            b1 = n0;
        }
        return fma(t, b1, __ldg(c) - b2);
    }
    if (q < N) return RYS_HERM_R2[RYS_HERM_OFFSET[N] + q] / x;
    return RYS_HERM_W[RYS_HERM_OFFSET[N] + q - N] * sqrt(1.0 / x);
}

// 2D integrals of one root and one Cartesian direction for the class
// (LI LJ | LK LL): VRR along i+j and k+l from the seed, then HRR to j (using
// AB = A - B) and to l (using CD = C - D).  The recurrences are those of the
// Rys method (cuobc/lib/gvhf/g2e.cu:32-490):
//   G(n+1, 0) = c00 G(n, 0) + n b10 G(n-1, 0)
//   G(n, m+1) = c0p G(n, m) + m b01 G(n, m-1) + n b00 G(n-1, m)
//   I(i, j+1) = I(i+1, j) + AB I(i, j)
// The result g[i][j][k][l] is written to out[(i*(LJ+1)+j)*RS + k*(LL+1)+l]; the
// row stride RS defaults to (LK+1)(LL+1) (dense) and can be padded.
template <int LI, int LJ, int LK, int LL, typename F, int RS = (LK + 1) * (LL + 1)>
__device__ __forceinline__ void gen_2d(F seed, F c00, F c0p, F b00, F b10, F b01, F ab, F cd,
                                       F *__restrict__ out) {
    constexpr int NM = LI + LJ + 1, MM = LK + LL + 1;
    F G[NM][MM];
    G[0][0] = seed;
#pragma unroll
    for (int n = 1; n < NM; n++) {
        F v = c00 * G[n - 1][0];
        if (n > 1) v += F(n - 1) * b10 * G[n - 2 < 0 ? 0 : n - 2][0];
        G[n][0] = v;
    }
#pragma unroll
    for (int m = 1; m < MM; m++) {
#pragma unroll
        for (int n = 0; n < NM; n++) {
            F v = c0p * G[n][m - 1];
            if (m > 1) v += F(m - 1) * b01 * G[n][m - 2 < 0 ? 0 : m - 2];
            if (n > 0) v += F(n) * b00 * G[n - 1 < 0 ? 0 : n - 1][m - 1];
            G[n][m] = v;
        }
    }
    F H[LI + 1][LJ + 1][MM];
#pragma unroll
    for (int m = 0; m < MM; m++) {
        F t[NM][LJ + 1];
#pragma unroll
        for (int n = 0; n < NM; n++) t[n][0] = G[n][m];
#pragma unroll
        for (int j = 1; j <= LJ; j++) {
#pragma unroll
            for (int i = 0; i < NM - j; i++) t[i][j] = t[i + 1][j - 1] + ab * t[i][j - 1];
        }
#pragma unroll
        for (int i = 0; i <= LI; i++) {
#pragma unroll
            for (int j = 0; j <= LJ; j++) H[i][j][m] = t[i][j];
        }
    }
#pragma unroll
    for (int i = 0; i <= LI; i++) {
#pragma unroll
        for (int j = 0; j <= LJ; j++) {
            F u[MM][LL + 1];
#pragma unroll
            for (int m = 0; m < MM; m++) u[m][0] = H[i][j][m];
#pragma unroll
            for (int l = 1; l <= LL; l++) {
#pragma unroll
                for (int k = 0; k < MM - l; k++) u[k][l] = u[k + 1][l - 1] + cd * u[k][l - 1];
            }
#pragma unroll
            for (int k = 0; k <= LK; k++) {
#pragma unroll
                for (int l = 0; l <= LL; l++)
                    out[(i * (LJ + 1) + j) * RS + k * (LL + 1) + l] = u[k][l];
            }
        }
    }
}

// Per-root recursion coefficients of the Rys method for one primitive
// quartet.  s = t^2 is the root, p = a_i + a_j, q = a_k + a_l.
struct RootCoef {
    double b00, b10, b01, qs, ps;
};
__device__ __forceinline__ RootCoef root_coef(double s, double p, double q, double inv_pq) {
    RootCoef c;
    c.b00 = 0.5 * s * inv_pq;
    c.qs = q * s * inv_pq;
    c.ps = p * s * inv_pq;
    c.b10 = 0.5 * (1.0 - c.qs) / p;
    c.b01 = 0.5 * (1.0 - c.ps) / q;
    return c;
}

}  // namespace bqc
