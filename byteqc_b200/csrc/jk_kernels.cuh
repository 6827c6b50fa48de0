// J/K kernels of the direct-SCF engine for sm_100a.
//
// One template instance per shell-quartet class (LI LJ | LK LL).  A launch
// covers one block of the quartet space of a class pair: bra pairs
// [a0, a0 + na) x ket pairs [b0, b0 + nb), cut into 16 x 16 tiles.  Each CTA
// takes one tile, screens its 256 quartets on the device against
// q_ij q_kl max|D| >= tol (the six density blocks a quartet touches) and
// evaluates the survivors:
//
// * jk_tile: one thread per quartet for classes with at most SMALL_NF
//   Cartesian components, a tile run as two CTAs of 8 x 16 quartets; the 2D
//   integrals and the contracted quartet block live in registers, the six J/K
//   targets are digested from registers with row / column / CTA reductions
//   where the CTA's pairs share a target.
// * jk_group: the survivors are packed into a shared-memory list and each
//   takes TPQ = nfi * nfj * NSPLIT threads; thread
//   (fi, fj, chunk) owns the ket components (fk in its chunk, all fl) of bra
//   component (fi, fj).  Per primitive quartet the group evaluates the Rys
//   roots and the per-root 2D tables (VRR + HRR) cooperatively into shared
//   memory, then every thread accumulates its components.  Digestion: J_ij is
//   a thread-local dot product; the K targets and J_kl are reduced through
//   shared memory before one FP64 atomic per output element.
//
// The per-quartet factors follow the reference (cuobc/lib/gvhf/g2e.cu:1021-1028,
// cuobc/lib/gint/pair_data.c:135-139): 1/2 when the bra and ket pairs are the
// same pair (a == b), and the 1/2 of a diagonal shell pair carried in e12.
#pragma once
#include <stdio.h>
#include <atomic>
#include "jk_device.cuh"

namespace bqc {

constexpr int TILE = 16;
// jk_tile runs a 16 x 16 tile as two CTAs of 8 bra pairs x 16 ket pairs
// (128 threads): two CTAs of the same size share an SM where one 256-thread
// CTA fills the register file, so one CTA's reductions and barriers overlap
// the other's integrals
constexpr int TILE_ROWS = 8;
constexpr int TILE_THREADS = TILE_ROWS * TILE;
constexpr int TILE_WARPS = TILE_THREADS / 32;
constexpr int SMALL_NF = 54;
constexpr double TWO_PI_2P5 = 34.986836655249725693;  // 2 pi^(5/2)

// 8-byte asynchronous global -> shared copies (cp.async, completed by the
// issuing thread's wait): the density blocks a quartet digests are fetched
// while its integrals are evaluated.
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// tile screening: returns false (uniformly) if the tile holds no quartet
__device__ __forceinline__ double dmax6(const double *__restrict__ dmc, int nbas, int i, int j,
                                        int k, int l) {
    double m = fmax(__ldg(dmc + i * nbas + j), __ldg(dmc + k * nbas + l));
    m = fmax(m, __ldg(dmc + i * nbas + k));
    m = fmax(m, __ldg(dmc + i * nbas + l));
    m = fmax(m, __ldg(dmc + j * nbas + k));
    return fmax(m, __ldg(dmc + j * nbas + l));
}

// Tile (row r, column c) of this block.  With tile_prefix (tile_prefix[r] =
// first block of tile row r, non-decreasing) the row is the largest r with
// tile_prefix[r] <= blockIdx.x, found by a 32-way search: each round every
// lane of the warp tests one of 32 evenly spaced candidates and a ballot
// keeps the last one that qualifies, so a row index of up to 2^20 takes four
// rounds of loads instead of twenty dependent ones.  All 32 lanes of every
// warp must call it.
__device__ __forceinline__ void tile_of_block(const JKTask &T, int x, int &r, int &c) {
    if (T.tile_prefix != nullptr) {
        const int lane = threadIdx.x & 31;
        int lo = 0, hi = T.nrows;   // tile_prefix[lo] <= x; answer in [lo, hi)
        while (hi - lo > 1) {
            const int step = (hi - lo + 31) >> 5;
            const int idx = lo + lane * step;
            const bool le = idx < hi && __ldg(T.tile_prefix + idx) <= x;
            const unsigned m = __ballot_sync(0xffffffffu, le);   // bit 0 always set
            lo += (31 - __clz(m)) * step;
            hi = min(hi, lo + step);
        }
        r = lo;
        c = x - __ldg(T.tile_prefix + r);
        if (T.tile_col0 != nullptr) c += __ldg(T.tile_col0 + r);
    } else {
        int ncols = ((T.rows_are_b ? T.na : T.nb) + TILE - 1) / TILE;
        r = x / ncols;
        c = x % ncols;
    }
}

// Surviving quartets of tile x into s_list (order unspecified).  With
// nparts > 1 (a power of two up to 16) only the quartets e = part (mod
// nparts) of the tile's 256 are screened, e = 16 * row + column: part p takes
// every nparts-th column of every row, so the parts are disjoint, cover the
// tile and get similar shares of a q-sorted tile.
__device__ __forceinline__ bool tile_screen(const JKArgs &A, const JKTask &T, int x, int *s_list,
                                            int *s_count, int &a_begin, int &b_begin,
                                            int &count, int part = 0, int nparts = 1) {
    int r, c;
    tile_of_block(T, x, r, c);
    int ta = T.rows_are_b ? c : r, tb = T.rows_are_b ? r : c;
    a_begin = T.a0 + ta * TILE;
    b_begin = T.b0 + tb * TILE;
    int a_end = min(T.a0 + T.na, a_begin + TILE);
    int b_end = min(T.b0 + T.nb, b_begin + TILE);
    if (T.diag && b_begin > a_end - 1) return false;
    if (threadIdx.x == 0) *s_count = 0;
    __syncthreads();
    for (int e0 = threadIdx.x; e0 < TILE * TILE / nparts; e0 += blockDim.x) {
        const int e = e0 * nparts + part;
        int a = a_begin + e / TILE, b = b_begin + e % TILE;
        bool keep = a < a_end && b < b_end && (!T.diag || a >= b);
        if (keep && A.pair_q != nullptr) {
            double bound = __ldg(A.pair_q + a) * __ldg(A.pair_q + b);
            if (A.dm_cond != nullptr) {
                int i = __ldg(A.pair_bra + a), j = __ldg(A.pair_ket + a);
                int k = __ldg(A.pair_bra + b), l = __ldg(A.pair_ket + b);
                bound *= dmax6(A.dm_cond, A.nbas, i, j, k, l);
            }
            keep = bound >= A.tol && (A.tol_hi <= 0. || bound < A.tol_hi);
        }
        if (keep) {
            int idx = atomicAdd(s_count, 1);
            s_list[idx] = ((a - a_begin) << 16) | (b - b_begin);
        }
    }
    __syncthreads();
    count = *s_count;
    return count > 0;
}

struct Quartet {
    int a, b, ish, jsh, ksh, lsh, i0, j0, k0, l0;
    double A[3], B[3], C[3], D[3];
    double fac;
};

__device__ __forceinline__ void load_quartet(const JKArgs &A, int a, int b, Quartet &q) {
    q.a = a;
    q.b = b;
    q.ish = __ldg(A.pair_bra + a);
    q.jsh = __ldg(A.pair_ket + a);
    q.ksh = __ldg(A.pair_bra + b);
    q.lsh = __ldg(A.pair_ket + b);
    q.i0 = __ldg(A.ao_loc + q.ish);
    q.j0 = __ldg(A.ao_loc + q.jsh);
    q.k0 = __ldg(A.ao_loc + q.ksh);
    q.l0 = __ldg(A.ao_loc + q.lsh);
    const int sh[4] = {q.ish, q.jsh, q.ksh, q.lsh};
    double *dst[4] = {q.A, q.B, q.C, q.D};
#pragma unroll
    for (int s = 0; s < 4; s++) {
        dst[s][0] = __ldg(A.bas_x + sh[s]);
        dst[s][1] = __ldg(A.bas_y + sh[s]);
        dst[s][2] = __ldg(A.bas_z + sh[s]);
    }
    q.fac = (a == b && A.eri == nullptr) ? 0.5 * TWO_PI_2P5 : TWO_PI_2P5;
}

// primitive-pair quantities of one primitive quartet
struct PrimQuartet {
    double p, q, inv_pq, inv_p, inv_q, x, pref;
    double PA[3], QC[3], PQ[3];
};

__device__ __forceinline__ void load_prim(const JKArgs &A, const Quartet &Q, int pi, int pk,
                                          PrimQuartet &P) {
    double aij = __ldg(A.a12 + pi), eij = __ldg(A.e12 + pi);
    double akl = __ldg(A.a12 + pk), ekl = __ldg(A.e12 + pk);
    double Pc[3] = {__ldg(A.x12 + pi), __ldg(A.y12 + pi), __ldg(A.z12 + pi)};
    double Qc[3] = {__ldg(A.x12 + pk), __ldg(A.y12 + pk), __ldg(A.z12 + pk)};
    P.p = aij;
    P.q = akl;
    const double s = aij + akl, pq = aij * akl;
    // 1/(p+q), 1/p and 1/q from one division
    const double t = 1.0 / (pq * s);
    P.inv_pq = pq * t;
    P.inv_p = akl * s * t;
    P.inv_q = aij * s * t;
    double rr = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        P.PA[d] = Pc[d] - Q.A[d];
        P.QC[d] = Qc[d] - Q.C[d];
        P.PQ[d] = Pc[d] - Qc[d];
        rr += P.PQ[d] * P.PQ[d];
    }
    P.x = pq * P.inv_pq * rr;
    P.pref = Q.fac * eij * ekl * (P.inv_p * P.inv_q) * rsqrt(s);
}

// recursion coefficients of root s, without a division
__device__ __forceinline__ RootCoef root_coef(double s, const PrimQuartet &P) {
    RootCoef c;
    c.b00 = 0.5 * s * P.inv_pq;
    c.qs = P.q * s * P.inv_pq;
    c.ps = P.p * s * P.inv_pq;
    c.b10 = 0.5 * (1.0 - c.qs) * P.inv_p;
    c.b01 = 0.5 * (1.0 - c.ps) * P.inv_q;
    return c;
}

// ---------------------------------------------------------------------------
// fixed-layout tile kernel: thread (row, col) of a 256-thread CTA evaluates
// quartet (bra pair a_begin + row, ket pair b_begin + col) in registers.
// Contributions that share a target are summed across the tile before the
// atomics: J_ij over the 16 kets of a row, J_kl over the 16 bras of a
// column (warp shuffles, then shared memory across the 8 warps); when all
// bra pairs of the tile share the bra shell i (the 'shell' pair layout of
// _tile_order guarantees it) K_il is summed over a column, when all ket
// pairs share k, K_jk over a row, and K_ik over both; otherwise these K
// targets take one atomic per quartet.
template <int NV>
__device__ __forceinline__ void row_reduce(double (&v)[NV]) {
#pragma unroll
    for (int n = 0; n < NV; n++) {
        double x = v[n];
        x += __shfl_xor_sync(0xffffffffu, x, 8);
        x += __shfl_xor_sync(0xffffffffu, x, 4);
        x += __shfl_xor_sync(0xffffffffu, x, 2);
        x += __shfl_xor_sync(0xffffffffu, x, 1);
        v[n] = x;
    }
}

// Sum v over the rows of the CTA for each column; afterwards threads
// call emit(col, n, sum) for the 16 * NV results.  Every thread must call.
// The shared buffer holds NRED values per (warp, column); longer vectors go
// through it in blocks of NRED.
template <int NV, int NRED, typename Emit>
__device__ __forceinline__ void col_reduce(double (&v)[NV], double (*s_red)[16][NRED], Emit emit) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int n0 = 0; n0 < NV; n0 += NRED) {
        constexpr int NB = NV < NRED ? NV : NRED;
#pragma unroll
        for (int m = 0; m < NB; m++) {
            if (n0 + m < NV) {
                double x = v[n0 + m] + __shfl_xor_sync(0xffffffffu, v[n0 + m], 16);
                if (lane < 16) s_red[warp][lane][m] = x;
            }
        }
        __syncthreads();
        const int nb = imin(NRED, NV - n0);
        for (int o = threadIdx.x; o < 16 * nb; o += blockDim.x) {
            int cc = o / nb, m = o % nb;
            double s = 0;
#pragma unroll
            for (int w = 0; w < TILE_WARPS; w++) s += s_red[w][cc][m];
            emit(cc, n0 + m, s);
        }
        __syncthreads();
    }
}

// K0, KN: the launch evaluates the ket components fk in [K0, K0 + KN) of shell
// k only (all of them by default).  Every J/K target is linear in the quartet
// block, so launches over disjoint fk ranges add up to the whole class; a
// class too large for one thread's registers runs as a few such launches.
// 128-thread CTAs per SM the register budget of jk_tile is sized for (64,
// 85, 128 and 255 registers): small blocks gain occupancy from a tight
// budget, large ones need every register.  Measured on B200 against the
// budgets under which ptxas spills nothing (80-168 registers for the blocks
// of 3-27 components): those removed up to 13e9 local-memory sectors per
// launch of the small classes but lost more to the lower occupancy
// (a full (H2O)_64 / cc-pVTZ build 7 % slower).
__host__ __device__ constexpr int tile_minb(int nf) {
    return nf <= 3 ? 8 : (nf <= 9 ? 6 : (nf <= 27 ? 4 : 2));
}

template <int LI, int LJ, int LK, int LL, typename F, int K0 = 0, int KN = ncart(LK)>
__global__ void __launch_bounds__(TILE_THREADS, tile_minb(ncart(LI) * ncart(LJ) * KN * ncart(LL)))
jk_tile(JKArgs A, JKTask T) {
    static_assert(K0 >= 0 && KN >= 1 && K0 + KN <= ncart(LK), "ket component range");
    // NFK: the components of shell k this launch evaluates, from K0 on
    constexpr int NFI = ncart(LI), NFJ = ncart(LJ), NFK = KN, NFL = ncart(LL);
    constexpr int NIJ = NFI * NFJ, NKL = NFK * NFL, NF = NIJ * NKL;
    constexpr int NR = (LI + LJ + LK + LL) / 2 + 1;
    constexpr int GSZ = (LI + 1) * (LJ + 1) * (LK + 1) * (LL + 1);
    // column-reduction buffer: at most 32 values per (warp, column), 32 KB
    constexpr int NRED = imin(32, imax(NKL, imax(NFI * NFL, NFI * NFK)));
    __shared__ double s_red[TILE_WARPS][16][NRED];

    // half tile vb: bra pairs [a_begin, a_end) x ket pairs [b_begin, b_end)
    auto half_tile = [&](const int vb) {
    int r, c;
    tile_of_block(T, vb >> 1, r, c);
    const int ta = T.rows_are_b ? c : r, tb = T.rows_are_b ? r : c;
    const int a_begin = T.a0 + ta * TILE + (vb & 1) * TILE_ROWS, b_begin = T.b0 + tb * TILE;
    const int a_end = min(T.a0 + T.na, a_begin + TILE_ROWS), b_end = min(T.b0 + T.nb, b_begin + TILE);
    if (a_begin >= a_end || (T.diag && b_begin > a_end - 1)) return;

    const int row = threadIdx.x >> 4, col = threadIdx.x & 15;
    const int a = a_begin + row, b = b_begin + col;
    const bool row_ok = a < a_end, col_ok = b < b_end;
    // shells shared across the half tile
    const int i_tile = __ldg(A.pair_bra + a_begin), k_tile = __ldg(A.pair_bra + b_begin);
    const int ish = row_ok ? __ldg(A.pair_bra + a) : i_tile;
    const int ksh = col_ok ? __ldg(A.pair_bra + b) : k_tile;
    const bool bra_uni = __syncthreads_and(ish == i_tile);
    const bool ket_uni = __syncthreads_and(ksh == k_tile);

    bool active = row_ok && col_ok && (!T.diag || a >= b);
    Quartet Q;
    if (active) {
        load_quartet(A, a, b, Q);
        Q.k0 += K0;   // first AO of the evaluated k components
        if (A.pair_q != nullptr) {
            double bound = __ldg(A.pair_q + a) * __ldg(A.pair_q + b);
            if (A.dm_cond != nullptr) bound *= dmax6(A.dm_cond, A.nbas, Q.ish, Q.jsh, Q.ksh, Q.lsh);
            active = bound >= A.tol && (A.tol_hi <= 0. || bound < A.tol_hi);
        }
    }
    if (!__syncthreads_or(active)) return;

    F acc[NF];
#pragma unroll
    for (int n = 0; n < NF; n++) acc[n] = F(0);
    if (active) {
        F AB[3], CD[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            AB[d] = F(Q.A[d] - Q.B[d]);
            CD[d] = F(Q.C[d] - Q.D[d]);
        }
        const int pa = T.pa0 + (a - T.a0) * T.nprim_a;
        const int pb = T.pb0 + (b - T.b0) * T.nprim_b;
        for (int ip = 0; ip < T.nprim_a; ip++) {
            for (int kp = 0; kp < T.nprim_b; kp++) {
                PrimQuartet P;
                load_prim(A, Q, pa + ip, pb + kp, P);
                double rt[NR], wt[NR];
                rys_roots<NR>(A.rys_lm, P.x, rt, wt);
#pragma unroll
                for (int rr = 0; rr < NR; rr++) {
                    RootCoef cf = root_coef(rt[rr], P);
                    F g[3][GSZ];
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        F seed = (d == 2) ? F(wt[rr] * P.pref) : F(1);
                        gen_2d<LI, LJ, LK, LL, F>(seed, F(P.PA[d] - cf.qs * P.PQ[d]),
                                                  F(P.QC[d] + cf.ps * P.PQ[d]), F(cf.b00),
                                                  F(cf.b10), F(cf.b01), AB[d], CD[d], g[d]);
                    }
#pragma unroll
                    for (int fi = 0; fi < NFI; fi++)
#pragma unroll
                    for (int fj = 0; fj < NFJ; fj++)
#pragma unroll
                    for (int fk = 0; fk < NFK; fk++)
#pragma unroll
                    for (int fl = 0; fl < NFL; fl++) {
                        constexpr int SJ = (LK + 1) * (LL + 1), SI = (LJ + 1) * SJ;
                        const int ix = cart_pow(LI, fi, 0) * SI + cart_pow(LJ, fj, 0) * SJ +
                                       cart_pow(LK, K0 + fk, 0) * (LL + 1) + cart_pow(LL, fl, 0);
                        const int iy = cart_pow(LI, fi, 1) * SI + cart_pow(LJ, fj, 1) * SJ +
                                       cart_pow(LK, K0 + fk, 1) * (LL + 1) + cart_pow(LL, fl, 1);
                        const int iz = cart_pow(LI, fi, 2) * SI + cart_pow(LJ, fj, 2) * SJ +
                                       cart_pow(LK, K0 + fk, 2) * (LL + 1) + cart_pow(LL, fl, 2);
                        acc[((fi * NFJ + fj) * NFK + fk) * NFL + fl] += g[0][ix] * g[1][iy] * g[2][iz];
                    }
                }
            }
        }
    }

    if (A.eri != nullptr) {
        // ERI output mode: add the block, no digestion
        if (active) {
            const long long s0 = A.eri_stride[0], s1 = A.eri_stride[1], s2 = A.eri_stride[2],
                            s3 = A.eri_stride[3];
            double *base = A.eri + (Q.i0 - A.eri_off[0]) * s0 + (Q.j0 - A.eri_off[1]) * s1 +
                           (Q.k0 - A.eri_off[2]) * s2 + (Q.l0 - A.eri_off[3]) * s3;
#pragma unroll
            for (int fi = 0; fi < NFI; fi++)
#pragma unroll
                for (int fj = 0; fj < NFJ; fj++)
#pragma unroll
                    for (int fk = 0; fk < NFK; fk++)
#pragma unroll
                        for (int fl = 0; fl < NFL; fl++)
                            atomicAdd(base + fi * s0 + fj * s1 + fk * s2 + fl * s3,
                                      (double)acc[((fi * NFJ + fj) * NFK + fk) * NFL + fl]);
        }
        return;
    }

    // ---- digestion: one density block and one target at a time ----
    const int nao = A.nao;
    const size_t nn = (size_t)nao * nao;
    const int i0t = __ldg(A.ao_loc + i_tile), k0t = __ldg(A.ao_loc + k_tile) + K0;
#define ACC(fi, fj, fk, fl) ((double)acc[(((fi) * NFJ + (fj)) * NFK + (fk)) * NFL + (fl)])
    for (int id = 0; id < A.n_dm; id++) {
        const double *__restrict__ D = A.dm + id * nn;
        auto ld = [&](int r0, int c0) { return __ldg(D + (size_t)r0 * nao + c0); };
        if (A.vj != nullptr) {
            double *VJ = A.vj + id * nn;
            double pij[NIJ];
#pragma unroll
            for (int n = 0; n < NIJ; n++) pij[n] = 0;
            if (active) {
#pragma unroll
                for (int kl = 0; kl < NKL; kl++) {
                    const double d = ld(Q.k0 + kl / NFL, Q.l0 + kl % NFL);
#pragma unroll
                    for (int ij = 0; ij < NIJ; ij++) pij[ij] += (double)acc[ij * NKL + kl] * d;
                }
            }
            row_reduce(pij);
            if (col == 0 && row_ok) {
                const int jr = __ldg(A.pair_ket + a);
                const int i0 = __ldg(A.ao_loc + ish), j0 = __ldg(A.ao_loc + jr);
#pragma unroll
                for (int n = 0; n < NIJ; n++)
                    if (pij[n] != 0) atomicAdd(VJ + (size_t)(i0 + n / NFJ) * nao + j0 + n % NFJ, pij[n]);
            }
            double pkl[NKL];
#pragma unroll
            for (int n = 0; n < NKL; n++) pkl[n] = 0;
            if (active) {
#pragma unroll
                for (int ij = 0; ij < NIJ; ij++) {
                    const double d = ld(Q.i0 + ij / NFJ, Q.j0 + ij % NFJ);
#pragma unroll
                    for (int kl = 0; kl < NKL; kl++) pkl[kl] += (double)acc[ij * NKL + kl] * d;
                }
            }
            col_reduce<NKL, NRED>(pkl, s_red, [&](int cc, int n, double v) {
                const int bb = b_begin + cc;
                if (v != 0 && bb < b_end) {
                    const int k0 = __ldg(A.ao_loc + __ldg(A.pair_bra + bb)) + K0;
                    const int l0 = __ldg(A.ao_loc + __ldg(A.pair_ket + bb));
                    atomicAdd(VJ + (size_t)(k0 + n / NFL) * nao + l0 + n % NFL, v);
                }
            });
        }
        if (A.vk != nullptr) {
            double *VK = A.vk + id * nn;
            // K_jl = sum_ik (ij|kl) D_ik: one target per quartet
            if (active) {
                double pjl[NFJ * NFL];
#pragma unroll
                for (int n = 0; n < NFJ * NFL; n++) pjl[n] = 0;
#pragma unroll
                for (int fi = 0; fi < NFI; fi++)
#pragma unroll
                    for (int fk = 0; fk < NFK; fk++) {
                        const double d = ld(Q.i0 + fi, Q.k0 + fk);
#pragma unroll
                        for (int fj = 0; fj < NFJ; fj++)
#pragma unroll
                            for (int fl = 0; fl < NFL; fl++) pjl[fj * NFL + fl] += ACC(fi, fj, fk, fl) * d;
                    }
#pragma unroll
                for (int n = 0; n < NFJ * NFL; n++)
                    if (pjl[n] != 0) atomicAdd(VK + (size_t)(Q.j0 + n / NFL) * nao + Q.l0 + n % NFL, pjl[n]);
            }
            // K_jk = sum_il (ij|kl) D_il: shared k -> sum over the row
            {
                double pjk[NFJ * NFK];
#pragma unroll
                for (int n = 0; n < NFJ * NFK; n++) pjk[n] = 0;
                if (active) {
#pragma unroll
                    for (int fi = 0; fi < NFI; fi++)
#pragma unroll
                        for (int fl = 0; fl < NFL; fl++) {
                            const double d = ld(Q.i0 + fi, Q.l0 + fl);
#pragma unroll
                            for (int fj = 0; fj < NFJ; fj++)
#pragma unroll
                                for (int fk = 0; fk < NFK; fk++) pjk[fj * NFK + fk] += ACC(fi, fj, fk, fl) * d;
                        }
                }
                if (ket_uni) {
                    row_reduce(pjk);
                    if (col == 0 && row_ok) {
                        const int j0 = __ldg(A.ao_loc + __ldg(A.pair_ket + a));
#pragma unroll
                        for (int n = 0; n < NFJ * NFK; n++)
                            if (pjk[n] != 0) atomicAdd(VK + (size_t)(j0 + n / NFK) * nao + k0t + n % NFK, pjk[n]);
                    }
                } else if (active) {
#pragma unroll
                    for (int n = 0; n < NFJ * NFK; n++)
                        if (pjk[n] != 0) atomicAdd(VK + (size_t)(Q.j0 + n / NFK) * nao + Q.k0 + n % NFK, pjk[n]);
                }
            }
            // K_il = sum_jk (ij|kl) D_jk: shared i -> sum over the column
            {
                double pil[NFI * NFL];
#pragma unroll
                for (int n = 0; n < NFI * NFL; n++) pil[n] = 0;
                if (active) {
#pragma unroll
                    for (int fj = 0; fj < NFJ; fj++)
#pragma unroll
                        for (int fk = 0; fk < NFK; fk++) {
                            const double d = ld(Q.j0 + fj, Q.k0 + fk);
#pragma unroll
                            for (int fi = 0; fi < NFI; fi++)
#pragma unroll
                                for (int fl = 0; fl < NFL; fl++) pil[fi * NFL + fl] += ACC(fi, fj, fk, fl) * d;
                        }
                }
                if (bra_uni) {
                    col_reduce<NFI * NFL, NRED>(pil, s_red, [&](int cc, int n, double v) {
                        const int bb = b_begin + cc;
                        if (v != 0 && bb < b_end) {
                            const int l0 = __ldg(A.ao_loc + __ldg(A.pair_ket + bb));
                            atomicAdd(VK + (size_t)(i0t + n / NFL) * nao + l0 + n % NFL, v);
                        }
                    });
                } else if (active) {
#pragma unroll
                    for (int n = 0; n < NFI * NFL; n++)
                        if (pil[n] != 0) atomicAdd(VK + (size_t)(Q.i0 + n / NFL) * nao + Q.l0 + n % NFL, pil[n]);
                }
            }
            // K_ik = sum_jl (ij|kl) D_jl
            {
                double pik[NFI * NFK];
#pragma unroll
                for (int n = 0; n < NFI * NFK; n++) pik[n] = 0;
                if (active) {
#pragma unroll
                    for (int fj = 0; fj < NFJ; fj++)
#pragma unroll
                        for (int fl = 0; fl < NFL; fl++) {
                            const double d = ld(Q.j0 + fj, Q.l0 + fl);
#pragma unroll
                            for (int fi = 0; fi < NFI; fi++)
#pragma unroll
                                for (int fk = 0; fk < NFK; fk++) pik[fi * NFK + fk] += ACC(fi, fj, fk, fl) * d;
                        }
                }
                if (bra_uni && ket_uni) {
                    row_reduce(pik);
                    col_reduce<NFI * NFK, NRED>(pik, s_red, [&](int cc, int n, double v) {
                        // after the row sums each column holds its row total, so
                        // column 0 carries the sum over the whole CTA
                        if (cc == 0 && v != 0)
                            atomicAdd(VK + (size_t)(i0t + n / NFK) * nao + k0t + n % NFK, v);
                    });
                } else if (bra_uni) {
                    col_reduce<NFI * NFK, NRED>(pik, s_red, [&](int cc, int n, double v) {
                        const int bb = b_begin + cc;
                        if (v != 0 && bb < b_end) {
                            const int k0 = __ldg(A.ao_loc + __ldg(A.pair_bra + bb)) + K0;
                            atomicAdd(VK + (size_t)(i0t + n / NFK) * nao + k0 + n % NFK, v);
                        }
                    });
                } else if (ket_uni) {
                    row_reduce(pik);
                    if (col == 0 && row_ok) {
                        const int i0 = __ldg(A.ao_loc + ish);
#pragma unroll
                        for (int n = 0; n < NFI * NFK; n++)
                            if (pik[n] != 0) atomicAdd(VK + (size_t)(i0 + n / NFK) * nao + k0t + n % NFK, pik[n]);
                    }
                } else if (active) {
#pragma unroll
                    for (int n = 0; n < NFI * NFK; n++)
                        if (pik[n] != 0) atomicAdd(VK + (size_t)(Q.i0 + n / NFK) * nao + Q.k0 + n % NFK, pik[n]);
                }
            }
        }
    }
#undef ACC
    };
    // one call site, so the body is instantiated once: without a device tile
    // count the grid is exactly the half tiles and the loop runs once
    const int nvb = T.ntiles_dev == nullptr ? (int)gridDim.x : 2 * __ldg(T.ntiles_dev);
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        half_tile(vb);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// group-per-quartet kernel
template <int LI, int LJ, int LK, int LL, int NSPLIT>
struct GroupCfg {
    static constexpr int NFI = ncart(LI), NFJ = ncart(LJ), NFK = ncart(LK), NFL = ncart(LL);
    static constexpr int NIJ = NFI * NFJ, NKL = NFK * NFL;
    static constexpr int NR = (LI + LJ + LK + LL) / 2 + 1;
    static constexpr int TPQ = NIJ * NSPLIT;
    static constexpr int GSZ = (LI + 1) * (LJ + 1) * (LK + 1) * (LL + 1);
    static constexpr int KLS = (LK + 1) * (LL + 1);
    // row stride of the 2D tables in shared memory, odd so that the rows
    // the threads of a group read start in different banks
    static constexpr int KLP = KLS | 1;
    static constexpr int GSZP = (LI + 1) * (LJ + 1) * KLP;
    static constexpr int CK = cdiv(NFK, NSPLIT);
    static constexpr int NACC = CK * NFL;
    static constexpr int GBUF = 3 * NR * GSZP;
    static constexpr int KSLOTS = 2 * NIJ * NFK + 2 * NIJ * NFL * NSPLIT;
    static constexpr int RB = imax(GBUF, KSLOTS);
    static constexpr int FKB = imax(1, RB / (NFL * NIJ));
    static constexpr int DBUF = NIJ + NKL + NFI * NFK + NFI * NFL + NFJ * NFK + NFJ * NFL;
    static constexpr int RW = 2 * NR;
    // doubles per group, odd so that neighbouring groups start in different banks
    static constexpr int PER_GROUP = (RB + DBUF + RW) | 1;
    // groups per CTA: up to NT_CAP threads and at most SMEM_BUDGET bytes of
    // shared memory (four CTAs per SM; small CTAs let the barrier-separated
    // phases of different CTAs overlap on an SM)
    static constexpr int NT_CAP = 128;
    static constexpr int SMEM_BUDGET = 56 * 1024;
    static constexpr int NG = imax(1, imin(NT_CAP / TPQ, SMEM_BUDGET / (PER_GROUP * 8)));
    static constexpr int NT = cdiv(NG * TPQ, 32) * 32;
    static constexpr size_t SMEM = (size_t)NG * PER_GROUP * sizeof(double);
    // CTAs per SM the register budget is sized for (128 registers a thread
    // where the shared memory lets that many CTAs reside; left to itself
    // ptxas picks a budget that can be far too small for the large classes
    // and spills heavily)
    static constexpr int MB_SMEM = (int)(227 * 1024 / (SMEM + 2048));
    static constexpr int MB_THR = NT <= 128 ? 4 : (NT <= 256 ? 2 : 1);
    static constexpr int MINB = imax(1, imin(MB_SMEM, MB_THR));
};

template <int LI, int LJ, int LK, int LL, int NSPLIT, typename F>
__global__ void __launch_bounds__(GroupCfg<LI, LJ, LK, LL, NSPLIT>::NT,
                                  GroupCfg<LI, LJ, LK, LL, NSPLIT>::MINB)
jk_group(JKArgs A, JKTask T) {
    using C = GroupCfg<LI, LJ, LK, LL, NSPLIT>;
    constexpr int NFI = C::NFI, NFJ = C::NFJ, NFK = C::NFK, NFL = C::NFL;
    constexpr int NR = C::NR, TPQ = C::TPQ, NG = C::NG, CK = C::CK;
    extern __shared__ double smem[];
    __shared__ int s_list[TILE * TILE];
    __shared__ int s_count;
    auto tile = [&](const int x, const int part, const int nparts) {
    int a_begin, b_begin, count;
    if (!tile_screen(A, T, x, s_list, &s_count, a_begin, b_begin, count, part, nparts)) return;

    const int g = threadIdx.x / TPQ;
    const int lane = threadIdx.x % TPQ;
    const bool in_group = g < NG;
    double *gbuf = smem + (in_group ? g : 0) * C::PER_GROUP;   // RB: g tables / reduction
    double *dbuf = gbuf + C::RB;                                // density blocks
    double *rw = dbuf + C::DBUF;                                // roots, weights
    F *gtab = reinterpret_cast<F *>(gbuf);                      // per-root 2D tables
    double *Dij = dbuf, *Dkl = Dij + C::NIJ, *Dik = Dkl + C::NKL, *Dil = Dik + NFI * NFK;
    double *Djk = Dil + NFI * NFL, *Djl = Djk + NFJ * NFK;

    const int fij = lane / NSPLIT, chunk = lane % NSPLIT;
    const int fi = fij / NFJ, fj = fij % NFJ;
    int pix = 0, piy = 0, piz = 0, pjx = 0, pjy = 0, pjz = 0;
#pragma unroll
    for (int c = 0; c < NFI; c++)
        if (c == fi) { pix = cart_pow(LI, c, 0); piy = cart_pow(LI, c, 1); piz = cart_pow(LI, c, 2); }
#pragma unroll
    for (int c = 0; c < NFJ; c++)
        if (c == fj) { pjx = cart_pow(LJ, c, 0); pjy = cart_pow(LJ, c, 1); pjz = cart_pow(LJ, c, 2); }
    constexpr int GSZP = C::GSZP;
    const int offx = (pix * (LJ + 1) + pjx) * C::KLP;
    const int offy = GSZP * NR + (piy * (LJ + 1) + pjy) * C::KLP;
    const int offz = 2 * GSZP * NR + (piz * (LJ + 1) + pjz) * C::KLP;

    const int nrounds = (count + NG - 1) / NG;
    for (int round = 0; round < nrounds; round++) {
        const int item = round * NG + g;
        const bool active = in_group && item < count;
        Quartet Q;
        double AB[3] = {0, 0, 0}, CD[3] = {0, 0, 0};
        int pa = 0, pb = 0;
        if (active) {
            int e = s_list[item];
            load_quartet(A, a_begin + (e >> 16), b_begin + (e & 0xffff), Q);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                AB[d] = Q.A[d] - Q.B[d];
                CD[d] = Q.C[d] - Q.D[d];
            }
            pa = T.pa0 + (Q.a - T.a0) * T.nprim_a;
            pb = T.pb0 + (Q.b - T.b0) * T.nprim_b;
        }
        F acc[C::NACC];
#pragma unroll
        for (int n = 0; n < C::NACC; n++) acc[n] = F(0);
        // The six density blocks of this quartet, lane-strided over the group
        // into dbuf (which the 2D tables do not touch); the first density's
        // copies run while the integrals are evaluated.
        auto stage = [&](const double *__restrict__ D) {
            for (int e = lane; e < C::DBUF; e += TPQ) {
                int r0 = 0, c0 = 0, nc = 1, o = e;
                if (o < C::NIJ) { r0 = Q.i0; c0 = Q.j0; nc = NFJ; }
                else if ((o -= C::NIJ) < C::NKL) { r0 = Q.k0; c0 = Q.l0; nc = NFL; }
                else if ((o -= C::NKL) < NFI * NFK) { r0 = Q.i0; c0 = Q.k0; nc = NFK; }
                else if ((o -= NFI * NFK) < NFI * NFL) { r0 = Q.i0; c0 = Q.l0; nc = NFL; }
                else if ((o -= NFI * NFL) < NFJ * NFK) { r0 = Q.j0; c0 = Q.k0; nc = NFK; }
                else { o -= NFJ * NFK; r0 = Q.j0; c0 = Q.l0; nc = NFL; }
                cp_async8(dbuf + e, D + (size_t)(r0 + o / nc) * A.nao + c0 + o % nc);
            }
            cp_async_commit();
        };
        if (active && A.eri == nullptr) stage(A.dm);

        for (int ip = 0; ip < T.nprim_a; ip++) {
            for (int kp = 0; kp < T.nprim_b; kp++) {
                PrimQuartet P;
                if (active) {
                    load_prim(A, Q, pa + ip, pb + kp, P);
                    for (int f = lane; f < 2 * NR; f += TPQ) rw[f] = rys_one<NR>(A.rys, P.x, f);
                }
                __syncthreads();
                if (active) {
                    for (int task = lane; task < 3 * NR; task += TPQ) {
                        int r = task / 3, d = task % 3;
                        RootCoef c = root_coef(rw[r], P);
                        double seed = (d == 2) ? rw[NR + r] * P.pref : 1.0;
                        // d is a runtime index, so P and AB/CD sit in local memory
                        // (L1): measured faster than selecting from registers
                        gen_2d<LI, LJ, LK, LL, F, C::KLP>(
                            F(seed), F(P.PA[d] - c.qs * P.PQ[d]), F(P.QC[d] + c.ps * P.PQ[d]),
                            F(c.b00), F(c.b10), F(c.b01), F(AB[d]), F(CD[d]),
                            gtab + (d * NR + r) * GSZP);
                    }
                }
                __syncthreads();
                if (active && lane < TPQ) {
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        const F *gx = gtab + offx + r * GSZP;
                        const F *gy = gtab + offy + r * GSZP;
                        const F *gz = gtab + offz + r * GSZP;
                        if constexpr (NSPLIT == 1) {
                            F xs[C::KLS], ys[C::KLS], zs[C::KLS];
#pragma unroll
                            for (int u = 0; u < C::KLS; u++) {
                                xs[u] = gx[u];
                                ys[u] = gy[u];
                                zs[u] = gz[u];
                            }
#pragma unroll
                            for (int fk = 0; fk < NFK; fk++)
#pragma unroll
                            for (int fl = 0; fl < NFL; fl++) {
                                int ux = cart_pow(LK, fk, 0) * (LL + 1) + cart_pow(LL, fl, 0);
                                int uy = cart_pow(LK, fk, 1) * (LL + 1) + cart_pow(LL, fl, 1);
                                int uz = cart_pow(LK, fk, 2) * (LL + 1) + cart_pow(LL, fl, 2);
                                acc[fk * NFL + fl] = fma(xs[ux] * ys[uy], zs[uz], acc[fk * NFL + fl]);
                            }
                        } else {
#pragma unroll
                            for (int ck = 0; ck < CK; ck++) {
                                int fk = chunk * CK + ck;
                                if (fk < NFK) {
                                    int kx = 0, ky = 0, kz = 0;
#pragma unroll
                                    for (int c = 0; c < NFK; c++)
                                        if (c == fk) { kx = cart_pow(LK, c, 0); ky = cart_pow(LK, c, 1); kz = cart_pow(LK, c, 2); }
                                    const F *rx = gx + kx * (LL + 1);
                                    const F *ry = gy + ky * (LL + 1);
                                    const F *rz = gz + kz * (LL + 1);
#pragma unroll
                                    for (int fl = 0; fl < NFL; fl++) {
                                        acc[ck * NFL + fl] = fma(rx[cart_pow(LL, fl, 0)] * ry[cart_pow(LL, fl, 1)],
                                                                 rz[cart_pow(LL, fl, 2)], acc[ck * NFL + fl]);
                                    }
                                }
                            }
                        }
                    }
                }
                __syncthreads();
            }
        }

        if (A.eri != nullptr) {
            // ERI output mode: add this thread's components, no digestion
            if (active && lane < TPQ) {
                const long long s0 = A.eri_stride[0], s1 = A.eri_stride[1], s2 = A.eri_stride[2],
                                s3 = A.eri_stride[3];
                double *base = A.eri + (Q.i0 + fi - A.eri_off[0]) * s0 +
                               (Q.j0 + fj - A.eri_off[1]) * s1 + (Q.k0 - A.eri_off[2]) * s2 +
                               (Q.l0 - A.eri_off[3]) * s3;
#pragma unroll
                for (int ck = 0; ck < CK; ck++) {
                    const int fk = chunk * CK + ck;
                    if (fk < NFK) {
#pragma unroll
                        for (int fl = 0; fl < NFL; fl++)
                            atomicAdd(base + fk * s2 + fl * s3, (double)acc[ck * NFL + fl]);
                    }
                }
            }
            continue;
        }

        // ---- digestion ----
        const int nao = A.nao;
        const size_t nn = (size_t)nao * nao;
        for (int id = 0; id < A.n_dm; id++) {
            if (id > 0 && active) stage(A.dm + id * nn);
            cp_async_wait_all();
            __syncthreads();
            if (A.vj != nullptr && active) {
                double s = 0;
#pragma unroll
                for (int ck = 0; ck < CK; ck++) {
                    int fk = chunk * CK + ck;
                    if (fk < NFK) {
#pragma unroll
                        for (int fl = 0; fl < NFL; fl++) s = fma((double)acc[ck * NFL + fl], Dkl[fk * NFL + fl], s);
                    }
                }
                atomicAdd(A.vj + id * nn + (size_t)(Q.i0 + fi) * nao + Q.j0 + fj, s);
            }
            if (A.vk != nullptr) {
                // K partials into shared slots
                double *Sik = gbuf;                              // [fi][fk][fj]
                double *Sjk = Sik + C::NIJ * NFK;                // [fj][fk][fi]
                double *Sil = Sjk + C::NIJ * NFK;                // [fi][fl][fj][chunk]
                double *Sjl = Sil + C::NIJ * NFL * NSPLIT;       // [fj][fl][fi][chunk]
                if (active) {
#pragma unroll
                    for (int ck = 0; ck < CK; ck++) {
                        int fk = chunk * CK + ck;
                        if (fk < NFK) {
                            double sik = 0, sjk = 0;
#pragma unroll
                            for (int fl = 0; fl < NFL; fl++) {
                                sik = fma((double)acc[ck * NFL + fl], Djl[fj * NFL + fl], sik);
                                sjk = fma((double)acc[ck * NFL + fl], Dil[fi * NFL + fl], sjk);
                            }
                            Sik[(fi * NFK + fk) * NFJ + fj] = sik;
                            Sjk[(fj * NFK + fk) * NFI + fi] = sjk;
                        }
                    }
#pragma unroll
                    for (int fl = 0; fl < NFL; fl++) {
                        double sil = 0, sjl = 0;
#pragma unroll
                        for (int ck = 0; ck < CK; ck++) {
                            int fk = chunk * CK + ck;
                            if (fk < NFK) {
                                sil = fma((double)acc[ck * NFL + fl], Djk[fj * NFK + fk], sil);
                                sjl = fma((double)acc[ck * NFL + fl], Dik[fi * NFK + fk], sjl);
                            }
                        }
                        Sil[((fi * NFL + fl) * NFJ + fj) * NSPLIT + chunk] = sil;
                        Sjl[((fj * NFL + fl) * NFI + fi) * NSPLIT + chunk] = sjl;
                    }
                }
                __syncthreads();
                if (active) {
                    double *VK = A.vk + id * nn;
                    constexpr int O1 = NFI * NFK, O2 = O1 + NFJ * NFK, O3 = O2 + NFI * NFL,
                                  O4 = O3 + NFJ * NFL;
                    for (int o = lane; o < O4; o += TPQ) {
                        double s = 0;
                        size_t dst;
                        if (o < O1) {
                            int a = o / NFK, k = o % NFK;
                            for (int j = 0; j < NFJ; j++) s += Sik[(a * NFK + k) * NFJ + j];
                            dst = (size_t)(Q.i0 + a) * nao + Q.k0 + k;
                        } else if (o < O2) {
                            int a = (o - O1) / NFK, k = (o - O1) % NFK;
                            for (int i = 0; i < NFI; i++) s += Sjk[(a * NFK + k) * NFI + i];
                            dst = (size_t)(Q.j0 + a) * nao + Q.k0 + k;
                        } else if (o < O3) {
                            int a = (o - O2) / NFL, l = (o - O2) % NFL;
                            for (int j = 0; j < NFJ * NSPLIT; j++) s += Sil[(a * NFL + l) * NFJ * NSPLIT + j];
                            dst = (size_t)(Q.i0 + a) * nao + Q.l0 + l;
                        } else {
                            int a = (o - O3) / NFL, l = (o - O3) % NFL;
                            for (int i = 0; i < NFI * NSPLIT; i++) s += Sjl[(a * NFL + l) * NFI * NSPLIT + i];
                            dst = (size_t)(Q.j0 + a) * nao + Q.l0 + l;
                        }
                        atomicAdd(VK + dst, s);
                    }
                }
                __syncthreads();
            }
            if (A.vj != nullptr) {
                double *VJ = A.vj + id * nn;
                const double dij = active ? Dij[fi * NFJ + fj] : 0.0;
                for (int fk0 = 0; fk0 < NFK; fk0 += C::FKB) {
                    double *Sj = gbuf;   // [fk - fk0][fl][fij]
                    if (active) {
#pragma unroll
                        for (int ck = 0; ck < CK; ck++) {
                            int fk = chunk * CK + ck;
                            if (fk >= fk0 && fk < fk0 + C::FKB && fk < NFK) {
#pragma unroll
                                for (int fl = 0; fl < NFL; fl++)
                                    Sj[((fk - fk0) * NFL + fl) * C::NIJ + fij] = (double)acc[ck * NFL + fl] * dij;
                            }
                        }
                    }
                    __syncthreads();
                    if (active) {
                        int nk = min(C::FKB, NFK - fk0);
                        for (int o = lane; o < nk * NFL; o += TPQ) {
                            double s = 0;
                            for (int t = 0; t < C::NIJ; t++) s += Sj[o * C::NIJ + t];
                            int fk = fk0 + o / NFL, fl = o % NFL;
                            atomicAdd(VJ + (size_t)(Q.k0 + fk) * nao + Q.l0 + fl, s);
                        }
                    }
                    __syncthreads();
                }
            }
        }
    }
    };
    // virtual block vb = part vb % S of tile vb / S
    int S, nvb;
    if (T.ntiles_dev == nullptr) {
        S = T.split;
        nvb = (int)gridDim.x;
    } else {
        const int n = __ldg(T.ntiles_dev);
        S = group_split(n, T.nsm);
        nvb = n * S;
    }
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        tile(vb / S, vb % S, S);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// dispatch

static inline int task_tiles(const JKTask &task) {
    return ((task.na + TILE - 1) / TILE) * ((task.nb + TILE - 1) / TILE);
}

// Raise the dynamic shared-memory limit of kernel K to `bytes`, once per
// device: the attribute belongs to the (kernel, device) pair, so a process
// that drives several GPUs sets it on each (flags per device, race-free).
constexpr int MAX_DEVICES = 64;
template <auto K>
static int smem_attr(int bytes) {
    static std::atomic<unsigned char> done[MAX_DEVICES];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return 1;
    if (!done[dev].load(std::memory_order_acquire)) {
        if (cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
            return 1;
        done[dev].store(1, std::memory_order_release);
    }
    return 0;
}

// SM count of the current device (cached per device; 0 on error)
static inline int device_sms() {
    static std::atomic<int> sms[MAX_DEVICES];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return 0;
    int n = sms[dev].load(std::memory_order_relaxed);
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        sms[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

template <int LI, int LJ, int LK, int LL, typename F, int K0, int KN>
static int launch_tile_range(const JKArgs &args, const JKTask &task, int ntiles, cudaStream_t stream) {
    jk_tile<LI, LJ, LK, LL, F, K0, KN><<<bqc_grid(task, ntiles, 2, 16), TILE_THREADS, 0, stream>>>(args, task);
    return 0;
}

template <int LI, int LJ, int LK, int LL>
static int launch_small(const JKArgs &args, const JKTask &task, int fp32, cudaStream_t stream) {
    int ntiles = task.tile_prefix ? task.ntiles : task_tiles(task);
    if (ntiles == 0) return 0;
    constexpr int KN = ncart(LK);
    if (fp32) return launch_tile_range<LI, LJ, LK, LL, float, 0, KN>(args, task, ntiles, stream);
    return launch_tile_range<LI, LJ, LK, LL, double, 0, KN>(args, task, ntiles, stream);
}

// Ket-split tile launches: jk_tile over fk in [K0, K0 + CK), [K0 + CK, ...)
// until shell k is covered (one launch each).
template <int LI, int LJ, int LK, int LL, typename F, int K0, int CK>
static int launch_split_f(const JKArgs &args, const JKTask &task, int ntiles, cudaStream_t stream) {
    constexpr int KN = imin(CK, ncart(LK) - K0);
    if (launch_tile_range<LI, LJ, LK, LL, F, K0, KN>(args, task, ntiles, stream)) return 1;
    if constexpr (K0 + CK < ncart(LK))
        return launch_split_f<LI, LJ, LK, LL, F, K0 + CK, CK>(args, task, ntiles, stream);
    return 0;
}

template <int LI, int LJ, int LK, int LL, int CK>
static int launch_split(const JKArgs &args, const JKTask &task, int fp32, cudaStream_t stream) {
    int ntiles = task.tile_prefix ? task.ntiles : task_tiles(task);
    if (ntiles == 0) return 0;
    bqc_count_launch(cdiv(ncart(LK), CK) - 1);   // the dispatcher counted one
    if (fp32) return launch_split_f<LI, LJ, LK, LL, float, 0, CK>(args, task, ntiles, stream);
    return launch_split_f<LI, LJ, LK, LL, double, 0, CK>(args, task, ntiles, stream);
}

template <int LI, int LJ, int LK, int LL, int NSPLIT, typename F>
static int launch_group_f(const JKArgs &args, const JKTask &task, cudaStream_t stream) {
    using C = GroupCfg<LI, LJ, LK, LL, NSPLIT>;
    static_assert(C::SMEM + 2048 <= 227 * 1024, "shared memory per CTA");
    static_assert(C::NT <= 1024, "threads per CTA");
    int ntiles = task.tile_prefix ? task.ntiles : task_tiles(task);
    if (ntiles == 0) return 0;
    if (smem_attr<jk_group<LI, LJ, LK, LL, NSPLIT, F>>((int)C::SMEM)) return 1;
    JKTask t = task;
    int grid;
    if (t.ntiles_dev == nullptr) {
        const int nsm = t.nsm > 0 ? t.nsm : device_sms();
        if (nsm <= 0) return 1;
        t.split = group_split(ntiles, nsm);
        grid = ntiles * t.split;
    } else {
        grid = bqc_grid(t, ntiles, 8, 8);   // the kernel cuts tiles into at most 8 parts
    }
    jk_group<LI, LJ, LK, LL, NSPLIT, F><<<grid, C::NT, C::SMEM, stream>>>(args, t);
    return 0;
}

template <int LI, int LJ, int LK, int LL, int NSPLIT>
static int launch_group(const JKArgs &args, const JKTask &task, int fp32, cudaStream_t stream) {
    if (fp32) return launch_group_f<LI, LJ, LK, LL, NSPLIT, float>(args, task, stream);
    return launch_group_f<LI, LJ, LK, LL, NSPLIT, double>(args, task, stream);
}

// Bra side = pair (LI, LJ) (threads), ket side = pair (LK, LL) (accumulators).
// Small classes run one thread per quartet; larger ones put the pair with
// fewer Cartesian components on the thread side and split the ket
// components into chunks of at most ~36 accumulators.
// Kernel choice per class (canonical order, bra pair index >= ket's):
// at most SMALL_NF Cartesian components: jk_tile; otherwise, when shell k
// splits into at most MAX_SPLIT ranges of fk whose blocks fit SMALL_NF,
// ket-split jk_tile launches or jk_group as bqc_class_variant()
// says (BQCset_class_variant; by default the split for classes of up to
// SPLIT_AUTO ranges); else jk_group.
constexpr int MAX_SPLIT = 3;
constexpr int SPLIT_AUTO = 3;

template <int L1, int L2, int L3, int L4>
static int launch_class(const JKArgs &args, const JKTask &task, int fp32, cudaStream_t stream) {
    constexpr int N12 = ncart(L1) * ncart(L2), N34 = ncart(L3) * ncart(L4);
    if constexpr (N12 * N34 <= SMALL_NF) {
        return launch_small<L1, L2, L3, L4>(args, task, fp32, stream);
    } else {
        constexpr int CK = SMALL_NF / (N12 * ncart(L4));
        constexpr int NCH = CK >= 1 ? cdiv(ncart(L3), CK) : 0;
        if constexpr (NCH >= 1 && NCH <= MAX_SPLIT) {
            const int v = bqc_class_variant(L1, L2, L3, L4);
            if (v == BQC_VARIANT_SPLIT || (v == BQC_VARIANT_AUTO && NCH <= SPLIT_AUTO))
                return launch_split<L1, L2, L3, L4, CK>(args, task, fp32, stream);
        }
        // the task with bra and ket exchanged (diag tasks have identical
        // lists on both sides; the a >= b rule stays)
        JKTask sw = task;
        sw.a0 = task.b0; sw.na = task.nb; sw.b0 = task.a0; sw.nb = task.na;
        sw.pa0 = task.pb0; sw.pb0 = task.pa0; sw.nprim_a = task.nprim_b; sw.nprim_b = task.nprim_a;
        sw.rows_are_b = !task.rows_are_b;
        // an s-s ket pair against a large bra pair ((fd|ss), (ff|ss)): split
        // the bra's first shell instead, with bra and ket exchanged
        constexpr int CKS = SMALL_NF / (N34 * ncart(L2));
        constexpr int NCHS = (NCH == 0 && N34 == 1 && CKS >= 1) ? cdiv(ncart(L1), CKS) : 0;
        if constexpr (NCHS >= 1 && NCHS <= MAX_SPLIT) {
            const int v = bqc_class_variant(L1, L2, L3, L4);
            if (v == BQC_VARIANT_SPLIT || v == BQC_VARIANT_AUTO)
                return launch_split<L3, L4, L1, L2, CKS>(jk_args_swap_eri(args), sw, fp32, stream);
        }
        if constexpr (N12 <= N34) {
            constexpr int NS = cdiv(N34, 36) > ncart(L3) ? ncart(L3) : cdiv(N34, 36);
            return launch_group<L1, L2, L3, L4, NS>(args, task, fp32, stream);
        } else {
            constexpr int NS = cdiv(N12, 36) > ncart(L1) ? ncart(L1) : cdiv(N12, 36);
            return launch_group<L3, L4, L1, L2, NS>(jk_args_swap_eri(args), sw, fp32, stream);
        }
    }
}

}  // namespace bqc
