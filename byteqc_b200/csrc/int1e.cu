// One-electron integrals (overlap, kinetic energy, nuclear attraction) over
// Cartesian AOs of single-contraction shells in pyscf layout.  In the
// reference these come from pyscf's libcint on the CPU (the SCF driver around
// get_jk); the engine computes them on the device so the whole SCF stays on
// the GPU.  One thread per shell pair (ish, jsh).
//   overlap: Obara-Saika 1D recursion
//     S(i+1, j) = PA S(i, j) + (i S(i-1, j) + j S(i, j-1)) / (2p)
//   kinetic: -1/2 d^2/dx^2 acting on the ket,
//     <i|d2|j> = j(j-1) S(i, j-2) - 2 b (2j+1) S(i, j) + 4 b^2 S(i, j+2)
//   nuclear attraction: one-centre Rys quadrature, per nucleus C
//     V = -Z 2 pi / p E_AB sum_r w_r Ix Iy Iz,  x = p |P - C|^2,
//     I(n+1, 0) = (PA - s PC) I(n, 0) + n (1 - s) / (2p) I(n-1, 0), then HRR.
#include <vector>
#include "jk_device.cuh"

#define ATM_SLOTS 6
#define BAS_SLOTS 8

namespace bqc {

template <int LI, int LJ>
__global__ void int1e_kernel(const int *__restrict__ atm, int natm, const int *__restrict__ bas,
                             int nbas, const double *__restrict__ env,
                             const int *__restrict__ ao_loc, int nao, double *S, double *T,
                             double *V, const int *__restrict__ pairs, int npairs,
                             const double *__restrict__ rys) {
    // one thread per (shell pair, Cartesian component fi of the bra shell)
    constexpr int NFI = ncart(LI), NFJ = ncart(LJ);
    constexpr int NR = (LI + LJ) / 2 + 1;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs * NFI) return;
    const int fi = t % NFI;
    t /= NFI;
    int pw[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < NFI; c++)
        if (c == fi) { pw[0] = cart_pow(LI, c, 0); pw[1] = cart_pow(LI, c, 1); pw[2] = cart_pow(LI, c, 2); }
    int ish = pairs[2 * t], jsh = pairs[2 * t + 1];
    const int *bi = bas + ish * BAS_SLOTS, *bj = bas + jsh * BAS_SLOTS;
    const double *A = env + atm[bi[0] * ATM_SLOTS + 1];
    const double *B = env + atm[bj[0] * ATM_SLOTS + 1];
    const double *ei = env + bi[5], *ej = env + bj[5];
    const double *ci = env + bi[6], *cj = env + bj[6];
    double norm = (LI == 0 ? 0.282094791773878143 : (LI == 1 ? 0.488602511902919921 : 1.0)) *
                  (LJ == 0 ? 0.282094791773878143 : (LJ == 1 ? 0.488602511902919921 : 1.0));
    double AB[3], r2 = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        AB[d] = A[d] - B[d];
        r2 += AB[d] * AB[d];
    }
    double s_acc[NFJ], t_acc[NFJ], v_acc[NFJ];
#pragma unroll
    for (int n = 0; n < NFJ; n++) s_acc[n] = t_acc[n] = v_acc[n] = 0;
    for (int ip = 0; ip < bi[2]; ip++) {
        for (int jp = 0; jp < bj[2]; jp++) {
            double a = ei[ip], b = ej[jp], p = a + b, ip2 = 0.5 / p;
            double cc = norm * ci[ip] * cj[jp];
            double Eab = exp(-a * b / p * r2);
            double P[3];
            // 1D overlaps S_d(i, j) for the bra power of this thread, j <= LJ + 2
            double Sx[3][LJ + 3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                P[d] = (a * A[d] + b * B[d]) / p;
                double PA = P[d] - A[d], PB = P[d] - B[d];
                double tab[LI + 1][LJ + 3];
#pragma unroll
                for (int i = 0; i <= LI; i++) {
#pragma unroll
                    for (int j = 0; j <= LJ + 2; j++) {
                        double v;
                        if (i == 0 && j == 0) {
                            v = 1.0;
                        } else if (j == 0) {
                            v = PA * tab[i > 0 ? i - 1 : 0][0];
                            if (i > 1) v += (i - 1) * ip2 * tab[i > 1 ? i - 2 : 0][0];
                        } else {
                            v = PB * tab[i][j - 1];
                            if (j > 1) v += (j - 1) * ip2 * tab[i][j > 1 ? j - 2 : 0];
                            if (i > 0) v += i * ip2 * tab[i > 0 ? i - 1 : 0][j - 1];
                        }
                        tab[i][j] = v;
                    }
                }
#pragma unroll
                for (int j = 0; j <= LJ + 2; j++) {
                    double v = 0;
#pragma unroll
                    for (int i = 0; i <= LI; i++)
                        if (i == pw[d]) v = tab[i][j];
                    Sx[d][j] = v;
                }
            }
            double s0 = pow(M_PI / p, 1.5) * Eab * cc;
#pragma unroll
            for (int fj = 0; fj < NFJ; fj++) {
                double sv[3], kv[3];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int j = cart_pow(LJ, fj, d);
                    sv[d] = Sx[d][j];
                    double k = -2 * b * (2 * j + 1) * Sx[d][j] + 4 * b * b * Sx[d][j + 2];
                    if (j >= 2) k += j * (j - 1) * Sx[d][j >= 2 ? j - 2 : 0];
                    kv[d] = k;
                }
                s_acc[fj] += s0 * sv[0] * sv[1] * sv[2];
                t_acc[fj] += -0.5 * s0 * (kv[0] * sv[1] * sv[2] + sv[0] * kv[1] * sv[2] +
                                          sv[0] * sv[1] * kv[2]);
            }
            if (V != nullptr) {
                for (int ia = 0; ia < natm; ia++) {
                    double Z = atm[ia * ATM_SLOTS];
                    const double *C = env + atm[ia * ATM_SLOTS + 1];
                    double PC[3], pc2 = 0;
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        PC[d] = P[d] - C[d];
                        pc2 += PC[d] * PC[d];
                    }
                    double rt[NR], wt[NR];
                    rys_roots<NR>(rys, p * pc2, rt, wt);
                    double pref = -Z * 2 * M_PI / p * Eab * cc;
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        double b10 = (1 - rt[r]) * ip2;
                        double Ij[3][LJ + 1];
#pragma unroll
                        for (int d = 0; d < 3; d++) {
                            double c00 = (P[d] - A[d]) - rt[r] * PC[d];
                            double I[LI + LJ + 1][LJ + 1];
                            I[0][0] = (d == 2) ? wt[r] * pref : 1.0;
#pragma unroll
                            for (int n = 1; n <= LI + LJ; n++) {
                                double v = c00 * I[n - 1][0];
                                if (n > 1) v += (n - 1) * b10 * I[n > 1 ? n - 2 : 0][0];
                                I[n][0] = v;
                            }
#pragma unroll
                            for (int j = 1; j <= LJ; j++)
#pragma unroll
                                for (int i = 0; i <= LI + LJ - j; i++)
                                    I[i][j] = I[i + 1][j - 1] + AB[d] * I[i][j - 1];
#pragma unroll
                            for (int j = 0; j <= LJ; j++) {
                                double v = 0;
#pragma unroll
                                for (int i = 0; i <= LI; i++)
                                    if (i == pw[d]) v = I[i][j];
                                Ij[d][j] = v;
                            }
                        }
#pragma unroll
                        for (int fj = 0; fj < NFJ; fj++)
                            v_acc[fj] += Ij[0][cart_pow(LJ, fj, 0)] * Ij[1][cart_pow(LJ, fj, 1)] *
                                         Ij[2][cart_pow(LJ, fj, 2)];
                    }
                }
            }
        }
    }
    int i0 = ao_loc[ish], j0 = ao_loc[jsh];
#pragma unroll
    for (int fj = 0; fj < NFJ; fj++) {
        size_t o = (size_t)(i0 + fi) * nao + j0 + fj;
        size_t ot = (size_t)(j0 + fj) * nao + i0 + fi;
        if (S) { S[o] = s_acc[fj]; S[ot] = s_acc[fj]; }
        if (T) { T[o] = t_acc[fj]; T[ot] = t_acc[fj]; }
        if (V) { V[o] = v_acc[fj]; V[ot] = v_acc[fj]; }
    }
}

}  // namespace bqc

using namespace bqc;

extern "C" int BQCint1e(const int *atm, int natm, const int *bas, int nbas, const double *env,
                        const int *ao_loc, int nao, double *S, double *T, double *V,
                        cudaStream_t stream) {
    const double *rys = bqc_rys_table_lm();
    if (rys == nullptr) return 1;
    // group shell pairs (ish >= jsh, l_i >= l_j after ordering) by class on the host
    std::vector<int> hbas(nbas * BAS_SLOTS);
    if (cudaMemcpy(hbas.data(), bas, sizeof(int) * nbas * BAS_SLOTS, cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return 1;
    std::vector<std::vector<int>> lists(16);
    for (int i = 0; i < nbas; i++) {
        if (hbas[i * BAS_SLOTS + 3] != 1) return 1;   // single contractions only
        int li = hbas[i * BAS_SLOTS + 1];
        if (li > BQC_LMAX) return 2;
        for (int j = 0; j <= i; j++) {
            int lj = hbas[j * BAS_SLOTS + 1];
            int a = i, b = j;
            if (li < lj) { a = j; b = i; }
            int la = hbas[a * BAS_SLOTS + 1], lb = hbas[b * BAS_SLOTS + 1];
            lists[la * 4 + lb].push_back(a);
            lists[la * 4 + lb].push_back(b);
        }
    }
    int *dpairs = nullptr;
    size_t tot = 0;
    for (auto &l : lists) tot += l.size();
    if (cudaMalloc(&dpairs, sizeof(int) * (tot > 0 ? tot : 1)) != cudaSuccess) return 1;
    size_t off = 0;
    int err = 0;
    for (int key = 0; key < 16 && !err; key++) {
        auto &l = lists[key];
        if (l.empty()) continue;
        cudaMemcpyAsync(dpairs + off, l.data(), sizeof(int) * l.size(), cudaMemcpyHostToDevice, stream);
        bqc_count_launch(1);
        int np = (int)l.size() / 2;
        int nb = (np * ((key / 4 + 1) * (key / 4 + 2) / 2) + 127) / 128;
        switch (key) {
#define BQC_1CASE(a, b)                                                                        \
    case a * 4 + b:                                                                            \
        int1e_kernel<a, b><<<nb, 128, 0, stream>>>(atm, natm, bas, nbas, env, ao_loc, nao, S, T, \
                                                   V, dpairs + off, np, rys);                       \
        break;
            BQC_1CASE(0, 0) BQC_1CASE(1, 0) BQC_1CASE(1, 1) BQC_1CASE(2, 0) BQC_1CASE(2, 1)
            BQC_1CASE(2, 2) BQC_1CASE(3, 0) BQC_1CASE(3, 1) BQC_1CASE(3, 2) BQC_1CASE(3, 3)
#undef BQC_1CASE
        default:
            err = 2;
        }
        off += l.size();
    }
    cudaStreamSynchronize(stream);
    cudaFree(dpairs);
    if (err) return err;
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
