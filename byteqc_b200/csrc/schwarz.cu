// Schwarz factors q_ij = sqrt(max over Cartesian components |(ij|ij)|) of
// every shell pair of one class, on the device.  The reference takes them
// from libcint on the CPU (cuobc/scf/hf.py:341, pyscf CVHFsetnr_direct_scf).
// One thread per pair; the loops over roots and directions are kept rolled
// (this is a one-time setup kernel, compact code matters more than speed).
#include "jk_kernels.cuh"

namespace bqc {

template <int LI, int LJ>
__global__ void schwarz_kernel(JKArgs A, int p0, int np, int pa0, int nprim, double diag_fac,
                               double *q_out) {
    constexpr int NFI = ncart(LI), NFJ = ncart(LJ);
    constexpr int NR = LI + LJ + 1;
    constexpr int GSZ = (LI + 1) * (LJ + 1) * (LI + 1) * (LJ + 1);
    constexpr int SJ = (LI + 1) * (LJ + 1), SI = (LJ + 1) * SJ;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    Quartet Q;
    load_quartet(A, p0 + t, p0 + t, Q);
    Q.fac = TWO_PI_2P5;
    double acc[NFI * NFJ], prod[NFI * NFJ];
#pragma unroll
    for (int n = 0; n < NFI * NFJ; n++) acc[n] = 0;
    int pa = pa0 + t * nprim;
    for (int ip = 0; ip < nprim; ip++) {
        for (int kp = 0; kp < nprim; kp++) {
            PrimQuartet P;
            load_prim(A, Q, pa + ip, pa + kp, P);
#pragma unroll 1
            for (int r = 0; r < NR; r++) {
                double s = rys_one<NR>(A.rys, P.x, r);
                double w = rys_one<NR>(A.rys, P.x, NR + r);
                RootCoef c = root_coef(s, P.p, P.q, P.inv_pq);
#pragma unroll 1
                for (int d = 0; d < 3; d++) {
                    double g[GSZ];
                    double ab = Q.A[d] - Q.B[d];
                    gen_2d<LI, LJ, LI, LJ, double>(d == 2 ? w * P.pref : 1.0,
                                                   P.PA[d] - c.qs * P.PQ[d],
                                                   P.QC[d] + c.ps * P.PQ[d], c.b00, c.b10,
                                                   c.b01, ab, ab, g);
#define BQC_DIAG(D)                                                                   \
    _Pragma("unroll") for (int fi = 0; fi < NFI; fi++)                                \
    _Pragma("unroll") for (int fj = 0; fj < NFJ; fj++) {                              \
        int ix = cart_pow(LI, fi, D), jx = cart_pow(LJ, fj, D);                       \
        double v = g[ix * SI + jx * SJ + ix * (LJ + 1) + jx];                        \
        if (D == 0) prod[fi * NFJ + fj] = v;                                          \
        else if (D == 1) prod[fi * NFJ + fj] *= v;                                    \
        else acc[fi * NFJ + fj] += prod[fi * NFJ + fj] * v;                           \
    }
                    if (d == 0) { BQC_DIAG(0) }
                    else if (d == 1) { BQC_DIAG(1) }
                    else { BQC_DIAG(2) }
#undef BQC_DIAG
                }
            }
        }
    }
    double m = 0;
#pragma unroll
    for (int n = 0; n < NFI * NFJ; n++) m = fmax(m, fabs(acc[n]));
    if (Q.ish == Q.jsh) m /= diag_fac * diag_fac;
    q_out[t] = sqrt(m);
}

}  // namespace bqc

using namespace bqc;

int bqc_launch_schwarz(int li, int lj, const JKArgs &args, int p0, int np, int pa0, int nprim,
                       double diag_fac, double *q_out, cudaStream_t stream) {
    if (np <= 0) return 0;
    int nb = (np + 127) / 128;
    bqc_count_launch(1);
    switch (li * 4 + lj) {
#define BQC_SCASE(a, b)                                                                        \
    case a * 4 + b:                                                                            \
        schwarz_kernel<a, b><<<nb, 128, 0, stream>>>(args, p0, np, pa0, nprim, diag_fac, q_out); \
        break;
        BQC_SCASE(0, 0) BQC_SCASE(1, 0) BQC_SCASE(1, 1) BQC_SCASE(2, 0) BQC_SCASE(2, 1)
        BQC_SCASE(2, 2) BQC_SCASE(3, 0) BQC_SCASE(3, 1) BQC_SCASE(3, 2) BQC_SCASE(3, 3)
#undef BQC_SCASE
    default:
        return 2;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
