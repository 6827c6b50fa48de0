// Class dispatch of the J/K kernels and the density screening kernel.
// Each class launcher bqc_class_<li lj lk ll> is compiled in its own
// translation unit (see byteqc_b200/build.py) so the 55 class templates
// compile in parallel.
#include <stdio.h>
#include <utility>
#include "jk_kernels.cuh"

#define BQC_CASE(a, b, c, d) \
    int bqc_class_##a##b##c##d(const JKArgs &, const JKTask &, int, cudaStream_t);
#include "jk_classes.inc"
#undef BQC_CASE


// (li, lj | lk, ll) with li >= lj, lk >= ll, l <= 3.
static unsigned long long g_launches = 0;

unsigned long long bqc_count_launch(int n) { return __atomic_add_fetch(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }

extern "C" unsigned long long BQClaunch_counter(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

// launch variant per canonical class (li >= lj, lk >= ll, bra pair index >=
// ket pair index); written by BQCset_class_variant, read at every launch
static int g_variant[BQC_LMAX + 1][BQC_LMAX + 1][BQC_LMAX + 1][BQC_LMAX + 1];

int bqc_class_variant(int li, int lj, int lk, int ll) { return g_variant[li][lj][lk][ll]; }

extern "C" int BQCset_class_variant(int li, int lj, int lk, int ll, int variant) {
    if (variant < BQC_VARIANT_AUTO || variant > BQC_VARIANT_SPLIT) return 3;
    if (li < lj) std::swap(li, lj);
    if (lk < ll) std::swap(lk, ll);
    if (li < 0 || lj < 0 || lk < 0 || ll < 0 || li > BQC_LMAX || lk > BQC_LMAX) return 2;
    if (li * (li + 1) / 2 + lj < lk * (lk + 1) / 2 + ll) {
        std::swap(li, lk);
        std::swap(lj, ll);
    }
    g_variant[li][lj][lk][ll] = variant;
    return 0;
}

int bqc_launch_jk(int li, int lj, int lk, int ll, const JKArgs &args, const JKTask &task,
                  int fp32, cudaStream_t stream) {
    bqc_count_launch(1);
    if (li < lj || lk < ll || li > BQC_LMAX || lk > BQC_LMAX) return 2;
    // canonical order: pair index (l1*(l1+1)/2 + l2) of the bra >= that of the ket
    int pij = li * (li + 1) / 2 + lj, pkl = lk * (lk + 1) / 2 + ll;
    JKTask t = task;
    JKArgs a_ = args;   // (not "a": the name is a parameter of BQC_CASE)
    if (pij < pkl) {
        a_ = jk_args_swap_eri(args);
        std::swap(li, lk);
        std::swap(lj, ll);
        t.a0 = task.b0; t.na = task.nb; t.b0 = task.a0; t.nb = task.na;
        t.pa0 = task.pb0; t.pb0 = task.pa0; t.nprim_a = task.nprim_b; t.nprim_b = task.nprim_a;
        t.rows_are_b = !task.rows_are_b;
        // a bra/ket swap of a non-diagonal task changes nothing else; for a
        // diagonal task both lists are identical and the a >= b rule is symmetric
    }
    int key = ((li * 4 + lj) * 4 + lk) * 4 + ll;
    int err = 0;
    switch (key) {
#define BQC_CASE(a, b, c, d) \
    case ((a * 4 + b) * 4 + c) * 4 + d: err = bqc_class_##a##b##c##d(a_, t, fp32, stream); break;
#include "jk_classes.inc"
#undef BQC_CASE
    default:
        return 2;
    }
    if (err) return err;
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) {
        fprintf(stderr, "bqc_launch_jk (%d%d|%d%d): %s\n", li, lj, lk, ll, cudaGetErrorString(ce));
        return 1;
    }
    return 0;
}


// ---------------------------------------------------------------------------
// density block maxima
__global__ void dm_cond_kernel(const double *__restrict__ dm, int n_dm, int nao,
                               const int *__restrict__ ao_loc, int nbas, double *dm_cond) {
    // block (8, 32): 8 lanes reduce one shell block, 32 shells jsh per block
    int ish = blockIdx.y;
    int jsh = blockIdx.x * blockDim.y + threadIdx.y;
    bool valid = jsh < nbas;
    double m = 0;
    if (valid) {
        int i0 = ao_loc[ish], i1 = ao_loc[ish + 1], j0 = ao_loc[jsh], j1 = ao_loc[jsh + 1];
        int ni = i1 - i0, nj = j1 - j0;
        for (int id = 0; id < n_dm; id++) {
            const double *D = dm + (size_t)id * nao * nao;
            for (int e = threadIdx.x; e < ni * nj; e += blockDim.x)
                m = fmax(m, fabs(D[(size_t)(i0 + e / nj) * nao + j0 + e % nj]));
        }
    }
    // every lane of the warp takes part in the shuffles
    for (int o = 4; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffff, m, o, 8));
    if (valid && threadIdx.x == 0) dm_cond[(size_t)ish * nbas + jsh] = m;
}

int bqc_launch_dm_cond(const double *dm, int n_dm, int nao, const int *ao_loc, int nbas,
                       double *dm_cond, cudaStream_t stream) {
    dim3 block(8, 32);
    dim3 grid((nbas + 31) / 32, nbas);
    bqc_count_launch(1);
    dm_cond_kernel<<<grid, block, 0, stream>>>(dm, n_dm, nao, ao_loc, nbas, dm_cond);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}


// ---------------------------------------------------------------------------
// surviving-quartet count of one task (same tiles and screening as the J/K
// kernels, no integrals): the denominator of the algorithmic FLOP count
__global__ void count_kernel(JKArgs A, JKTask T, unsigned long long *count) {
    __shared__ int s_list[bqc::TILE * bqc::TILE];
    __shared__ int s_count;
    const int ntiles = T.ntiles_dev != nullptr ? __ldg(T.ntiles_dev) : (int)gridDim.x;
    for (int x = blockIdx.x; x < ntiles; x += gridDim.x) {
        int a_begin, b_begin, n;
        if (bqc::tile_screen(A, T, x, s_list, &s_count, a_begin, b_begin, n) && threadIdx.x == 0)
            atomicAdd(count, (unsigned long long)n);
        __syncthreads();
    }
}

int bqc_launch_count(const JKArgs &args, const JKTask &task, unsigned long long *count,
                     cudaStream_t stream) {
    int ntiles = task.tile_prefix ? task.ntiles : bqc::task_tiles(task);
    if (ntiles == 0) return 0;
    bqc_count_launch(1);
    count_kernel<<<bqc_grid(task, ntiles, 1, 8), 256, 0, stream>>>(args, task, count);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
