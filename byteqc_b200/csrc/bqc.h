// Internal declarations shared by the CUDA translation units of libbyteqc_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "byteqc_b200.h"

#define BQC_LMAX 3          // s, p, d, f
#define BQC_NCART_MAX 10

// Everything a J/K kernel launch reads.  Device pointers unless noted.
struct JKArgs {
    const int *pair_bra;      // shell i of each pair        (bas_pair2bra)
    const int *pair_ket;      // shell j of each pair        (bas_pair2ket)
    const double *a12, *e12, *x12, *y12, *z12;  // primitive-pair data
    const double *bas_x, *bas_y, *bas_z;        // shell centres
    const int *ao_loc;        // Cartesian AO offsets of the sorted, decontracted basis
    const double *pair_q;     // Schwarz factor of each pair, or NULL (no screening)
    const double *dm_cond;    // [nbas*nbas] max |D| over each shell block, or NULL
    const double *dm;         // [n_dm][nao][nao]
    double *vj, *vk;          // [n_dm][nao][nao] accumulated (NULL disables)
    int nao, nbas, n_dm;
    double tol;               // drop quartets with q_ij q_kl max|D| < tol
    double tol_hi;            // and, when > 0, those with a bound >= tol_hi (FP32 band)
    int *status;              // device error word (0 = ok), may be NULL
    const double *rys;        // Rys coefficient table, interval-major (bqc_rys_table())
    const double *rys_lm;     // the same, level-major (bqc_rys_table_lm())
    // ERI output mode (GINTfill_int2e) when eri != NULL: no density screen,
    // no 1/2 for a == b, and instead of the J/K digestion every quartet adds
    // its block (ij|kl) at eri[sum_n (ao_n - eri_off[n]) * eri_stride[n]]
    double *eri;
    long long eri_stride[4];
    int eri_off[4];
};

// the same launch arguments with the bra and ket roles of the ERI output
// exchanged (a kernel that evaluates (kl|ij) for (ij|kl))
static inline JKArgs jk_args_swap_eri(const JKArgs &a) {
    JKArgs s = a;
    s.eri_stride[0] = a.eri_stride[2];
    s.eri_stride[1] = a.eri_stride[3];
    s.eri_stride[2] = a.eri_stride[0];
    s.eri_stride[3] = a.eri_stride[1];
    s.eri_off[0] = a.eri_off[2];
    s.eri_off[1] = a.eri_off[3];
    s.eri_off[2] = a.eri_off[0];
    s.eri_off[3] = a.eri_off[1];
    return s;
}

// One rectangular (or triangular, when diag) block of the quartet space.
struct JKTask {
    int a0, na;        // bra pairs [a0, a0 + na) (global pair indices)
    int b0, nb;        // ket pairs
    int pa0, pb0;      // primitive-pair offset of the first bra / ket pair
    int nprim_a, nprim_b;  // primitive pairs per bra / ket pair
    int diag;          // bra and ket lists are the same: keep a >= b only
    int skip_lower;    // reference rule: skip global pair index a < b
    // Optional tile pruning.  Tiles are rows x columns of 16 x 16 quartets,
    // rows over the a list (or the b list when rows_are_b).  With
    // tile_prefix (device, nrows + 1 entries) row r holds the columns
    // [0, tile_prefix[r+1] - tile_prefix[r]) and block x maps to the tile
    // with tile_prefix[r] <= x < tile_prefix[r+1]; without it the grid is
    // the full rectangle.
    const int *tile_prefix;
    const int *tile_col0;   // optional first column of each row (batched molecules)
    int nrows;
    int ntiles;        // number of tiles (blocks) when tile_prefix is set
    int rows_are_b;
    // Persistent launch: when set, the tile count lives on the device (a
    // schedule computed there) and a fixed grid of CTAs strides over the
    // tiles [0, *ntiles_dev); ntiles is then only an upper bound, and the
    // grid holds at most a few CTAs per SM of the nsm SMs.
    const int *ntiles_dev;
    int nsm;
    // parts per tile of a group-kernel launch without ntiles_dev (set by the
    // launcher; with ntiles_dev the kernel derives it from the device count)
    int split;
};

// Parts a group-kernel tile is cut into: a launch with fewer than 16 tiles
// per SM cuts each tile into 2, 4 or 8 interleaved parts (one CTA each), so
// that small builds still fill every SM; larger ones keep one CTA per tile.
__host__ __device__ inline int group_split(int ntiles, int nsm) {
    int s = 1;
    while (s < 8 && (long long)ntiles * s < 16LL * nsm) s *= 2;
    return s;
}

// grid of a launch over ntiles tiles of per_tile CTAs each; persistent
// launches cap it at ctas_per_sm CTAs on each SM
static inline int bqc_grid(const JKTask &t, int ntiles, int per_tile, int ctas_per_sm) {
    const long long n = (long long)ntiles * per_tile;
    if (t.ntiles_dev == nullptr) return (int)n;
    const long long cap = (long long)t.nsm * ctas_per_sm;
    return (int)(n < cap ? n : cap);
}

// number of kernel launches issued by the library so far (all threads)
unsigned long long bqc_count_launch(int n);

// launch variant of a class (canonical order), see launch_class
#define BQC_VARIANT_AUTO 0
#define BQC_VARIANT_GROUP 1
#define BQC_VARIANT_SPLIT 2
int bqc_class_variant(int li, int lj, int lk, int ll);

// device address of the Rys coefficient table on the current device (rys_table.cu)
const double *bqc_rys_table();
const double *bqc_rys_table_lm();

// launchers (jk_dispatch.cu, schwarz.cu)
int bqc_launch_jk(int li, int lj, int lk, int ll, const JKArgs &args, const JKTask &task,
                  int fp32, cudaStream_t stream);
int bqc_launch_count(const JKArgs &args, const JKTask &task, unsigned long long *count,
                     cudaStream_t stream);
int bqc_launch_dm_cond(const double *dm, int n_dm, int nao, const int *ao_loc, int nbas,
                       double *dm_cond, cudaStream_t stream);
int bqc_launch_schwarz(int li, int lj, const JKArgs &args, int p0, int np, int pa0, int nprim,
                       double diag_fac, double *q_out, cudaStream_t stream);
