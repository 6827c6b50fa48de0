/*
 * C ABI of libbyteqc_b200.so, the B200 (sm_100a) direct-SCF J/K engine.
 *
 * Two levels of entry points:
 *
 * 1. Drop-in replacements for the reference's libgint/libgvhf symbols that
 *    cuobc/scf/hf.py binds through ctypes.  Names, argument order, argument
 *    meaning, struct layouts and return codes are the reference's, so hf.py
 *    can load this library in place of libgint.so and libgvhf.so.
 *
 * 2. Native whole-build entry points (BQC*), used by this package's own
 *    get_jk: one call screens every quartet on the device against
 *    q_ij q_kl max|D| and builds J and K for all class pairs, replacing the
 *    host loop over class pairs and bins (cuobc/scf/hf.py:111-166).
 *
 * Conventions shared by both levels: Cartesian AOs of the sorted,
 * decontracted basis; dm, vj, vk are n_dm x nao x nao FP64 device arrays;
 * vj/vk are accumulated (the caller zeroes them) with the per-quartet
 * contributions V, and the caller forms J = 2 (V + V^T), K = V + V^T
 * (cuobc/scf/hf.py:171-181).  A NULL vj or vk disables that output.
 * Return codes: 0 ok, 1 CUDA error or unsupported class, 2 angular momentum
 * beyond f (the reference returns 2 for nroots >= 12).
 */
#ifndef BYTEQC_B200_H
#define BYTEQC_B200_H

#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as the reference's ContractionProdType
 * (cuobc/lib/gint/gint.h:101-107). */
typedef struct {
    int l_bra;
    int l_ket;
    int nprim_12;
    int npairs;
} ContractionProdType;

/* Same layout as the reference's BasisProdCache (cuobc/lib/gint/gint.h:118-147);
 * hf.py reads aexyz and primitive_pairs_locs through ctypes. */
typedef struct {
    int nbas;
    int ncptype;
    ContractionProdType *cptype;
    int *bas_pairs_locs;
    int *primitive_pairs_locs;
    int *bas_pair2shls;
    double *aexyz;

    double *bas_coords;
    int *bas_pair2bra;
    int *bas_pair2ket;
    int *ao_loc;
    double *a12;
    double *e12;
    double *x12;
    double *y12;
    double *z12;
} BasisProdCache;

/* ---- level 1: the reference's entry points -------------------------------- */

/* Replaces GINTinit_basis_prod_cpu (cuobc/lib/gint/nr_fill_ao_ints.cu:452-470):
 * builds the class table and the host primitive-pair block
 * aexyz = [a12 | e12 | x12 | y12 | z12] and fills bas_coords (3 x nbas, host). */
void GINTinit_basis_prod_cpu(BasisProdCache **pbp, double diag_fac, double *bas_coords,
                             int *bas_pair2shls, int *bas_pairs_locs, int ncptype,
                             int *atm, int natm, int *bas, int nbas, double *env);

/* Replaces GINTinit_basis_prod_gpu (cuobc/lib/gint/nr_fill_ao_ints.cu:472-491):
 * copies the host cache and points it at device copies of ao_loc, bas_coords,
 * aexyz and bas_pair2shls (device pointers owned by the caller). */
void GINTinit_basis_prod_gpu(BasisProdCache **pbpin, BasisProdCache **pbp, int *ao_loc,
                             double *bas_coords, double *aexyz, int *bas_pair2shls);

/* Replaces GINTdel_basis_prod (cuobc/lib/gint/nr_fill_ao_ints.cu:394-410). */
void GINTdel_basis_prod(BasisProdCache **pbp);

/* Replaces GINTbuild_jk (cuobc/lib/gvhf/nr_jk_driver.cu:227-284): J/K
 * contributions of class pair (cp_ij_id, cp_kl_id) over the binned pair
 * ranges, kl bin b paired with ij bins [0, nbins - b). */
int GINTbuild_jk(BasisProdCache *bpcache, double *vj, double *vk, double *dm, int nao,
                 int n_dm, int *bins_locs_ij, int *bins_locs_kl, int nbins, int cp_ij_id,
                 int cp_kl_id, cudaStream_t stream);

/* ---- level 2: native whole-build entry points ------------------------------ */

/* All class pairs of one J/K build (no reference counterpart; it replaces the
 * per-class-pair loop of cuobc/scf/hf.py:111-166).  pair_q: device Schwarz
 * factor of every pair (same order as bas_pair2shls, sorted descending within
 * each class); pair_q_host: the same on the host, used to launch only the
 * 16 x 16 quartet tiles whose largest bound q_ij q_kl dm_max reaches tol
 * (NULL launches every tile); dm_cond: device nbas x nbas block max |D| (see
 * BQCdm_cond), NULL screens on Schwarz alone; dm_max: max of dm_cond.
 * tol: the direct-SCF threshold.  fp32_below: quartets whose bound
 * q_ij q_kl max|D| is below it are evaluated in FP32 (0 keeps all FP64).
 * status_dev: optional device int set nonzero on an internal error. */
int BQCbuild_jk(const BasisProdCache *bpcache, const double *pair_q, const double *pair_q_host,
                const double *dm_cond, double dm_max, double *vj, double *vk, const double *dm,
                int nao, int n_dm, double tol, double fp32_below, int *status_dev,
                cudaStream_t stream);

/* BQCbuild_jk over the pair lists of many independent molecules at once (no
 * reference counterpart; the batched form).  pair_mol_host gives the
 * molecule of every pair; within each class the 16-pair tiles hold pairs of
 * one molecule, are grouped by molecule in increasing order and sorted by
 * their first q within a molecule.  Only quartets within one molecule are
 * formed; one launch per class pair covers every molecule.  dm/vj/vk are the
 * block-diagonal matrices of all molecules (nao = total AO count). */
int BQCbuild_jk_mol(const BasisProdCache *bpcache, const double *pair_q, const double *pair_q_host,
                    const int *pair_mol_host, const double *dm_cond, double dm_max, double *vj,
                    double *vk, const double *dm, int nao, int n_dm, double tol, double fp32_below,
                    int *status_dev, cudaStream_t stream);

/* One class pair (cp_ij >= cp_kl) of BQCbuild_jk, same arguments otherwise;
 * lets a caller time or profile the kernels class by class. */
int BQCbuild_jk_class(const BasisProdCache *bpcache, int cp_ij, int cp_kl, const double *pair_q,
                      const double *pair_q_host, const double *dm_cond, double dm_max,
                      double *vj, double *vk, const double *dm, int nao, int n_dm, double tol,
                      double fp32_below, int *status_dev, cudaStream_t stream);

/* ERI writer, cuobc/lib/gint/nr_fill_ao_ints.cu:493-551 (GINTfill_int2e):
 * every quartet of class pair (cp_ij_id, cp_kl_id) in the bins
 * ij_bin + kl_bin < nbins (bins_locs_*: host, nbins + 1 offsets into the
 * class's pair list) adds its Cartesian block (ij|kl), i and j from the bra
 * pair, to eri[sum_n (ao_n - ao_offsets[n]) * strides[n]] (strides and
 * ao_offsets: host, 4 entries for i, j, k, l).  No density screening, no
 * symmetry: the caller fills the other index orders (cuobc/lib/int4c.py).
 * The cache should be built with diag factor 1 for plain integrals.
 * Returns 0, 1 on a CUDA error, 2 for l > 3, 3 for bad arguments. */
int GINTfill_int2e(BasisProdCache *bpcache, double *eri, int nao, int *strides, int *ao_offsets,
                   int *bins_locs_ij, int *bins_locs_kl, int nbins, int cp_ij_id, int cp_kl_id,
                   cudaStream_t stream);

/* Number of quartets of class pair (cp_ij, cp_kl) (all class pairs when
 * cp_ij < 0) that pass the screening of BQCbuild_jk, added to the device
 * counter *count_dev; no integrals are evaluated. */
int BQCcount_quartets(const BasisProdCache *bpcache, int cp_ij, int cp_kl, const double *pair_q,
                      const double *pair_q_host, const double *dm_cond, double dm_max,
                      double tol, unsigned long long *count_dev, cudaStream_t stream);

/* FP64 FMA throughput of the current device in FLOP/s, measured by a
 * dependent-chain DFMA microbenchmark (the roofline denominator of the J/K
 * kernels); ms_out (may be NULL) receives the timed kernel's duration. */
int BQCfp64_fma_peak(double *flops_per_s, float *ms_out);

/* Block max |D| per shell pair: dm_cond[i * nbas + j] = max over n_dm and the
 * AOs of shells i, j of |dm|.  ao_loc is a device array (nbas + 1). */
int BQCdm_cond(const double *dm, int n_dm, int nao, const int *ao_loc, int nbas,
               double *dm_cond, cudaStream_t stream);

/* Schwarz factors sqrt(max |(ij|ij)|) of the pairs [p0, p0 + np) of class cp,
 * computed on the device (the reference takes them from libcint on the CPU,
 * cuobc/scf/hf.py:341).  The e12 diagonal factor is undone. */
int BQCschwarz(const BasisProdCache *bpcache, int cp, double diag_fac, double *q_out,
               cudaStream_t stream);

/* One-electron integrals over the Cartesian AOs of shells given in pyscf
 * layout (device copies of atm, bas, env, ao_loc): overlap, kinetic and
 * nuclear attraction, each nao x nao (any may be NULL). */
int BQCint1e(const int *atm, int natm, const int *bas, int nbas, const double *env,
             const int *ao_loc, int nao, double *S, double *T, double *V,
             cudaStream_t stream);

/* BQCbuild_jk for callers that cannot let the library allocate device memory
 * (no reference counterpart).  It allocates nothing: the density-screening
 * scratch is a fixed array inside the library (2 MiB per GPU, held until the
 * process exits), so it accepts at most 512 shells of the sorted, decontracted
 * basis and returns 3 beyond that; it screens on the device against
 * q_ij q_kl max|D| >= tol (pair_q is required: NULL returns 3) and launches
 * every quartet tile.  The first call on
 * a device looks up the array's device address; make that first call before
 * any stream capture.  All calls share the array: calls that overlap on the
 * GPU (different streams, or concurrent host threads) race on it. */
int BQCbuild_jk_noalloc(const BasisProdCache *bpcache, const double *pair_q, double *vj,
                        double *vk, const double *dm, int nao, int n_dm, double tol,
                        cudaStream_t stream);

/* ---- device-scheduled builds ----------------------------------------------
 * No reference counterpart (the reference prunes the quartet tiles on the
 * host and launches one kernel per class pair and log-q bin,
 * cuobc/scf/hf.py:111-166, cuobc/lib/gvhf/nr_jk_driver.cu:252-280).
 *
 * A plan is created once per basis-product cache (device copy, kept alive by
 * the caller) from the host Schwarz factors of its pair list (pair_q_host,
 * descending within each tile of 16 pairs and along the tiles' first
 * pairs; pair_mol_host: the molecule of every pair for batched molecules,
 * else NULL).  BQCbuild_jk_plan then computes dm_max, the surviving 16 x 16
 * tiles of every class pair and their offsets on the device and launches
 * fixed grids that stride over them: no host work, no allocation and the
 * same launches every build, so a build can be captured in a CUDA graph.
 * Its results equal BQCbuild_jk's with the same arguments.  Returns 0, 1 on
 * a CUDA error, 2 for l > 3, 3 for missing arguments. */
typedef struct BQCPlan BQCPlan;
int BQCplan_create(const BasisProdCache *bpcache, const double *pair_q_host,
                   const int *pair_mol_host, BQCPlan **plan);
void BQCplan_destroy(BQCPlan *plan);
int BQCbuild_jk_plan(const BQCPlan *plan, const double *pair_q, const double *dm_cond, double *vj,
                     double *vk, const double *dm, int nao, int n_dm, double tol,
                     double fp32_below, cudaStream_t stream);

/* ---- learned initial density: BF16 tensor-core MLP kernels ----------------
 * No reference counterpart (the reference starts from pyscf's minao guess).
 * Row-major X (M x K, BF16), W (N x K, BF16); M, N, K multiples of 16
 * (return 3 otherwise).  FP32 accumulation. */

/* Z = X W^T + b (FP32, may be NULL); Yf / Yb = act(Z) in FP32 / BF16 (either
 * may be NULL); act = ReLU when relu != 0, identity otherwise. */
int BQCmlp_linear_fwd(const void *X, const void *W, const float *b, float *Z, float *Yf,
                      void *Yb, int M, int N, int K, int relu, cudaStream_t stream);

/* Backward of the layer: dZ = dY * (Z > 0) (Z == NULL: no activation), kept
 * as BF16 in dZ_buf (M x N); dW = dZ^T X, db = sum_m dZ, dX = dZ W (dX may be
 * NULL).  dW, db, dX are overwritten. */
int BQCmlp_linear_bwd(const float *dY, const float *Z, const void *X, const void *W, void *dZ_buf,
                      float *dX, float *dW, float *db, int M, int N, int K, cudaStream_t stream);

/* Adam step on FP32 master weights w (n) with moments m, v; step counts from
 * 1; refreshes the BF16 copy w_bf16 when not NULL. */
int BQCmlp_adam(float *w, const float *g, float *m, float *v, void *w_bf16, int n, float lr,
                float b1, float b2, float eps, int step, cudaStream_t stream);

/* y = bf16(x), n elements. */
int BQCmlp_to_bf16(const float *x, void *y, size_t n, cudaStream_t stream);

/* Kernel choice for shell-quartet class (li lj | lk ll) in this process, any
 * order of the four: variant 0 = built-in rule, 1 = group kernel (threads
 * per quartet share the 2D tables in shared memory), 2 = ket-split tile
 * kernel (one thread per quartet, shell k's components in a few launches,
 * or for an s-s ket against a large bra pair the bra's first shell with bra
 * and ket exchanged; only classes that split into at most 3 such launches,
 * others ignore it).
 * The choice changes speed only, never results.  Returns 0, 2 for l > 3,
 * 3 for an unknown variant.  No reference counterpart (the reference has one
 * fixed kernel per class, cuobc/lib/gvhf/nr_jk_driver.cu:40-225). */
int BQCset_class_variant(int li, int lj, int lk, int ll, int variant);

/* Number of kernel launches the library has issued in this process. */
unsigned long long BQClaunch_counter(void);

/* Library version string. */
const char *BQCversion(void);

#ifdef __cplusplus
}
#endif
#endif
