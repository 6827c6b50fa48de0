// C ABI of libbyteqc_b200: the reference-compatible GINT* entry points and the
// native whole-build BQC* entry points (declared in include/byteqc_b200.h).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include "bqc.h"

#define ATM_SLOTS 6
#define BAS_SLOTS 8
#define PTR_COORD 1
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define PTR_EXP 5
#define PTR_COEFF 6

// normalisation constant of a Cartesian s or p function (the remaining
// spherical-harmonic normalisation of l >= 2 sits in the cart2sph matrix)
static double fac_sp(int l) {
    return l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0);
}

extern "C" {

// Class table and primitive-pair block, as cuobc/lib/gint/pair_data.c:30-142
// defines them: one class per (l_bra, l_ket, nprim_bra * nprim_ket) group of
// consecutive pairs; per primitive pair a12 = ai + aj,
// e12 = fac_sp(li) fac_sp(lj) ci cj exp(-ai aj |AB|^2 / a12) (times diag_fac
// when ish == jsh) and the Gaussian product centre.
void GINTinit_basis_prod_cpu(BasisProdCache **pbp, double diag_fac, double *bas_coords,
                             int *bas_pair2shls, int *bas_pairs_locs, int ncptype, int *atm,
                             int natm, int *bas, int nbas, double *env) {
    (void)natm;
    BasisProdCache *bp = (BasisProdCache *)calloc(1, sizeof(BasisProdCache));
    *pbp = bp;
    bp->nbas = nbas;
    bp->ncptype = ncptype;
    bp->bas_pairs_locs = bas_pairs_locs;
    bp->bas_pair2shls = bas_pair2shls;
    const int npairs_tot = bas_pairs_locs[ncptype];
    const int *bra = bas_pair2shls, *ket = bas_pair2shls + npairs_tot;
    bp->cptype = (ContractionProdType *)malloc(sizeof(ContractionProdType) * (ncptype > 0 ? ncptype : 1));
    bp->primitive_pairs_locs = (int *)malloc(sizeof(int) * (ncptype + 1));
    bp->primitive_pairs_locs[0] = 0;
    for (int c = 0; c < ncptype; c++) {
        int p0 = bas_pairs_locs[c], np = bas_pairs_locs[c + 1] - p0;
        ContractionProdType *t = bp->cptype + c;
        if (np > 0) {
            int ish = bra[p0], jsh = ket[p0];
            t->l_bra = bas[ish * BAS_SLOTS + ANG_OF];
            t->l_ket = bas[jsh * BAS_SLOTS + ANG_OF];
            t->nprim_12 = bas[ish * BAS_SLOTS + NPRIM_OF] * bas[jsh * BAS_SLOTS + NPRIM_OF];
        } else {
            t->l_bra = t->l_ket = 0;
            t->nprim_12 = 1;
        }
        t->npairs = np;
        bp->primitive_pairs_locs[c + 1] = bp->primitive_pairs_locs[c] + np * t->nprim_12;
    }
    const int nprim_tot = bp->primitive_pairs_locs[ncptype];
    double *aexyz = (double *)malloc(sizeof(double) * 5 * (nprim_tot > 0 ? nprim_tot : 1));
    bp->aexyz = aexyz;
    double *a12 = aexyz, *e12 = a12 + nprim_tot, *x12 = e12 + nprim_tot;
    double *y12 = x12 + nprim_tot, *z12 = y12 + nprim_tot;
    int off = 0;
    for (int p = 0; p < npairs_tot; p++) {
        int ish = bra[p], jsh = ket[p];
        const int *bi = bas + ish * BAS_SLOTS, *bj = bas + jsh * BAS_SLOTS;
        const double *ri = env + atm[bi[ATOM_OF] * ATM_SLOTS + PTR_COORD];
        const double *rj = env + atm[bj[ATOM_OF] * ATM_SLOTS + PTR_COORD];
        const double *ai = env + bi[PTR_EXP], *aj = env + bj[PTR_EXP];
        const double *ci = env + bi[PTR_COEFF], *cj = env + bj[PTR_COEFF];
        double norm = fac_sp(bi[ANG_OF]) * fac_sp(bj[ANG_OF]);
        if (ish == jsh) norm *= diag_fac;
        double dx = ri[0] - rj[0], dy = ri[1] - rj[1], dz = ri[2] - rj[2];
        double r2 = dx * dx + dy * dy + dz * dz;
        for (int ip = 0; ip < bi[NPRIM_OF]; ip++) {
            for (int jp = 0; jp < bj[NPRIM_OF]; jp++, off++) {
                double aij = ai[ip] + aj[jp];
                a12[off] = aij;
                e12[off] = norm * ci[ip] * cj[jp] * exp(-r2 * ai[ip] * aj[jp] / aij);
                x12[off] = (ai[ip] * ri[0] + aj[jp] * rj[0]) / aij;
                y12[off] = (ai[ip] * ri[1] + aj[jp] * rj[1]) / aij;
                z12[off] = (ai[ip] * ri[2] + aj[jp] * rj[2]) / aij;
            }
        }
    }
    for (int ib = 0; ib < nbas; ib++) {
        const double *r = env + atm[bas[ib * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
        bas_coords[ib] = r[0];
        bas_coords[ib + nbas] = r[1];
        bas_coords[ib + 2 * nbas] = r[2];
    }
}

void GINTinit_basis_prod_gpu(BasisProdCache **pbpin, BasisProdCache **pbp, int *ao_loc,
                             double *bas_coords, double *aexyz, int *bas_pair2shls) {
    BasisProdCache *bp = (BasisProdCache *)malloc(sizeof(BasisProdCache));
    memcpy(bp, *pbpin, sizeof(BasisProdCache));
    *pbp = bp;
    // The copy shares the host class table, primitive-pair offsets and host
    // aexyz block with the cpu cache (the reference's ownership,
    // cuobc/lib/gint/nr_fill_ao_ints.cu:472-491): GINTdel_basis_prod on
    // either struct frees them, and cuobc/scf/hf.py:439-442 deletes only
    // the device copy.
    bp->ao_loc = ao_loc;
    bp->bas_coords = bas_coords;
    int npairs = bp->bas_pairs_locs[bp->ncptype];
    int nprim = bp->primitive_pairs_locs[bp->ncptype];
    bp->a12 = aexyz;
    bp->e12 = aexyz + nprim;
    bp->x12 = aexyz + 2 * (size_t)nprim;
    bp->y12 = aexyz + 3 * (size_t)nprim;
    bp->z12 = aexyz + 4 * (size_t)nprim;
    bp->bas_pair2bra = bas_pair2shls;
    bp->bas_pair2ket = bas_pair2shls + npairs;
}

// Frees the struct and the host blocks it points at (class table,
// primitive-pair offsets, host aexyz), as cuobc/lib/gint/nr_fill_ao_ints.cu:394-410
// does.  A cpu cache and its device copies share those blocks: a caller that
// keeps both deletes one of them, or clears the shared pointers of the other
// first.
void GINTdel_basis_prod(BasisProdCache **pbp) {
    BasisProdCache *bp = *pbp;
    if (bp == NULL) return;
    if (bp->cptype != NULL) {
        free(bp->cptype);
        free(bp->primitive_pairs_locs);
    }
    if (bp->aexyz != NULL) free(bp->aexyz);
    free(bp);
    *pbp = NULL;
}

static JKArgs make_args(const BasisProdCache *bp, double *vj, double *vk, const double *dm,
                        int nao, int n_dm) {
    JKArgs a;
    memset(&a, 0, sizeof(a));
    a.tol_hi = 0.;
    a.pair_bra = bp->bas_pair2bra;
    a.pair_ket = bp->bas_pair2ket;
    a.a12 = bp->a12;
    a.e12 = bp->e12;
    a.x12 = bp->x12;
    a.y12 = bp->y12;
    a.z12 = bp->z12;
    a.bas_x = bp->bas_coords;
    a.bas_y = bp->bas_coords + bp->nbas;
    a.bas_z = bp->bas_coords + 2 * bp->nbas;
    a.ao_loc = bp->ao_loc;
    a.dm = dm;
    a.vj = vj;
    a.vk = vk;
    a.nao = nao;
    a.nbas = bp->nbas;
    a.n_dm = n_dm;
    a.rys = bqc_rys_table();
    a.rys_lm = bqc_rys_table_lm();
    a.eri = NULL;
    return a;
}

int GINTbuild_jk(BasisProdCache *bpcache, double *vj, double *vk, double *dm, int nao, int n_dm,
                 int *bins_locs_ij, int *bins_locs_kl, int nbins, int cp_ij_id, int cp_kl_id,
                 cudaStream_t stream) {
    const ContractionProdType *cij = bpcache->cptype + cp_ij_id;
    const ContractionProdType *ckl = bpcache->cptype + cp_kl_id;
    int L = cij->l_bra + cij->l_ket + ckl->l_bra + ckl->l_ket;
    if (L / 2 + 1 >= 12) return 2;
    if (cij->l_bra > BQC_LMAX || ckl->l_bra > BQC_LMAX) return 2;
    JKArgs args = make_args(bpcache, vj, vk, dm, nao, n_dm);
    for (int kl_bin = 0; kl_bin < nbins; kl_bin++) {
        int kl0 = bins_locs_kl[kl_bin], kl1 = bins_locs_kl[kl_bin + 1];
        if (kl1 <= kl0) continue;
        int ij0 = bins_locs_ij[0], ij1 = bins_locs_ij[nbins - kl_bin];
        if (ij1 <= ij0) continue;
        JKTask t;
        memset(&t, 0, sizeof(t));
        t.a0 = bpcache->bas_pairs_locs[cp_ij_id] + ij0;
        t.na = ij1 - ij0;
        t.b0 = bpcache->bas_pairs_locs[cp_kl_id] + kl0;
        t.nb = kl1 - kl0;
        t.pa0 = bpcache->primitive_pairs_locs[cp_ij_id] + ij0 * cij->nprim_12;
        t.pb0 = bpcache->primitive_pairs_locs[cp_kl_id] + kl0 * ckl->nprim_12;
        t.nprim_a = cij->nprim_12;
        t.nprim_b = ckl->nprim_12;
        t.diag = cp_ij_id == cp_kl_id;
        t.skip_lower = 1;
        int err = bqc_launch_jk(cij->l_bra, cij->l_ket, ckl->l_bra, ckl->l_ket, args, t, 0, stream);
        if (err) return err;
    }
    return 0;
}

// ERI writer (cuobc/lib/gint/nr_fill_ao_ints.cu:493-551): every quartet of the
// class pair (cp_ij, cp_kl) whose bins satisfy ij_bin + kl_bin < nbins adds its
// Cartesian block (ij|kl) to eri at sum_n (ao_n - ao_offsets[n]) strides[n];
// all ij x kl pairs (no a >= b restriction, no 1/2 on identical pairs).
int GINTfill_int2e(BasisProdCache *bpcache, double *eri, int nao, int *strides, int *ao_offsets,
                   int *bins_locs_ij, int *bins_locs_kl, int nbins, int cp_ij_id, int cp_kl_id,
                   cudaStream_t stream) {
    if (eri == NULL || strides == NULL || ao_offsets == NULL) return 3;
    if (cp_ij_id < 0 || cp_kl_id < 0 || cp_ij_id >= bpcache->ncptype || cp_kl_id >= bpcache->ncptype)
        return 3;
    const ContractionProdType *cij = bpcache->cptype + cp_ij_id;
    const ContractionProdType *ckl = bpcache->cptype + cp_kl_id;
    if (cij->l_bra > BQC_LMAX || ckl->l_bra > BQC_LMAX) return 2;
    JKArgs args = make_args(bpcache, NULL, NULL, NULL, nao, 1);
    args.eri = eri;
    for (int n = 0; n < 4; n++) {
        args.eri_stride[n] = strides[n];
        args.eri_off[n] = ao_offsets[n];
    }
    for (int kl_bin = 0; kl_bin < nbins; kl_bin++) {
        int kl0 = bins_locs_kl[kl_bin], kl1 = bins_locs_kl[kl_bin + 1];
        if (kl1 <= kl0) continue;
        int ij0 = bins_locs_ij[0], ij1 = bins_locs_ij[nbins - kl_bin];
        if (ij1 <= ij0) continue;
        JKTask t;
        memset(&t, 0, sizeof(t));
        t.a0 = bpcache->bas_pairs_locs[cp_ij_id] + ij0;
        t.na = ij1 - ij0;
        t.b0 = bpcache->bas_pairs_locs[cp_kl_id] + kl0;
        t.nb = kl1 - kl0;
        t.pa0 = bpcache->primitive_pairs_locs[cp_ij_id] + ij0 * cij->nprim_12;
        t.pb0 = bpcache->primitive_pairs_locs[cp_kl_id] + kl0 * ckl->nprim_12;
        t.nprim_a = cij->nprim_12;
        t.nprim_b = ckl->nprim_12;
        int err = bqc_launch_jk(cij->l_bra, cij->l_ket, ckl->l_bra, ckl->l_ket, args, t, 0, stream);
        if (err) return err;
    }
    return 0;
}

// Tile rows of one class-pair task: row r (16 pairs of the a list, q sorted
// descending) keeps the columns whose first (largest) q_b satisfies
// q_a[16 r] q_b[16 c] dm_max >= tol; on a diagonal task also c <= r.
static int tile_rows(const double *qa, int na, const double *qb, int nb, double dm_max, double tol,
                     int diag, std::vector<int> &prefix) {
    int nta = (na + 15) / 16, ntb = (nb + 15) / 16;
    prefix.push_back(0);
    int base = (int)prefix.size() - 1;
    for (int r = 0; r < nta; r++) {
        double qr = qa[16 * r] * dm_max;
        int lo = 0, hi = ntb;   // count of leading columns with qb[16 c] * qr >= tol
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (qb[16 * mid] * qr >= tol) lo = mid + 1; else hi = mid;
        }
        int n = lo;
        if (diag && n > r + 1) n = r + 1;
        prefix.push_back(prefix.back() + n);
    }
    return prefix.back() - prefix[base];
}

// Launch (or, with count_dev, only count the surviving quartets of) every
// class pair, or the single class pair (only_ij, only_kl) when only_ij >= 0.
// Tile rows when the pairs of several independent molecules share the lists:
// tiles hold pairs of one molecule, grouped by molecule in increasing order and
// sorted by their first q within a molecule.  Row r may only meet the ket
// tiles of its own molecule, [c0, c1); col0 receives c0 per row.
static int tile_rows_mol(const double *qa, const int *ma, int na, const double *qb, const int *mb,
                         int nb, double dm_max, double tol, int diag, std::vector<int> &prefix,
                         std::vector<int> &col0) {
    int nta = (na + 15) / 16, ntb = (nb + 15) / 16;
    prefix.push_back(0);
    int base = (int)prefix.size() - 1;
    for (int r = 0; r < nta; r++) {
        const int m = ma[16 * r];
        int lo = 0, hi = ntb;   // first ket tile of molecule >= m
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (mb[16 * mid] < m) lo = mid + 1; else hi = mid;
        }
        const int c0 = lo;
        hi = ntb;               // first ket tile of molecule > m
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (mb[16 * mid] <= m) lo = mid + 1; else hi = mid;
        }
        const int c1 = lo;
        const double qr = qa[16 * r] * dm_max;
        lo = c0;
        hi = c1;
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (qb[16 * mid] * qr >= tol) lo = mid + 1; else hi = mid;
        }
        int n = lo - c0;
        if (diag && n > r - c0 + 1) n = r - c0 + 1;
        if (n < 0) n = 0;
        prefix.push_back(prefix.back() + n);
        col0.push_back(c0);
    }
    return prefix.back() - prefix[base];
}

static int build_jk_band(const BasisProdCache *bp, JKArgs args, const double *pair_q_host,
                         const int *pair_mol_host, double dm_max, int fp32, int only_ij,
                         int only_kl, unsigned long long *count_dev, cudaStream_t stream) {
    std::vector<JKTask> tasks;
    std::vector<int> shape;   // (li, lj, lk, ll) per task
    std::vector<int> prefix, col0;
    std::vector<size_t> prefix_off, col0_off;
    for (int cij = 0; cij < bp->ncptype; cij++) {
        const ContractionProdType *tij = bp->cptype + cij;
        if (tij->npairs == 0) continue;
        if (only_ij >= 0 && cij != only_ij) continue;
        for (int ckl = 0; ckl <= cij; ckl++) {
            const ContractionProdType *tkl = bp->cptype + ckl;
            if (tkl->npairs == 0) continue;
            if (only_kl >= 0 && ckl != only_kl) continue;
            if (tij->l_bra > BQC_LMAX || tkl->l_bra > BQC_LMAX) return 2;
            JKTask t;
            memset(&t, 0, sizeof(t));
            t.a0 = bp->bas_pairs_locs[cij];
            t.na = tij->npairs;
            t.b0 = bp->bas_pairs_locs[ckl];
            t.nb = tkl->npairs;
            t.pa0 = bp->primitive_pairs_locs[cij];
            t.pb0 = bp->primitive_pairs_locs[ckl];
            t.nprim_a = tij->nprim_12;
            t.nprim_b = tkl->nprim_12;
            t.diag = cij == ckl;
            t.skip_lower = 1;
            if (pair_q_host != nullptr) {
                size_t off = prefix.size(), coff = col0.size();
                int n;
                if (pair_mol_host != nullptr)
                    n = tile_rows_mol(pair_q_host + t.a0, pair_mol_host + t.a0, t.na,
                                      pair_q_host + t.b0, pair_mol_host + t.b0, t.nb, dm_max,
                                      args.tol, t.diag, prefix, col0);
                else
                    n = tile_rows(pair_q_host + t.a0, t.na, pair_q_host + t.b0, t.nb, dm_max,
                                  args.tol, t.diag, prefix);
                if (n == 0) {
                    prefix.resize(off);
                    col0.resize(coff);
                    continue;
                }
                t.nrows = (t.na + 15) / 16;
                t.ntiles = n;
                prefix_off.push_back(off);
                col0_off.push_back(coff);
            }
            tasks.push_back(t);
            shape.push_back(tij->l_bra);
            shape.push_back(tij->l_ket);
            shape.push_back(tkl->l_bra);
            shape.push_back(tkl->l_ket);
        }
    }
    int *d_prefix = nullptr;
    if (pair_q_host != nullptr && !prefix.empty()) {
        const size_t n_all = prefix.size() + col0.size();
        if (cudaMallocAsync((void **)&d_prefix, sizeof(int) * n_all, stream) != cudaSuccess)
            return 1;
        prefix.insert(prefix.end(), col0.begin(), col0.end());
        cudaMemcpyAsync(d_prefix, prefix.data(), sizeof(int) * n_all, cudaMemcpyHostToDevice,
                        stream);
    }
    const size_t col0_base = prefix.size() - col0.size();
    int err = 0;
    for (size_t i = 0; i < tasks.size() && !err; i++) {
        if (d_prefix) tasks[i].tile_prefix = d_prefix + prefix_off[i];
        if (d_prefix && pair_mol_host != nullptr) tasks[i].tile_col0 = d_prefix + col0_base + col0_off[i];
        if (count_dev != nullptr)
            err = bqc_launch_count(args, tasks[i], count_dev, stream);
        else
            err = bqc_launch_jk(shape[4 * i], shape[4 * i + 1], shape[4 * i + 2], shape[4 * i + 3],
                                args, tasks[i], fp32, stream);
    }
    if (d_prefix) cudaFreeAsync(d_prefix, stream);
    return err;
}

// Launch (or, with count_dev, only count the surviving quartets of) every
// class pair, or the single class pair (only_ij, only_kl) when only_ij >= 0.
// With fp32_below > tol the quartets split into two bands: bound >= fp32_below
// in FP64 and tol <= bound < fp32_below in FP32 (count_dev counts both).
static int build_jk_impl(const BasisProdCache *bp, const double *pair_q, const double *pair_q_host,
                         const int *pair_mol_host, const double *dm_cond, double dm_max,
                         double *vj, double *vk,
                         const double *dm, int nao, int n_dm, double tol, double fp32_below,
                         int *status_dev, int only_ij, int only_kl,
                         unsigned long long *count_dev, cudaStream_t stream) {
    JKArgs args = make_args(bp, vj, vk, dm, nao, n_dm);
    args.pair_q = pair_q;
    args.dm_cond = dm_cond;
    args.tol = tol;
    args.tol_hi = 0.;
    args.status = status_dev;
    if (dm_cond == nullptr) dm_max = 1.0;
    if (pair_q == nullptr || fp32_below <= tol)
        return build_jk_band(bp, args, pair_q_host, pair_mol_host, dm_max, 0, only_ij, only_kl,
                             count_dev, stream);
    JKArgs hi = args;
    hi.tol = fp32_below;
    int err = build_jk_band(bp, hi, pair_q_host, pair_mol_host, dm_max, 0, only_ij, only_kl,
                            count_dev, stream);
    if (err) return err;
    JKArgs lo = args;
    lo.tol_hi = fp32_below;
    return build_jk_band(bp, lo, pair_q_host, pair_mol_host, dm_max, 1, only_ij, only_kl,
                         count_dev, stream);
}

int BQCbuild_jk(const BasisProdCache *bp, const double *pair_q, const double *pair_q_host,
                const double *dm_cond, double dm_max, double *vj, double *vk, const double *dm,
                int nao, int n_dm, double tol, double fp32_below, int *status_dev,
                cudaStream_t stream) {
    return build_jk_impl(bp, pair_q, pair_q_host, nullptr, dm_cond, dm_max, vj, vk, dm, nao, n_dm, tol,
                         fp32_below, status_dev, -1, -1, nullptr, stream);
}

int BQCbuild_jk_mol(const BasisProdCache *bp, const double *pair_q, const double *pair_q_host,
                    const int *pair_mol_host, const double *dm_cond, double dm_max, double *vj,
                    double *vk, const double *dm, int nao, int n_dm, double tol, double fp32_below,
                    int *status_dev, cudaStream_t stream) {
    if (pair_q_host == nullptr || pair_mol_host == nullptr) return 1;
    return build_jk_impl(bp, pair_q, pair_q_host, pair_mol_host, dm_cond, dm_max, vj, vk, dm, nao,
                         n_dm, tol, fp32_below, status_dev, -1, -1, nullptr, stream);
}

int BQCbuild_jk_class(const BasisProdCache *bp, int cp_ij, int cp_kl, const double *pair_q,
                      const double *pair_q_host, const double *dm_cond, double dm_max, double *vj,
                      double *vk, const double *dm, int nao, int n_dm, double tol,
                      double fp32_below, int *status_dev, cudaStream_t stream) {
    if (cp_ij < 0 || cp_kl < 0 || cp_kl > cp_ij || cp_ij >= bp->ncptype) return 1;
    return build_jk_impl(bp, pair_q, pair_q_host, nullptr, dm_cond, dm_max, vj, vk, dm, nao, n_dm, tol,
                         fp32_below, status_dev, cp_ij, cp_kl, nullptr, stream);
}

int BQCcount_quartets(const BasisProdCache *bp, int cp_ij, int cp_kl, const double *pair_q,
                      const double *pair_q_host, const double *dm_cond, double dm_max, double tol,
                      unsigned long long *count_dev, cudaStream_t stream) {
    if (count_dev == nullptr) return 1;
    return build_jk_impl(bp, pair_q, pair_q_host, nullptr, dm_cond, dm_max, nullptr, nullptr, nullptr, 0, 0,
                         tol, 0., nullptr, cp_ij, cp_kl, count_dev, stream);
}

int BQCdm_cond(const double *dm, int n_dm, int nao, const int *ao_loc, int nbas, double *dm_cond,
               cudaStream_t stream) {
    return bqc_launch_dm_cond(dm, n_dm, nao, ao_loc, nbas, dm_cond, stream);
}

int BQCschwarz(const BasisProdCache *bp, int cp, double diag_fac, double *q_out,
               cudaStream_t stream) {
    const ContractionProdType *t = bp->cptype + cp;
    if (t->npairs == 0) return 0;
    if (t->l_bra > BQC_LMAX) return 2;
    JKArgs args = make_args(bp, NULL, NULL, NULL, 0, 0);
    return bqc_launch_schwarz(t->l_bra, t->l_ket, args, bp->bas_pairs_locs[cp], t->npairs,
                              bp->primitive_pairs_locs[cp], t->nprim_12, diag_fac, q_out, stream);
}

// ---------------------------------------------------------------------------
// J/K build that allocates nothing.
//
// Some callers cannot let the library allocate device memory: a host program
// that sizes its device memory once from a fixed arena and forbids any other
// allocation (so nothing can fragment or contend with its own pool), or one
// whose only device buffers are the inputs and outputs it passes in.
// BQCbuild_jk reserves stream-ordered scratch for its tile tables and expects
// the caller to provide the density-screening table; this variant needs
// neither.  Its only scratch, the per-shell-pair density maxima, lives in the
// file-scope array below (BQC_NOALLOC_MAX_NBAS^2 doubles = 2 MiB, held on
// every GPU that loads the library until the process exits), and it launches
// every quartet tile of every class pair (device screening only, no
// host-side tile pruning), which suits the small systems that fit the limit.
#define BQC_NOALLOC_MAX_NBAS 512
static __device__ __align__(256) double g_noalloc_dm_cond[BQC_NOALLOC_MAX_NBAS * BQC_NOALLOC_MAX_NBAS];

// Device address of g_noalloc_dm_cond on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device (with that device current) and cached.
static double *noalloc_scratch() {
    static double *addr[128] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return nullptr;
    if (addr[dev] == nullptr) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_dm_cond) != cudaSuccess) return nullptr;
        addr[dev] = static_cast<double *>(p);
    }
    return addr[dev];
}

int BQCbuild_jk_noalloc(const BasisProdCache *bp, const double *pair_q, double *vj, double *vk,
                        const double *dm, int nao, int n_dm, double tol, cudaStream_t stream) {
    if (bp->nbas > BQC_NOALLOC_MAX_NBAS) {
        fprintf(stderr, "BQCbuild_jk_noalloc: %d shells exceed the limit of %d\n", bp->nbas,
                BQC_NOALLOC_MAX_NBAS);
        return 3;
    }
    // without Schwarz factors the kernels would screen nothing at all
    if (pair_q == nullptr) return 3;
    double *dm_cond = noalloc_scratch();
    if (dm_cond == nullptr) return 1;
    // every entry of the nbas x nbas table is overwritten before it is read
    int err = bqc_launch_dm_cond(dm, n_dm, nao, bp->ao_loc, bp->nbas, dm_cond, stream);
    if (err) return err;
    return build_jk_impl(bp, pair_q, nullptr, nullptr, dm_cond, 1.0, vj, vk, dm, nao, n_dm, tol, 0.,
                         nullptr, -1, -1, nullptr, stream);
}

const char *BQCversion(void) { return "byteqc_b200 0.1 sm_100a"; }

}  // extern "C"
