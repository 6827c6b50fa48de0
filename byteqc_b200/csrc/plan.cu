// J/K builds scheduled on the device (no reference counterpart; the
// reference prunes on the host, cuobc/scf/hf.py:111-166, and launches one
// kernel per kl bin, cuobc/lib/gvhf/nr_jk_driver.cu:252-280).
//
// A plan holds, per basis-product cache, everything of a J/K build that does
// not depend on the density: the class-pair task list, the Schwarz factor of
// the first (largest) pair of every 16-pair tile, and device scratch for the
// schedule.  A build then runs entirely on the stream without a host
// round trip or an allocation:
//
//   dm_max   = max over the density-block table (one reduction kernel);
//   counts   : per tile row r of every task, the number of leading column
//              tiles c with q_row[r] q_col[c] dm_max >= tol (the tiles are
//              sorted by their first q, so a binary search), at most r + 1 on
//              a diagonal task; for batched molecules only the row's own
//              molecule's columns count;
//   prefix   : per task, the exclusive scan of its row counts and the task's
//              tile total;
//   launches : one per task and precision band, a fixed grid of CTAs that
//              strides over the task's [0, total) tiles (JKTask::ntiles_dev).
//
// Every launch of a build has the same shape each time, so a build can be
// captured in a CUDA graph and replayed.
#include <algorithm>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include "bqc.h"

namespace {

constexpr int TILE = 16;

// density-independent description of one task for the schedule kernels
struct SchedTask {
    int row_off;   // first global row of the task (rows over the a list)
    int nrows, ncols;
    int a_tile0;   // first tile of the a list in the tile arrays
    int b_tile0;
    int diag;
    int pfx_off;   // first prefix entry of the task (nrows + 1 entries)
};

struct TaskHost {
    JKTask base;
    int li, lj, lk, ll;
    int max_tiles;
    int row_off, pfx_off;   // the task's rows and prefix entries in the schedule
};

// Largest n in [lo, hi] such that q[c] * qr >= tol for all c < n (q
// descending): the number of leading columns that reach tol.
__device__ __forceinline__ int leading_cols(const double *__restrict__ q, int lo, int hi, double qr,
                                            double tol) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(q + mid) * qr >= tol) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// first index in [lo, hi) whose molecule is >= m (molecules ascending)
__device__ __forceinline__ int first_mol(const int *__restrict__ mol, int lo, int hi, int m) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(mol + mid) < m) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// max over the non-negative entries of x (as ordered 64-bit patterns)
__global__ void max_kernel(const double *__restrict__ x, size_t n, unsigned long long *out) {
    double m = 0.;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = fmax(m, __ldg(x + i));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// per global row: the column counts of the two precision bands (band 1 only
// when tol1 > 0) and, for batched molecules, the row's first column
__global__ void count_rows_kernel(const SchedTask *__restrict__ tasks, const int *__restrict__ row_task,
                                  int nrows_all, const double *__restrict__ tile_q,
                                  const int *__restrict__ tile_mol, const unsigned long long *dm_max_bits,
                                  double tol0, double tol1, int *__restrict__ cnt0,
                                  int *__restrict__ cnt1, int *__restrict__ col0) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nrows_all) return;
    const SchedTask t = tasks[__ldg(row_task + g)];
    const int r = g - t.row_off;
    const double dm_max = __longlong_as_double((long long)*dm_max_bits);
    const double qr = __ldg(tile_q + t.a_tile0 + r) * dm_max;
    const double *qb = tile_q + t.b_tile0;
    int c0 = 0, c1 = t.ncols;
    if (tile_mol != nullptr) {
        const int m = __ldg(tile_mol + t.a_tile0 + r);
        const int *mb = tile_mol + t.b_tile0;
        c0 = first_mol(mb, 0, t.ncols, m);
        c1 = first_mol(mb, c0, t.ncols, m + 1);
        col0[g] = c0;
    }
    const int lim = t.diag ? r - c0 + 1 : c1 - c0;
    int n0 = leading_cols(qb, c0, c1, qr, tol0) - c0;
    cnt0[g] = max(0, min(n0, lim));
    if (tol1 > 0.) {
        int n1 = leading_cols(qb, c0, c1, qr, tol1) - c0;
        cnt1[g] = max(0, min(n1, lim));
    }
}

// one CTA per task: exclusive scan of its row counts into the prefix and the
// task's total
__global__ void scan_rows_kernel(const SchedTask *__restrict__ tasks, const int *__restrict__ cnt,
                                 int *__restrict__ prefix, int *__restrict__ ntiles) {
    const SchedTask t = tasks[blockIdx.x];
    __shared__ int s_warp[32];
    __shared__ int s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < t.nrows; base += blockDim.x) {
        const int r = base + threadIdx.x;
        const int v = r < t.nrows ? __ldg(cnt + t.row_off + r) : 0;
        int x = v;   // inclusive scan within the warp
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_warp[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = lane < nw ? s_warp[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < nw) s_warp[lane] = w;
        }
        __syncthreads();
        const int incl = x + (warp > 0 ? s_warp[warp - 1] : 0) + s_carry;
        if (r < t.nrows) prefix[t.pfx_off + r + 1] = incl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        prefix[t.pfx_off] = 0;
        ntiles[blockIdx.x] = s_carry;
    }
}

}  // namespace

struct BQCPlan {
    const BasisProdCache *bp;
    int device;
    int nsm;
    std::vector<TaskHost> tasks;
    int ntasks, nrows_all, npfx;
    // device
    SchedTask *d_tasks;
    int *d_row_task;
    double *d_tile_q;
    int *d_tile_mol;   // NULL unless batched molecules
    int *d_cnt;        // 2 x nrows_all
    int *d_col0;       // nrows_all (batched molecules)
    int *d_prefix;     // 2 x npfx
    int *d_ntiles;     // 2 x ntasks
    unsigned long long *d_dm_max;
};

extern "C" {

int BQCplan_create(const BasisProdCache *bp, const double *pair_q_host, const int *pair_mol_host,
                   BQCPlan **out) {
    if (bp == nullptr || pair_q_host == nullptr || out == nullptr) return 3;
    *out = nullptr;
    BQCPlan *p = new BQCPlan();   // value-initialised: every pointer NULL
    p->bp = bp;
    if (cudaGetDevice(&p->device) != cudaSuccess) { delete p; return 1; }
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess) {
        delete p;
        return 1;
    }
    p->nsm = nsm;
    // tiles of every class: q of the first pair (the tile's largest)
    std::vector<int> class_tile0(bp->ncptype + 1, 0);
    for (int c = 0; c < bp->ncptype; c++)
        class_tile0[c + 1] = class_tile0[c] + (bp->cptype[c].npairs + TILE - 1) / TILE;
    const int ntile_all = class_tile0[bp->ncptype];
    std::vector<double> tile_q(std::max(ntile_all, 1));
    std::vector<int> tile_mol(pair_mol_host ? std::max(ntile_all, 1) : 0);
    for (int c = 0; c < bp->ncptype; c++) {
        const int p0 = bp->bas_pairs_locs[c], np = bp->cptype[c].npairs;
        for (int t = 0; t * TILE < np; t++) {
            tile_q[class_tile0[c] + t] = pair_q_host[p0 + t * TILE];
            if (pair_mol_host) tile_mol[class_tile0[c] + t] = pair_mol_host[p0 + t * TILE];
        }
    }
    std::vector<SchedTask> st;
    std::vector<int> row_task;
    int pfx = 0;
    for (int cij = 0; cij < bp->ncptype; cij++) {
        const ContractionProdType *tij = bp->cptype + cij;
        if (tij->npairs == 0) continue;
        for (int ckl = 0; ckl <= cij; ckl++) {
            const ContractionProdType *tkl = bp->cptype + ckl;
            if (tkl->npairs == 0) continue;
            if (tij->l_bra > BQC_LMAX || tkl->l_bra > BQC_LMAX) { delete p; return 2; }
            TaskHost th;
            memset(&th, 0, sizeof(th));
            JKTask &t = th.base;
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
            const int nrows = (t.na + TILE - 1) / TILE, ncols = (t.nb + TILE - 1) / TILE;
            t.nrows = nrows;
            th.li = tij->l_bra;
            th.lj = tij->l_ket;
            th.lk = tkl->l_bra;
            th.ll = tkl->l_ket;
            th.max_tiles = t.diag ? nrows * (nrows + 1) / 2 : nrows * ncols;
            SchedTask s;
            s.row_off = (int)row_task.size();
            s.nrows = nrows;
            s.ncols = ncols;
            s.a_tile0 = class_tile0[cij];
            s.b_tile0 = class_tile0[ckl];
            s.diag = t.diag;
            s.pfx_off = pfx;
            th.row_off = s.row_off;
            th.pfx_off = pfx;
            pfx += nrows + 1;
            for (int r = 0; r < nrows; r++) row_task.push_back((int)st.size());
            st.push_back(s);
            p->tasks.push_back(th);
        }
    }
    p->ntasks = (int)st.size();
    p->nrows_all = (int)row_task.size();
    p->npfx = pfx;
    const size_t nt = std::max(p->ntasks, 1), nr = std::max(p->nrows_all, 1), np_ = std::max(pfx, 1);
    bool ok = cudaMalloc(&p->d_tasks, sizeof(SchedTask) * nt) == cudaSuccess &&
              cudaMalloc(&p->d_row_task, sizeof(int) * nr) == cudaSuccess &&
              cudaMalloc(&p->d_tile_q, sizeof(double) * tile_q.size()) == cudaSuccess &&
              cudaMalloc(&p->d_cnt, sizeof(int) * 2 * nr) == cudaSuccess &&
              cudaMalloc(&p->d_col0, sizeof(int) * nr) == cudaSuccess &&
              cudaMalloc(&p->d_prefix, sizeof(int) * 2 * np_) == cudaSuccess &&
              cudaMalloc(&p->d_ntiles, sizeof(int) * 2 * nt) == cudaSuccess &&
              cudaMalloc(&p->d_dm_max, sizeof(unsigned long long)) == cudaSuccess;
    if (ok && pair_mol_host) ok = cudaMalloc(&p->d_tile_mol, sizeof(int) * tile_mol.size()) == cudaSuccess;
    if (ok && p->ntasks > 0)
        ok = cudaMemcpy(p->d_tasks, st.data(), sizeof(SchedTask) * st.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(p->d_row_task, row_task.data(), sizeof(int) * row_task.size(),
                        cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok)
        ok = cudaMemcpy(p->d_tile_q, tile_q.data(), sizeof(double) * tile_q.size(), cudaMemcpyHostToDevice) ==
             cudaSuccess;
    if (ok && pair_mol_host)
        ok = cudaMemcpy(p->d_tile_mol, tile_mol.data(), sizeof(int) * tile_mol.size(),
                        cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        BQCplan_destroy(p);
        return 1;
    }
    *out = p;
    return 0;
}

void BQCplan_destroy(BQCPlan *p) {
    if (p == nullptr) return;
    cudaFree(p->d_tasks);
    cudaFree(p->d_row_task);
    cudaFree(p->d_tile_q);
    cudaFree(p->d_tile_mol);
    cudaFree(p->d_cnt);
    cudaFree(p->d_col0);
    cudaFree(p->d_prefix);
    cudaFree(p->d_ntiles);
    cudaFree(p->d_dm_max);
    delete p;
}

int BQCbuild_jk_plan(const BQCPlan *p, const double *pair_q, const double *dm_cond, double *vj,
                     double *vk, const double *dm, int nao, int n_dm, double tol, double fp32_below,
                     cudaStream_t stream) {
    if (p == nullptr || pair_q == nullptr || dm_cond == nullptr || dm == nullptr) return 3;
    if (p->ntasks == 0) return 0;
    const BasisProdCache *bp = p->bp;
    const bool two = fp32_below > tol;
    // 1. dm_max on the device
    if (cudaMemsetAsync(p->d_dm_max, 0, sizeof(unsigned long long), stream) != cudaSuccess) return 1;
    const size_t nn = (size_t)bp->nbas * bp->nbas;
    bqc_count_launch(3);
    max_kernel<<<std::min<size_t>(1024, (nn + 255) / 256), 256, 0, stream>>>(dm_cond, nn, p->d_dm_max);
    // 2. column counts per row (band 0: FP64, bound >= fp32_below when two
    //    bands, else >= tol; band 1: FP32, bound >= tol) and their scans
    int *cnt0 = p->d_cnt, *cnt1 = p->d_cnt + std::max(p->nrows_all, 1);
    count_rows_kernel<<<(p->nrows_all + 255) / 256, 256, 0, stream>>>(
        p->d_tasks, p->d_row_task, p->nrows_all, p->d_tile_q, p->d_tile_mol, p->d_dm_max,
        two ? fp32_below : tol, two ? tol : 0., cnt0, cnt1, p->d_col0);
    int *pfx0 = p->d_prefix, *pfx1 = p->d_prefix + std::max(p->npfx, 1);
    int *nt0 = p->d_ntiles, *nt1 = p->d_ntiles + std::max(p->ntasks, 1);
    scan_rows_kernel<<<p->ntasks, 1024, 0, stream>>>(p->d_tasks, cnt0, pfx0, nt0);
    if (two) {
        bqc_count_launch(1);
        scan_rows_kernel<<<p->ntasks, 1024, 0, stream>>>(p->d_tasks, cnt1, pfx1, nt1);
    }
    if (cudaGetLastError() != cudaSuccess) return 1;
    // 3. the class kernels, persistent over the device tile counts
    JKArgs args;
    memset(&args, 0, sizeof(args));
    args.pair_bra = bp->bas_pair2bra;
    args.pair_ket = bp->bas_pair2ket;
    args.a12 = bp->a12;
    args.e12 = bp->e12;
    args.x12 = bp->x12;
    args.y12 = bp->y12;
    args.z12 = bp->z12;
    args.bas_x = bp->bas_coords;
    args.bas_y = bp->bas_coords + bp->nbas;
    args.bas_z = bp->bas_coords + 2 * bp->nbas;
    args.ao_loc = bp->ao_loc;
    args.pair_q = pair_q;
    args.dm_cond = dm_cond;
    args.dm = dm;
    args.vj = vj;
    args.vk = vk;
    args.nao = nao;
    args.nbas = bp->nbas;
    args.n_dm = n_dm;
    args.rys = bqc_rys_table();
    args.rys_lm = bqc_rys_table_lm();
    for (int band = 0; band < (two ? 2 : 1); band++) {
        JKArgs a = args;
        a.tol = band == 0 ? (two ? fp32_below : tol) : tol;
        a.tol_hi = band == 0 ? 0. : fp32_below;
        const int *pfx = band == 0 ? pfx0 : pfx1;
        const int *nt = band == 0 ? nt0 : nt1;
        for (int i = 0; i < p->ntasks; i++) {
            const TaskHost &th = p->tasks[i];
            JKTask t = th.base;
            t.tile_prefix = pfx + th.pfx_off;
            t.tile_col0 = p->d_tile_mol ? p->d_col0 + th.row_off : nullptr;
            t.ntiles = th.max_tiles;
            t.ntiles_dev = nt + i;
            t.nsm = p->nsm;
            int err = bqc_launch_jk(th.li, th.lj, th.lk, th.ll, a, t, band == 1, stream);
            if (err) return err;
        }
    }
    return 0;
}

}  // extern "C"
