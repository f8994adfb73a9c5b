// hzb_sa.cu -- smoothed aggregation: the setup pieces of amg_setup_sa
// (amg_setup_ua.c:76 -> amg_setup_smoothP_smoothR, :1461-1700) beyond the
// aggregation it shares with the unsmoothed path.
//
//   smooth_aggregation_p (amg_setup_ua.c:472-560), with the default filter:
//     the strength graph N (A's strongly coupled entries, diagonal kept)
//     takes each row's dropped weight on its diagonal,
//     N_ii += sum_{j != i} A_ij - sum_{j != i} N_ij, then the damped Jacobi
//     smoother S = I - omega D_N^{-1} N (omega = tentative_smooth; a diagonal
//     below 1e-6 in magnitude counts as 1), and P = S P_tent through dcsr_mxm
//     (sparse.c:1832-1907): row i of P lists the aggregates of row i's
//     neighbours in first-encounter order, each value the sum from 0 of the
//     row's S entries into that aggregate, in CSR order.  Without the filter
//     S is built the same way from A itself;
//   R = P^T by dcsr_trans (sparse.c:770-862): rows list fine rows ascending;
//   A_c = R A P by dcsr_rap (sparse.c:2401-2520): coarse row ic reserves
//     slot 0 for column ic (value 0.0, later products added), then every
//     (R entry, A entry, P entry) in that nested CSR order adds
//     (r * a) * p to its column's slot, a new column taking the next slot
//     and the product as its value.
//
// Each coarse row of the Galerkin product is one warp walking the
// reference's traversal in order, 32 entries of a P row at a time (their
// columns are distinct), so every sum is formed in the same order and the
// result is bit for bit the reference's; the column -> slot map is a
// per-warp open-addressing table in global scratch (a persistent grid
// reuses it row after row).  The smoother and P are row-local kernels.
#include "hzb_setup.cuh"
#include <algorithm>

namespace hzb {

namespace {
constexpr int RAP_THREADS = 128;
// A warp's table holds cap = 2^lg hash positions: keys and slots by
// position, then the positions in slot order (to clear only what a row
// used); at most cap / 2 columns go in.

// With the filter, N_ii += (sum of A's off-diagonal row) - (sum of N's
// off-diagonal row); then N becomes S = I - omega D^{-1} N in place (d: N's
// first diagonal).  Without it N is a copy of A.
__global__ void k_sa_smoother(int m, const int *__restrict__ aia, const int *__restrict__ aja,
                              const double *__restrict__ aval, const int *__restrict__ nia,
                              const int *__restrict__ nja, double *__restrict__ nval,
                              double omega, bool filter) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (filter) {
            double rsa = 0.0, rsn = 0.0;
            for (int k = aia[i]; k < aia[i + 1]; ++k)
                if (aja[k] != i) rsa += aval[k];
            for (int k = nia[i]; k < nia[i + 1]; ++k)
                if (nja[k] != i) rsn += nval[k];
            for (int k = nia[i]; k < nia[i + 1]; ++k)
                if (nja[k] == i) nval[k] += rsa - rsn;
        }
        double d = 0.0;
        for (int k = nia[i]; k < nia[i + 1]; ++k)
            if (nja[k] == i) { d = nval[k]; break; }
        if (fabs(d) < 1e-6) d = 1.0;
        for (int k = nia[i]; k < nia[i + 1]; ++k) {
            const double v = nval[k];
            nval[k] = nja[k] == i ? 1 - omega * v / d : -omega * v / d;
        }
    }
}

// entries of row i of P = S P_tent: the distinct aggregates of the row's
// columns (rows outside any aggregate contribute nothing)
__global__ void k_sa_p_count(int m, const int *__restrict__ sia, const int *__restrict__ sja,
                             const int *__restrict__ agg, int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int c = 0;
        for (int k = sia[i]; k < sia[i + 1]; ++k) {
            const int a = agg[sja[k]];
            if (a < 0) continue;
            bool seen = false;
            for (int q = sia[i]; q < k && !seen; ++q) seen = agg[sja[q]] == a;
            c += !seen;
        }
        cnt[i] = c;
    }
}

// columns in first-encounter order; value = 0 + the row's S entries into the
// aggregate, added in CSR order
__global__ void k_sa_p_fill(int m, const int *__restrict__ sia, const int *__restrict__ sja,
                            const double *__restrict__ sval, const int *__restrict__ agg,
                            const int *__restrict__ pia, int *__restrict__ pja,
                            double *__restrict__ pval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const int p0 = pia[i];
        int c = 0;
        for (int k = sia[i]; k < sia[i + 1]; ++k) {
            const int a = agg[sja[k]];
            if (a < 0) continue;
            int slot = -1;
            for (int q = 0; q < c; ++q)
                if (pja[p0 + q] == a) { slot = q; break; }
            if (slot < 0) {
                slot = c++;
                pja[p0 + slot] = a;
                pval[p0 + slot] = 0.0;
            }
            pval[p0 + slot] += sval[k] * 1.0;
        }
    }
}

// rectangular transpose: counts per column, then rows in ascending order
__global__ void k_tr_count_rect(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = ia[i]; k < ia[i + 1]; ++k) atomicAdd(cnt + ja[k], 1);
}
__global__ void k_tr_fill_rect(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                               const double *__restrict__ val, const int *__restrict__ tia,
                               int *fill, int *tja, double *tval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            const int c = ja[k];
            const int pos = tia[c] + atomicAdd(fill + c, 1);
            tja[pos] = i;
            tval[pos] = val[k];
        }
}
// each transposed row sorted by fine row (insertion sort; the rows are short)
__global__ void k_tr_sort_rect(int nc, const int *__restrict__ tia, int *tja, double *tval) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const int b = tia[c], e = tia[c + 1];
        for (int k = b + 1; k < e; ++k) {
            const int j = tja[k];
            const double v = tval[k];
            int q = k - 1;
            while (q >= b && tja[q] > j) {
                tja[q + 1] = tja[q];
                tval[q + 1] = tval[q];
                --q;
            }
            tja[q + 1] = j;
            tval[q + 1] = v;
        }
    }
}

__device__ __forceinline__ unsigned rap_hash(int c, int lg) {
    return ((unsigned)c * 2654435761u) >> (32 - lg);
}

// One coarse row per warp (persistent grid; each warp's table is reused row
// after row).  The warp walks (R entry, A entry) pairs in order; its lanes
// take 32 consecutive entries of the P row at a time.  The columns of one P
// row are distinct, so within a batch every lane owns its own column: each
// column's sum still receives its products in the reference's traversal
// order, and new columns take slots in entry order (ballot + prefix count).
// FILL = false counts the row's distinct columns; FILL = true writes them in
// slot order with their sums.  err receives 1 when a row has more distinct
// columns than half the table.
template <bool FILL>
__global__ void __launch_bounds__(RAP_THREADS)
k_rap_general(int nc, const int *__restrict__ ria, const int *__restrict__ rja,
              const double *__restrict__ rval, const int *__restrict__ aia,
              const int *__restrict__ aja, const double *__restrict__ aval,
              const int *__restrict__ pia, const int *__restrict__ pja,
              const double *__restrict__ pval, int lg, int *table, int *cnt, const int *cia,
              int *cja, double *cval, int *err) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int cap = 1 << lg;
    int *keys = table + (size_t)warp * 3 * cap, *slots = keys + cap, *used = slots + cap;
    for (int h = lane; h < cap; h += 32) keys[h] = -1;
    __syncwarp();
    for (int ic = warp; ic < nc; ic += nwarps) {
        const int base = FILL ? cia[ic] : 0;
        if (lane == 0) {   // slot 0: the diagonal, value 0.0
            const unsigned h = rap_hash(ic, lg);   // the table is empty here
            keys[h] = ic;
            slots[h] = 0;
            used[0] = (int)h;
            if (FILL) {
                cja[base] = ic;
                cval[base] = 0.0;
            }
        }
        int count = 1;
        bool full = false;
        __syncwarp();
        for (int j1 = ria[ic]; j1 < ria[ic + 1] && !full; ++j1) {
            const int i1 = rja[j1];
            const double r = FILL ? rval[j1] : 0.0;
            for (int j2 = aia[i1]; j2 < aia[i1 + 1] && !full; ++j2) {
                const int i2 = aja[j2];
                const double ra = FILL ? __dmul_rn(r, aval[j2]) : 0.0;
                const int p1 = pia[i2 + 1];
                for (int jb = pia[i2]; jb < p1 && !full; jb += 32) {
                    const int j3 = jb + lane;
                    const bool act = j3 < p1;
                    const int c = act ? pja[j3] : -1;
                    int h = -1;
                    bool fresh = false, lost = false;
                    if (act) {
                        unsigned q = rap_hash(c, lg);
                        lost = true;
                        for (int probe = 0; probe < cap; ++probe, q = (q + 1) & (cap - 1)) {
                            const int old = atomicCAS(keys + q, -1, c);
                            if (old == -1 || old == c) {
                                fresh = old == -1;
                                h = (int)q;
                                lost = false;
                                break;
                            }
                        }
                    }
                    const unsigned nb = __ballot_sync(0xffffffffu, fresh);
                    const int added = __popc(nb);
                    if (__any_sync(0xffffffffu, lost) || count + added > cap / 2) {
                        full = true;   // every lane sees the same
                        break;
                    }
                    int slot = -1;
                    if (fresh) {
                        slot = count + __popc(nb & ((1u << lane) - 1));
                        slots[h] = slot;
                        used[slot] = h;
                    } else if (act) {
                        slot = slots[h];
                    }
                    count += added;
                    if (FILL && act) {
                        const double v = __dmul_rn(ra, pval[j3]);
                        if (fresh) {
                            cja[base + slot] = c;
                            cval[base + slot] = v;
                        } else {
                            cval[base + slot] = __dadd_rn(cval[base + slot], v);
                        }
                    }
                    __syncwarp();
                }
            }
        }
        if (full && lane == 0) *err = 1;
        if (!FILL && lane == 0) cnt[ic] = count;
        __syncwarp();
        for (int q = lane; q < count && q < cap / 2; q += 32) keys[used[q]] = -1;
        __syncwarp();
    }
}
}  // namespace

int sa_prolongation(const DCsr<double> &A, const int *nia, const int *nja, double *nval,
                    int nc, const int *agg, double omega, bool filter, int **pia_out,
                    int **pja_out, double **pval_out, int *pnnz, cudaStream_t s) {
    const int m = A.n;
    const int g = grid_for(m);
    int *cnt = nullptr, *tmp = nullptr, *pia = nullptr, *pja = nullptr;
    double *pval = nullptr;
    int rc = SUCCESS, nnz = 0;
    (void)nc;
    k_sa_smoother<<<g, 256, 0, s>>>(m, A.ia, A.ja, A.val, nia, nja, nval, omega, filter);
    count_launch();
    if ((rc = dalloc(&cnt, m)) || (rc = dalloc(&tmp, scan_tmp_size(m + 1))) ||
        (rc = dalloc(&pia, m + 1)))
        goto fail;
    k_sa_p_count<<<g, 256, 0, s>>>(m, nia, nja, agg, cnt);
    count_launch();
    if ((rc = scan_exclusive(cnt, pia, m, tmp, s))) goto fail;
    HZB_CUDA(cudaMemcpyAsync(&nnz, pia + m, sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    if ((rc = dalloc(&pja, nnz > 0 ? nnz : 1)) || (rc = dalloc(&pval, nnz > 0 ? nnz : 1)))
        goto fail;
    k_sa_p_fill<<<g, 256, 0, s>>>(m, nia, nja, nval, agg, pia, pja, pval);
    count_launch();
    HZB_LAUNCH_CHECK();
    dfree(cnt);
    dfree(tmp);
    *pia_out = pia; *pja_out = pja; *pval_out = pval; *pnnz = nnz;
    return SUCCESS;
fail:
    dfree(cnt); dfree(tmp); dfree(pia); dfree(pja); dfree(pval);
    return rc;
}

int transpose_rect(int n, int ncols, int nnz, const int *ia, const int *ja, const double *val,
                   int **tia_out, int **tja_out, double **tval_out, cudaStream_t s) {
    int *tia = nullptr, *tja = nullptr, *cnt = nullptr, *tmp = nullptr;
    double *tval = nullptr;
    int rc = SUCCESS;
    if ((rc = dalloc(&tia, ncols + 1)) || (rc = dalloc(&tja, nnz > 0 ? nnz : 1)) ||
        (rc = dalloc(&tval, nnz > 0 ? nnz : 1)) || (rc = dalloc(&cnt, ncols)) ||
        (rc = dalloc(&tmp, scan_tmp_size(ncols + 1))))
        goto fail;
    HZB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ncols, s));
    k_tr_count_rect<<<grid_for(n), 256, 0, s>>>(n, ia, ja, cnt);
    count_launch();
    if ((rc = scan_exclusive(cnt, tia, ncols, tmp, s))) goto fail;
    HZB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ncols, s));
    k_tr_fill_rect<<<grid_for(n), 256, 0, s>>>(n, ia, ja, val, tia, cnt, tja, tval);
    k_tr_sort_rect<<<grid_for(ncols), 256, 0, s>>>(ncols, tia, tja, tval);
    count_launch(2);
    HZB_LAUNCH_CHECK();
    dfree(cnt);
    dfree(tmp);
    *tia_out = tia; *tja_out = tja; *tval_out = tval;
    return SUCCESS;
fail:
    dfree(tia); dfree(tja); dfree(tval); dfree(cnt); dfree(tmp);
    return rc;
}

int rap_general(int nc, const int *ria, const int *rja, const double *rval,
                const DCsr<double> &A, const int *pia, const int *pja, const double *pval,
                int **cia_out, int **cja_out, double **cval_out, int *cnnz, cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // table size: every column of a small coarse level fits at once; larger
    // levels start at 2^11 positions and grow when a row overflows
    int lg_all = 5;
    while ((1 << lg_all) < 2 * nc) ++lg_all;
    int lg = std::min(lg_all, 11);
    int *table = nullptr, *cnt = nullptr, *tmp = nullptr, *err = nullptr, *cia = nullptr,
        *cja = nullptr;
    double *cval = nullptr;
    int rc = SUCCESS, nnz = 0, herr = 0, blocks = 1;
    if ((rc = dalloc(&cnt, nc)) || (rc = dalloc(&tmp, scan_tmp_size(nc + 1))) ||
        (rc = dalloc(&err, 1)) || (rc = dalloc(&cia, nc + 1)))
        goto fail;
    for (;;) {
        // a persistent grid of warps whose tables take at most about 1 GB
        const int wpb = RAP_THREADS / 32;
        const size_t per_warp = (size_t)3 * ((size_t)1 << lg) * sizeof(int);
        const size_t max_warps = std::max<size_t>(wpb, ((size_t)1 << 30) / per_warp);
        blocks = (int)std::max<size_t>(1, std::min<size_t>(
                     {(size_t)sms * 8, max_warps / wpb, (size_t)(nc + wpb - 1) / wpb}));
        if ((rc = dalloc(&table, (size_t)blocks * wpb * 3 * ((size_t)1 << lg)))) goto fail;
        HZB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
        k_rap_general<false><<<blocks, RAP_THREADS, 0, s>>>(nc, ria, rja, rval, A.ia, A.ja,
                                                             A.val, pia, pja, pval, lg, table,
                                                             cnt, nullptr, nullptr, nullptr, err);
        count_launch();
        HZB_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        HZB_CUDA(cudaStreamSynchronize(s));
        if (!herr) break;
        dfree(table);
        if (lg >= lg_all) {   // cannot happen: a row has at most nc columns
            set_error_msg("Galerkin product table overflow");
            rc = ERROR_MISC;
            goto fail;
        }
        lg = std::min(lg + 2, lg_all);
    }
    if ((rc = scan_exclusive(cnt, cia, nc, tmp, s))) goto fail;
    HZB_CUDA(cudaMemcpyAsync(&nnz, cia + nc, sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    if ((rc = dalloc(&cja, nnz)) || (rc = dalloc(&cval, nnz))) goto fail;
    k_rap_general<true><<<blocks, RAP_THREADS, 0, s>>>(nc, ria, rja, rval, A.ia, A.ja, A.val,
                                                        pia, pja, pval, lg, table, nullptr, cia,
                                                        cja, cval, err);
    count_launch();
    HZB_LAUNCH_CHECK();
    dfree(table); dfree(cnt); dfree(tmp); dfree(err);
    *cia_out = cia; *cja_out = cja; *cval_out = cval; *cnnz = nnz;
    return SUCCESS;
fail:
    dfree(table); dfree(cnt); dfree(tmp); dfree(err); dfree(cia); dfree(cja); dfree(cval);
    return rc;
}

}  // namespace hzb
