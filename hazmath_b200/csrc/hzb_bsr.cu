// hzb_bsr.cu -- UA-AMG for block (BSR) matrices: amg_setup_ua_bsr
// (amg_setup_ua.c:145 -> amg_setup_unsmoothP_unsmoothR_bsr, :2183-2425),
// mgcycle_bsr (mgcycle.c:952-1160) and precond_dbsr_amg (precond.c:1311-1335),
// behind linear_solver_dbsr_krylov_amg (itsolver.c:2104-2190).
//
// Setup, per level while the level has more than max(coarse_dof, 50) block
// rows: the inverses of the diagonal blocks (dbsr_getdiaginv, sparse.c:6122,
// Gauss-Jordan as ddense_inv_inplace, dense.c:1266); the condensed scalar
// matrix (condenseBSRLinf, sparse.c:6223: each block's max row sum of |a|,
// negated off the diagonal, entries <= 1e-8 dropped) aggregated by heavy
// edge matching or VMB as aggregation_type says; the boolean P (identity blocks, form_boolean_p_bsr); and
// A_c = R A P by dbsr_rap (sparse.c:5840-5980): with identity blocks every
// coarse block is the sum of A's blocks in the traversal order (R row, A
// row), the diagonal block first (from zero), new blocks copied.  The
// threshold does not adapt on this path.
//
// Cycle: block Jacobi, or block Gauss-Seidel ascending before and descending
// after the coarse correction (SGS: both), each block row
// x_I = D_I^{-1} (b_I - sum_{J != I} A_IJ x_J) in the reference's element
// order, Gauss-Seidel on level schedules of the block pattern; both
// smoothings take presmooth_iter sweeps (mgcycle_bsr uses that count after
// the coarse correction too).  Residuals, transfers and the Krylov method
// run on the level's scalar expansion (row I nb + r lists block columns in
// block order, components in order); the boolean transfers are the scalar
// aggregate maps agg_s[I nb + r] = agg[I] nb + r.  precond_dbsr_amg rebuilds
// its cycle parameters from param_amg_init without the coarse solver, so
// the coarsest level is always solved by GMRES(25) to 1e-6 (at most
// min(n^2, 200) steps) from zero, as here.
#include "hzb_solver.cuh"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>
#include <vector>

namespace hzb {

namespace {
constexpr int BSR_MAXNB = 8;   // largest block size the kernels hold in registers

// inverse of the diagonal block of every block row (the last diagonal block
// of the row, as dbsr_getdiaginv copies them); *bad > 0 on a near-zero pivot
__global__ void k_bsr_diaginv(int nrow, int nb, const int *__restrict__ ia,
                              const int *__restrict__ ja, const double *__restrict__ val,
                              double *__restrict__ dinv, int *bad) {
    const int nb2 = nb * nb;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow; i += gridDim.x * blockDim.x) {
        double *a = dinv + (size_t)i * nb2;
        for (int q = 0; q < nb2; ++q) a[q] = 0.0;
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (ja[k] == i)
                for (int q = 0; q < nb2; ++q) a[q] = val[(size_t)k * nb2 + q];
        if (nb == 1) {
            a[0] = 1.0 / a[0];
            continue;
        }
        for (int k = 0; k < nb; ++k) {
            const int kn = k * nb, l = kn + k;
            if (fabs(a[l]) < SMALLREAL) { atomicAdd(bad, 1); break; }
            const double alinv = 1.0 / a[l];
            a[l] = alinv;
            for (int j = 0; j < k; ++j) a[kn + j] *= alinv;
            for (int j = k + 1; j < nb; ++j) a[kn + j] *= alinv;
            for (int r = 0; r < k; ++r) {
                const int rn = r * nb;
                for (int j = 0; j < nb; ++j)
                    if (j != k) a[rn + j] -= a[rn + k] * a[kn + j];
            }
            for (int r = k + 1; r < nb; ++r) {
                const int rn = r * nb;
                for (int j = 0; j < nb; ++j)
                    if (j != k) a[rn + j] -= a[rn + k] * a[kn + j];
            }
            for (int r = 0; r < k; ++r) a[r * nb + k] *= -alinv;
            for (int r = k + 1; r < nb; ++r) a[r * nb + k] *= -alinv;
        }
    }
}

// condensed value of block k: max over rows of sum |a|, negated off the
// diagonal
__device__ __forceinline__ double bsr_linf(const double *b, int nb) {
    double norm = 0.0;
    for (int r = 0; r < nb; ++r) {
        double v = 0.0;
        for (int c = 0; c < nb; ++c) v = v + fabs(b[r * nb + c]);
        norm = fmax(norm, v);
    }
    return norm;
}

__global__ void k_bsr_condense_count(int nrow, int nb, const int *__restrict__ ia,
                                     const int *__restrict__ ja, const double *__restrict__ val,
                                     int *cnt) {
    const int nb2 = nb * nb;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow; i += gridDim.x * blockDim.x) {
        int c = 0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) c += bsr_linf(val + (size_t)k * nb2, nb) > 1e-8;
        cnt[i] = c;
    }
}

__global__ void k_bsr_condense_fill(int nrow, int nb, const int *__restrict__ ia,
                                    const int *__restrict__ ja, const double *__restrict__ val,
                                    const int *__restrict__ cia, int *cja, double *cval) {
    const int nb2 = nb * nb;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow; i += gridDim.x * blockDim.x) {
        int p = cia[i];
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            double v = bsr_linf(val + (size_t)k * nb2, nb);
            if (ja[k] != i) v = -v;
            if (fabs(v) > 1e-8) {
                cja[p] = ja[k];
                cval[p] = v;
                ++p;
            }
        }
    }
}

// scalar expansion: row I nb + r lists the blocks of row I in order, the
// block's columns in order
__global__ void k_bsr_expand(int nrow, int nb, const int *__restrict__ ia,
                             const int *__restrict__ ja, const double *__restrict__ val,
                             int *sia, int *sja, double *sval) {
    const int nb2 = nb * nb;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow * nb;
         i += gridDim.x * blockDim.x) {
        const int I = i / nb, r = i - I * nb;
        const int len = (ia[I + 1] - ia[I]) * nb;
        int p = ia[I] * nb2 + r * len;
        sia[i] = p;
        if (i == nrow * nb - 1) sia[i + 1] = ia[nrow] * nb2;
        for (int k = ia[I]; k < ia[I + 1]; ++k)
            for (int c = 0; c < nb; ++c, ++p) {
                sja[p] = ja[k] * nb + c;
                sval[p] = val[(size_t)k * nb2 + r * nb + c];
            }
    }
}

__global__ void k_bsr_scalar_agg(int nrow, int nb, const int *__restrict__ agg, int *sagg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow * nb;
         i += gridDim.x * blockDim.x) {
        const int I = i / nb, a = agg[I];
        sagg[i] = a < 0 ? -1 : a * nb + (i - I * nb);
    }
}

// block Galerkin product with boolean P: blocks of coarse row C, the
// diagonal first, others in first-encounter order over (R row, A row)
__global__ void k_bsr_rap_count(int nc, const int *__restrict__ ria, const int *__restrict__ rja,
                                const int *__restrict__ ia, const int *__restrict__ ja,
                                const int *__restrict__ agg, int *cnt, int *list, int cap,
                                int *err) {
    for (int C = blockIdx.x * blockDim.x + threadIdx.x; C < nc; C += gridDim.x * blockDim.x) {
        int *seen = list + (size_t)C * cap;   // caller-sized scratch per coarse row
        int c = 1;
        seen[0] = C;
        for (int j1 = ria[C]; j1 < ria[C + 1]; ++j1) {
            const int I = rja[j1];
            for (int k = ia[I]; k < ia[I + 1]; ++k) {
                const int D = agg[ja[k]];
                if (D < 0) continue;
                bool found = false;
                for (int q = 0; q < c && !found; ++q) found = seen[q] == D;
                if (!found) {
                    if (c >= cap) { *err = 1; break; }
                    seen[c++] = D;
                }
            }
        }
        cnt[C] = c;
    }
}

__global__ void k_bsr_rap_fill(int nc, int nb, const int *__restrict__ ria,
                               const int *__restrict__ rja, const int *__restrict__ ia,
                               const int *__restrict__ ja, const double *__restrict__ val,
                               const int *__restrict__ agg, const int *__restrict__ cia,
                               int *cja, double *cval) {
    const int nb2 = nb * nb;
    for (int C = blockIdx.x * blockDim.x + threadIdx.x; C < nc; C += gridDim.x * blockDim.x) {
        const int base = cia[C];
        int c = 1;
        cja[base] = C;
        for (int q = 0; q < nb2; ++q) cval[(size_t)base * nb2 + q] = 0.0;
        for (int j1 = ria[C]; j1 < ria[C + 1]; ++j1) {
            const int I = rja[j1];
            for (int k = ia[I]; k < ia[I + 1]; ++k) {
                const int D = agg[ja[k]];
                if (D < 0) continue;
                int slot = -1;
                for (int q = 0; q < c; ++q)
                    if (cja[base + q] == D) { slot = q; break; }
                // R_CI A_IJ P_JD by ddense_mul with identity blocks: sums
                // from 0.0, so each entry is A's value with -0.0 made +0.0
                const double *src = val + (size_t)k * nb2;
                double *dst = cval + (size_t)(base + (slot < 0 ? c : slot)) * nb2;
                if (slot < 0) {
                    cja[base + c] = D;
                    ++c;
                    for (int q = 0; q < nb2; ++q) dst[q] = src[q] + 0.0;
                } else {
                    for (int q = 0; q < nb2; ++q) dst[q] += src[q] + 0.0;
                }
            }
        }
    }
}

// w = b - A x for block row I, the subtractions in row order (blocks in
// order, a block's columns in order): dbsr_aAxpy(-1, A, x, w) on w = b
// negates w, adds the products and negates back, which rounds as this
template <int NB>
__global__ void __launch_bounds__(128)
k_bsr_residual(int nrow, const int *__restrict__ ia, const int *__restrict__ ja,
               const double *__restrict__ val, const double *__restrict__ b,
               const double *__restrict__ x, double *__restrict__ w) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nrow; I += gridDim.x * blockDim.x) {
        double t[NB];
#pragma unroll
        for (int r = 0; r < NB; ++r) t[r] = b[I * NB + r];
        for (int k = ia[I]; k < ia[I + 1]; ++k) {
            const double *a = val + (size_t)k * (NB * NB);
            const int J = ja[k];
            double xj[NB];
#pragma unroll
            for (int c = 0; c < NB; ++c) xj[c] = x[J * NB + c];
#pragma unroll
            for (int r = 0; r < NB; ++r)
#pragma unroll
                for (int c = 0; c < NB; ++c) t[r] -= a[r * NB + c] * xj[c];
        }
#pragma unroll
        for (int r = 0; r < NB; ++r) w[I * NB + r] = t[r];
    }
}

// one block row of Jacobi / Gauss-Seidel: x_I = D_I^{-1} (b_I - sum_{J != I}
// A_IJ x_J), reading x from xin and writing xout (the same array for GS);
// CG: x read and written at L2 (other SMs wrote it in the same launch)
template <bool CG>
__device__ __forceinline__ double ldx(const double *p) { return CG ? __ldcg(p) : *p; }
template <bool CG>
__device__ __forceinline__ void stx(double *p, double v) {
    if (CG) __stcg(p, v);
    else *p = v;
}

template <int NB, bool CG = false>
__device__ __forceinline__ void bsr_relax_row(int I, const int *__restrict__ ia,
                                              const int *__restrict__ ja,
                                              const double *__restrict__ val,
                                              const double *__restrict__ dinv,
                                              const double *__restrict__ b, const double *xin,
                                              double *xout) {
    double t[NB];
#pragma unroll
    for (int r = 0; r < NB; ++r) t[r] = b[I * NB + r];
    const int k1 = ia[I + 1];
    int k = ia[I];
    // U blocks at a time: their column indices, then their x gathers, are
    // issued together before the products (same order of subtractions)
    constexpr int U = NB <= 2 ? 8 : 4;
    for (; k + U <= k1; k += U) {
        int J[U];
#pragma unroll
        for (int u = 0; u < U; ++u) J[u] = ja[k + u];
        double xj[U][NB];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int c = 0; c < NB; ++c) xj[u][c] = J[u] == I ? 0.0 : ldx<CG>(xin + J[u] * NB + c);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (J[u] == I) continue;
            const double *a = val + (size_t)(k + u) * (NB * NB);
#pragma unroll
            for (int r = 0; r < NB; ++r)
#pragma unroll
                for (int c = 0; c < NB; ++c) t[r] -= a[r * NB + c] * xj[u][c];
        }
    }
    for (; k < k1; ++k) {
        const int J = ja[k];
        if (J == I) continue;
        const double *a = val + (size_t)k * (NB * NB);
        double xj[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) xj[c] = ldx<CG>(xin + J * NB + c);
#pragma unroll
        for (int r = 0; r < NB; ++r)
#pragma unroll
            for (int c = 0; c < NB; ++c) t[r] -= a[r * NB + c] * xj[c];
    }
    const double *d = dinv + (size_t)I * (NB * NB);
#pragma unroll
    for (int r = 0; r < NB; ++r) {
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < NB; ++c) v += d[r * NB + c] * t[c];
        stx<CG>(xout + I * NB + r, v);
    }
}

template <int NB>
__global__ void __launch_bounds__(128)
k_bsr_jacobi(int nrow, const int *__restrict__ ia, const int *__restrict__ ja,
             const double *__restrict__ val, const double *__restrict__ dinv,
             const double *__restrict__ b, const double *__restrict__ x,
             double *__restrict__ xn) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nrow; I += gridDim.x * blockDim.x)
        bsr_relax_row<NB>(I, ia, ja, val, dinv, b, x, xn);
}

// the rows of one level set, in parallel
template <int NB>
__global__ void __launch_bounds__(128)
k_bsr_gs_set(const int *__restrict__ rows, int cnt, const int *__restrict__ ia,
             const int *__restrict__ ja, const double *__restrict__ val,
             const double *__restrict__ dinv, const double *__restrict__ b, double *x) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x)
        bsr_relax_row<NB>(rows[q], ia, ja, val, dinv, b, x, x);
}

// a run of small level sets [first, last) by one CTA, sets in order
template <int NB>
__global__ void __launch_bounds__(256)
k_bsr_gs_run(const int *__restrict__ rows, const int *__restrict__ set_ptr, int first,
             int last, const int *__restrict__ ia, const int *__restrict__ ja,
             const double *__restrict__ val, const double *__restrict__ dinv,
             const double *__restrict__ b, double *x) {
    for (int k = first; k < last; ++k) {
        for (int q = set_ptr[k] + threadIdx.x; q < set_ptr[k + 1]; q += blockDim.x)
            bsr_relax_row<NB>(rows[q], ia, ja, val, dinv, b, x, x);
        __syncthreads();
    }
}

// consecutive large level sets [first, last) in one cooperative launch,
// the sets separated by the bounded grid barrier
template <int NB>
__global__ void __launch_bounds__(128)
k_bsr_gs_sets_grid(const int *__restrict__ rows, const int *__restrict__ set_ptr, int first,
                   int last, const int *__restrict__ ia, const int *__restrict__ ja,
                   const double *__restrict__ val, const double *__restrict__ dinv,
                   const double *__restrict__ b, double *x, unsigned *bar, int *err) {
    const int nthr = gridDim.x * blockDim.x;
    for (int k = first; k < last; ++k) {
        const int q1 = set_ptr[k + 1];
        for (int q = set_ptr[k] + blockIdx.x * blockDim.x + threadIdx.x; q < q1; q += nthr)
            bsr_relax_row<NB, true>(rows[q], ia, ja, val, dinv, b, x, x);
        if (k + 1 < last && !grid_barrier(bar, gridDim.x, err)) return;
    }
}

template <int NB>
int bsr_gs_sets_grid(const int *rows, const int *set_ptr, int first, int last, int max_set,
                     const int *ia, const int *ja, const double *val, const double *dinv,
                     const double *b, double *x, unsigned *bar, int *err, cudaStream_t s) {
    static int per_sm = 0;
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bsr_gs_sets_grid<NB>, 128,
                                                          0) != cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    const int grid = std::max(1, std::min(per_sm * sm_count(), div_up(max_set, 128)));
    HZB_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HZB_CUDA(cudaLaunchKernelEx(&cfg, k_bsr_gs_sets_grid<NB>, rows, set_ptr, first, last, ia,
                                ja, val, dinv, b, x, bar, err));
    return SUCCESS;
}

// f(std::integral_constant<int, nb>) for the block sizes the kernels hold
template <typename F>
void with_nb(int nb, F &&f) {
    switch (nb) {
    case 1: f(std::integral_constant<int, 1>()); break;
    case 2: f(std::integral_constant<int, 2>()); break;
    case 3: f(std::integral_constant<int, 3>()); break;
    case 4: f(std::integral_constant<int, 4>()); break;
    case 5: f(std::integral_constant<int, 5>()); break;
    case 6: f(std::integral_constant<int, 6>()); break;
    case 7: f(std::integral_constant<int, 7>()); break;
    default: f(std::integral_constant<int, 8>()); break;
    }
}
}  // namespace

struct BsrLevel {
    int nrow = 0, nnzb = 0, nb = 1, nc = 0;
    int *ia = nullptr, *ja = nullptr;
    double *val = nullptr, *dinv = nullptr;
    int *agg = nullptr;
    // scalar expansion and scalar aggregate transfer
    Level s;
    Schedule asc, desc;
    void release() {
        dfree(ia); dfree(ja); dfree(val); dfree(dinv); dfree(agg);
        s.release();
        asc.release();
        desc.release();
    }
};

struct BsrHier {
    std::vector<BsrLevel> lv;
    int nl = 0, nb = 1;
    KrylovWork kwc;   // inner products of the coarse scaling (level-0 length)
    void release() {
        for (auto &L : lv) L.release();
        lv.clear();
        kwc.release();
        nl = 0;
    }
};

// device temporaries of one setup step, freed (stream-ordered) with it
struct Scratch {
    std::vector<void *> p;
    template <typename T>
    int get(T **x, size_t n) {
        const int rc = dalloc(x, n);
        if (rc == SUCCESS) p.push_back((void *)*x);
        return rc;
    }
    ~Scratch() {
        for (void *q : p) cudaFreeAsync(q, cur_stream());
    }
};

void bsr_release(hzb_solver *S) {
    if (!S->bsr) return;
    S->bsr->release();
    delete S->bsr;
    S->bsr = nullptr;
}

static int expand(BsrLevel &L, cudaStream_t s) {
    const int n = L.nrow * L.nb, nnz = L.nnzb * L.nb * L.nb;
    Level &E = L.s;
    E.n = n;
    E.nnz = nnz;
    E.own_A = true;
    HZB_TRY(dalloc(&E.ia, n + 1));
    HZB_TRY(dalloc(&E.ja, nnz));
    HZB_TRY(dalloc(&E.val, nnz));
    k_bsr_expand<<<grid_for(n), 256, 0, s>>>(L.nrow, L.nb, L.ia, L.ja, L.val, E.ia, E.ja, E.val);
    count_launch();
    HZB_LAUNCH_CHECK();
    HZB_TRY(bundle_capacity(n, E.ia, s, &E.bundle_cap));
    HZB_TRY(dalloc(&E.b, n));
    HZB_TRY(dalloc(&E.x, n));
    HZB_TRY(dalloc(&E.w, n));
    HZB_TRY(dalloc(&E.t, n));
    HZB_TRY(dalloc(&E.r1, n));   // A P e of the coarse scaling
    return SUCCESS;
}

static int bsr_build(hzb_solver *S, int nrow, int nnzb, int nb, const int *d_ia,
                     const int *d_ja, const double *d_val) {
    if (nb < 1 || nb > BSR_MAXNB) {
        set_error_msg("block size must be 1 .. 8");
        return ERROR_INPUT_PAR;
    }
    if (nrow < 1 || nnzb < 1) return ERROR_MAT_SIZE;
    bsr_release(S);
    cudaStream_t s = S->s;
    HZB_CUDA(cudaEventRecord(S->e0, s));
    S->bsr = new BsrHier();
    BsrHier &H = *S->bsr;
    H.nb = nb;
    const int nb2 = nb * nb;
    H.lv.emplace_back();
    {
        BsrLevel &L0 = H.lv[0];
        L0.nrow = nrow; L0.nnzb = nnzb; L0.nb = nb;
        HZB_TRY(dalloc(&L0.ia, nrow + 1));
        HZB_TRY(dalloc(&L0.ja, nnzb));
        HZB_TRY(dalloc(&L0.val, (size_t)nnzb * nb2));
        HZB_CUDA(cudaMemcpyAsync(L0.ia, d_ia, sizeof(int) * (nrow + 1), cudaMemcpyDefault, s));
        HZB_CUDA(cudaMemcpyAsync(L0.ja, d_ja, sizeof(int) * nnzb, cudaMemcpyDefault, s));
        HZB_CUDA(cudaMemcpyAsync(L0.val, d_val, sizeof(double) * nnzb * nb2, cudaMemcpyDefault,
                                 s));
    }
    const int min_cdof = std::max<int>(S->amg.coarse_dof, 50);
    const int max_levels = std::min<int>(S->amg.max_levels, MAX_AMG_LVL);
    const bool vmb = S->amg.aggregation_type == VMB;
    const bool par = !vmb && (S->bp.matching == HZB_MATCH_PARALLEL ||
                              S->amg.aggregation_type == HEC);
    int lvl = 0, rc = SUCCESS;
    for (;;) {
        // device temporaries of this level, freed when the step ends (also on
        // the early returns)
        Scratch tmpv;
        BsrLevel &L = H.lv[lvl];
        if ((rc = expand(L, s))) break;
        if (!(L.nrow > min_cdof && lvl < max_levels - 1)) break;
        // the diagonal inverses of the levels that get a coarser one (the
        // smoothed levels); a near-zero pivot ends the process in the
        // reference, an error here
        const int m = L.nrow;
        int *bad = nullptr, *tmp = nullptr;
        if ((rc = dalloc(&L.dinv, (size_t)m * nb2)) || (rc = tmpv.get(&bad, 1)) ||
            (rc = tmpv.get(&tmp, scan_tmp_size(m + 2))))
            break;
        HZB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
        k_bsr_diaginv<<<grid_for(m), 128, 0, s>>>(m, nb, L.ia, L.ja, L.val, L.dinv, bad);
        count_launch();
        int hbad = 0;
        HZB_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        HZB_CUDA(cudaStreamSynchronize(s));
        if (hbad) {
            set_error_msg("a diagonal block has a pivot close to zero");
            rc = ERROR_DATA_ZERODIAG;
            break;
        }
        // condensed scalar matrix, then the aggregation on its strength graph
        int *cnt = nullptr, *pia = nullptr, *pja = nullptr, *nia = nullptr, *nja = nullptr,
            *work = nullptr, pnnz = 0, nnnz = 0, nagg = 0;
        double *pval = nullptr, *nval = nullptr;
        if ((rc = tmpv.get(&cnt, m)) || (rc = tmpv.get(&pia, m + 1))) break;
        k_bsr_condense_count<<<grid_for(m), 256, 0, s>>>(m, nb, L.ia, L.ja, L.val, cnt);
        count_launch();
        if ((rc = scan_exclusive(cnt, pia, m, tmp, s))) break;
        HZB_CUDA(cudaMemcpyAsync(&pnnz, pia + m, sizeof(int), cudaMemcpyDeviceToHost, s));
        HZB_CUDA(cudaStreamSynchronize(s));
        if ((rc = tmpv.get(&pja, pnnz > 0 ? pnnz : 1)) ||
            (rc = tmpv.get(&pval, pnnz > 0 ? pnnz : 1)))
            break;
        k_bsr_condense_fill<<<grid_for(m), 256, 0, s>>>(m, nb, L.ia, L.ja, L.val, pia, pja, pval);
        count_launch();
        DCsr<double> PP;
        PP.n = m; PP.nnz = pnnz; PP.ia = pia; PP.ja = pja; PP.val = pval;
        if ((rc = bundle_capacity(m, pia, s, &PP.bundle_cap))) break;
        if ((rc = tmpv.get(&nia, m + 1)) || (rc = tmpv.get(&nja, pnnz > 0 ? pnnz : 1)) ||
            (rc = tmpv.get(&nval, pnnz > 0 ? pnnz : 1)) || (rc = dalloc(&L.agg, m)) ||
            (rc = tmpv.get(&work, par ? (size_t)6 * m + scan_tmp_size(m + 1) + 8
                                      : (size_t)(vmb ? 2 : 1) * m)))
            break;
        rc = strength_graph(PP, S->amg.strong_coupled, nia, nja, nval, &nnnz, tmp, s);
        if (!rc) {
            if (vmb)
                rc = vmb_aggregate(m, nia, nja, S->amg.max_aggregation, L.agg, &nagg, work, s);
            else if (par) rc = hem_parallel(m, nia, nja, nval, L.agg, &nagg, work, s);
            else rc = hem_exact(m, nia, nja, nval, L.agg, &nagg, work, s);
        }
        if (rc) break;
        if (nagg < 1) break;   // the reference stops coarsening here
        L.nc = nagg;
        // R (block pattern, fine rows ascending) and the scalar aggregate maps
        int *ria = nullptr, *rja = nullptr, *stmp = nullptr;
        if ((rc = tmpv.get(&ria, nagg + 1)) || (rc = tmpv.get(&rja, m))) break;
        if ((rc = restriction_pattern(m, nagg, L.agg, ria, rja, tmp, s))) break;
        Level &E = L.s;
        E.nc = nagg * nb;
        if ((rc = dalloc(&E.agg, E.n))) break;
        k_bsr_scalar_agg<<<grid_for(E.n), 256, 0, s>>>(m, nb, L.agg, E.agg);
        count_launch();
        if ((rc = dalloc(&E.ria, E.nc + 1)) || (rc = dalloc(&E.rja, E.n)) ||
            (rc = tmpv.get(&stmp, scan_tmp_size(E.n + 1))) ||
            (rc = restriction_pattern(E.n, E.nc, E.agg, E.ria, E.rja, stmp, s)))
            break;
        // coarse blocks per row: distinct aggregates met, in a table per row
        // that grows when a row overflows it
        int *ccnt = nullptr, *list = nullptr, *err = nullptr, herr = 0;
        if ((rc = tmpv.get(&ccnt, nagg)) || (rc = tmpv.get(&err, 1))) break;
        for (int cap = std::min(64, nagg);; cap = std::min(cap * 4, nagg)) {
            if ((rc = tmpv.get(&list, (size_t)nagg * cap))) break;
            HZB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
            k_bsr_rap_count<<<grid_for(nagg), 128, 0, s>>>(nagg, ria, rja, L.ia, L.ja, L.agg,
                                                            ccnt, list, cap, err);
            count_launch();
            HZB_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
            HZB_CUDA(cudaStreamSynchronize(s));
            if (!herr || cap >= nagg) break;
        }
        if (rc) break;
        // the coarse level joins the hierarchy before its arrays exist, so a
        // failure from here on is released with it
        H.lv.emplace_back();
        BsrLevel &C = H.lv.back();
        BsrLevel &Lf = H.lv[lvl];   // re-bind: emplace_back may move the levels
        C.nrow = nagg; C.nb = nb;
        if ((rc = dalloc(&C.ia, nagg + 1)) || (rc = scan_exclusive(ccnt, C.ia, nagg, tmp, s)))
            break;
        HZB_CUDA(cudaMemcpyAsync(&C.nnzb, C.ia + nagg, sizeof(int), cudaMemcpyDeviceToHost, s));
        HZB_CUDA(cudaStreamSynchronize(s));
        if ((rc = dalloc(&C.ja, C.nnzb)) || (rc = dalloc(&C.val, (size_t)C.nnzb * nb2))) break;
        k_bsr_rap_fill<<<grid_for(nagg), 128, 0, s>>>(nagg, nb, ria, rja, Lf.ia, Lf.ja, Lf.val,
                                                       Lf.agg, C.ia, C.ja, C.val);
        count_launch();
        HZB_LAUNCH_CHECK();
        ++lvl;
    }
    if (rc) return rc;
    H.nl = lvl + 1;
    // Gauss-Seidel level sets of the block pattern on the smoothed levels
    if (S->amg.smoother == SMOOTHER_GS || S->amg.smoother == SMOOTHER_SGS)
        for (int l = 0; l < H.nl - 1; ++l) {
            BsrLevel &L = H.lv[l];
            HZB_TRY(gs_schedule(L.nrow, L.ia, L.ja, L.nnzb, 0, &L.asc, s));
            HZB_TRY(gs_schedule(L.nrow, L.ia, L.ja, L.nnzb, 1, &L.desc, s));
        }
    HZB_TRY(H.kwc.alloc(H.lv[0].s.n));
    HZB_TRY(S->kw.alloc(H.lv[0].s.n));
    HZB_CUDA(cudaEventRecord(S->e1, s));
    HZB_CUDA(cudaEventSynchronize(S->e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, S->e0, S->e1);
    S->st.setup_seconds = ms * 1e-3;
    S->st.num_levels = H.nl;
    for (int l = 0; l < H.nl && l < MAX_AMG_LVL; ++l) {
        S->st.rows[l] = H.lv[l].nrow;
        S->st.nnz[l] = H.lv[l].nnzb;
    }
    return SUCCESS;
}

int bsr_setup(hzb_solver *S, int nrow, int nnzb, int nb, const int *d_ia, const int *d_ja,
              const double *d_val) {
    const int rc = bsr_build(S, nrow, nnzb, nb, d_ia, d_ja, d_val);
    if (rc != SUCCESS) bsr_release(S);
    return rc;
}

DCsr<double> bsr_scalar_A(hzb_solver *S) { return S->bsr->lv[0].s.A64(); }

int bsr_block_size(const hzb_solver *S) { return S->bsr ? S->bsr->nb : 0; }

int bsr_level_copy(const hzb_solver *S, int l, int *nrow, int *nnzb, int *ia, int *ja,
                   double *val, int *agg) {
    if (!S->bsr || l < 0 || l >= S->bsr->nl) return ERROR_INPUT_PAR;
    const BsrLevel &L = S->bsr->lv[l];
    if (nrow) *nrow = L.nrow;
    if (nnzb) *nnzb = L.nnzb;
    const int nb2 = L.nb * L.nb;
    if (ia) HZB_CUDA(cudaMemcpy(ia, L.ia, sizeof(int) * (L.nrow + 1), cudaMemcpyDeviceToHost));
    if (ja) HZB_CUDA(cudaMemcpy(ja, L.ja, sizeof(int) * L.nnzb, cudaMemcpyDeviceToHost));
    if (val)
        HZB_CUDA(cudaMemcpy(val, L.val, sizeof(double) * (size_t)L.nnzb * nb2,
                            cudaMemcpyDeviceToHost));
    if (agg && l < S->bsr->nl - 1)
        HZB_CUDA(cudaMemcpy(agg, L.agg, sizeof(int) * L.nrow, cudaMemcpyDeviceToHost));
    return SUCCESS;
}

static int bsr_smooth(hzb_solver *S, BsrLevel &L, int kind, int sweeps) {
    cudaStream_t s = S->s;
    Level &E = L.s;
    for (int it = 0; it < sweeps; ++it) {
        if (kind == 0) {   // Jacobi: a new iterate from the old one
            with_nb(L.nb, [&](auto c) {
                constexpr int NB = decltype(c)::value;
                k_bsr_jacobi<NB><<<grid_for(L.nrow, 128), 128, 0, s>>>(L.nrow, L.ia, L.ja, L.val,
                                                                       L.dinv, E.b, E.x, E.t);
            });
            count_launch();
            HZB_TRY(vcopy<double>(E.n, E.t, E.x, s));
            continue;
        }
        const Schedule &sc = kind == 1 ? L.asc : L.desc;
        int *err = wait_err(S);
        const size_t nr = sc.run_first.size();
        for (size_t q = 0; q < nr; ++q) {
            const int f = sc.run_first[q], l = sc.run_last[q];
            // consecutive large sets: one cooperative launch when the
            // barrier has its words and a place to report to
            size_t q2 = q;
            while (l < 0 && q2 < nr && sc.run_last[q2] < 0) ++q2;
            int rc = SUCCESS;
            with_nb(L.nb, [&](auto c) {
                constexpr int NB = decltype(c)::value;
                if (l < 0 && sc.bar && err && q2 - q > 1) {
                    int max_set = 0;
                    for (size_t r = q; r < q2; ++r) max_set = std::max(max_set, sc.run_max[r]);
                    rc = bsr_gs_sets_grid<NB>(sc.rows, sc.set_ptr, f, sc.run_first[q2 - 1] + 1,
                                              max_set, L.ia, L.ja, L.val, L.dinv, E.b, E.x,
                                              sc.bar, err, s);
                    q = q2 - 1;
                } else if (l < 0) {
                    const int cnt = sc.h_ptr[f + 1] - sc.h_ptr[f];
                    k_bsr_gs_set<NB><<<grid_for(cnt, 128), 128, 0, s>>>(
                        sc.rows + sc.h_ptr[f], cnt, L.ia, L.ja, L.val, L.dinv, E.b, E.x);
                } else {
                    k_bsr_gs_run<NB><<<1, 256, 0, s>>>(sc.rows, sc.set_ptr, f, l, L.ia, L.ja,
                                                        L.val, L.dinv, E.b, E.x);
                }
            });
            HZB_TRY(rc);
            count_launch();
        }
    }
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

// w = b - A x on level L (block residual of mgcycle_bsr)
static void bsr_residual(BsrLevel &L, const double *b, const double *x, double *w,
                         cudaStream_t s) {
    with_nb(L.nb, [&](auto c) {
        constexpr int NB = decltype(c)::value;
        k_bsr_residual<NB><<<grid_for(L.nrow, 128), 128, 0, s>>>(L.nrow, L.ia, L.ja, L.val, b,
                                                                 x, w);
    });
    count_launch();
}

// the smoothing of mgcycle_bsr: Jacobi, GS (ascending before, descending
// after), SGS (both)
static int bsr_smoothing(hzb_solver *S, BsrLevel &L, const AMG_param &cyc, bool pre) {
    const int steps = cyc.presmooth_iter;
    if (steps <= 0) return SUCCESS;
    switch (cyc.smoother) {
    case SMOOTHER_JACOBI: return bsr_smooth(S, L, 0, steps);
    case SMOOTHER_GS: return bsr_smooth(S, L, pre ? 1 : 2, steps);
    case SMOOTHER_SGS:
        for (int i = 0; i < steps; ++i) {
            HZB_TRY(bsr_smooth(S, L, 1, 1));
            HZB_TRY(bsr_smooth(S, L, 2, 1));
        }
        return SUCCESS;
    }
    set_error_msg("block smoothers: Jacobi, GS, SGS");
    return ERROR_AMG_SMOOTH_TYPE;
}

int bsr_cycle(hzb_solver *S, const AMG_param &cyc) {
    BsrHier &H = *S->bsr;
    cudaStream_t s = S->s;
    const int nl = H.nl;
    int nu[MAX_AMG_LVL] = {0};
    int l = 0;
forward:
    while (l < nl - 1) {
        BsrLevel &L = H.lv[l];
        Level &E = L.s;
        nu[l]++;
        HZB_TRY(bsr_smoothing(S, L, cyc, true));
        bsr_residual(L, E.b, E.x, E.w, s);
        Level &Cn = H.lv[l + 1].s;
        HZB_TRY(restrict_agg<double>(E.nc, E.ria, E.rja, E.w, Cn.b, s));
        ++l;
        HZB_TRY(vzero<double>(Cn.n, Cn.x, s));
    }
    {
        // GMRES(25) to the tolerance of param_amg_init, at most min(n^2, 200)
        Level &Cn = H.lv[nl - 1].s;
        const int csize = Cn.n;
        const int cmaxit = (int)std::min<long long>((long long)csize * csize, 200);
        double rel = 0.0;
        const int it = gmres(S, Cn.A64(), Cn.b, Cn.x, PC_NONE, nullptr, cyc.tol, cmaxit, 25,
                             STOP_REL_RES, 0, false, &rel, MAX_AMG_LVL + 1);
        if (it == ERROR_SOLVER_MISC || it == ERROR_ALLOC_MEM) return it;
    }
    while (l > 0) {
        --l;
        BsrLevel &L = H.lv[l];
        Level &E = L.s, &Cn = H.lv[l + 1].s;
        if (cyc.coarse_scaling == ON) {
            // PeH = P e, Aeh = A PeH, alpha = min((Aeh, w) / (Aeh, Aeh), 1),
            // x += alpha PeH (mgcycle.c:1075-1090)
            KrylovWork &w = H.kwc;
            HZB_TRY(vzero<double>(E.n, E.t, s));
            HZB_TRY(prolong_agg<double>(E.n, E.agg, Cn.x, E.t, 1.0, s));
            HZB_TRY(spmv<double>(E.A64(), SPMV_Y, E.t, nullptr, E.r1, 1.0, nullptr, s));
            HZB_TRY(dot(E.n, E.r1, E.w, w.part, w.sc + 8, s));
            HZB_TRY(dot(E.n, E.r1, E.r1, w.part, w.sc + 9, s));
            HZB_CUDA(cudaMemcpyAsync(w.h_sc + 8, w.sc + 8, 2 * sizeof(double),
                                     cudaMemcpyDeviceToHost, s));
            HZB_CUDA(cudaStreamSynchronize(s));
            const double alpha = std::min(w.h_sc[8] / w.h_sc[9], 1.0);
            HZB_TRY(prolong_agg<double>(E.n, E.agg, Cn.x, E.x, alpha, s));
        } else {
            HZB_TRY(prolong_agg<double>(E.n, E.agg, Cn.x, E.x, 1.0, s));
        }
        HZB_TRY(bsr_smoothing(S, L, cyc, false));
        if (nu[l] < cyc.cycle_type) break;
        nu[l] = 0;
    }
    if (l > 0) goto forward;
    return SUCCESS;
}

// reps launches of one block kernel on level l between the handle's events:
// the residual (x, b -> w), a Jacobi sweep (x -> t) or an ascending
// Gauss-Seidel sweep over the level sets (x in place); algorithmic bytes per
// launch: blocks, block columns, row pointers (+ the diagonal inverses for a
// sweep) and three n-vectors
int bsr_time_kernel(hzb_solver *S, int which, int l, int reps, double *ms_per_launch,
                    double *bytes_per_launch) {
    if (!S->bsr || l < 0 || l >= S->bsr->nl || reps < 1) return ERROR_INPUT_PAR;
    BsrLevel &L = S->bsr->lv[l];
    Level &E = L.s;
    const bool sweep = which == HZB_K_BSR_JAC || which == HZB_K_BSR_GS;
    if (which != HZB_K_BSR_RES && !sweep) return ERROR_INPUT_PAR;
    if (sweep && !L.dinv) return ERROR_INPUT_PAR;   // the coarsest level is not smoothed
    if (which == HZB_K_BSR_GS && L.asc.run_first.empty()) return ERROR_INPUT_PAR;
    const double nb2 = (double)L.nb * L.nb;
    double bytes = L.nnzb * (8.0 * nb2 + 4.0) + 4.0 * (L.nrow + 1) + 3.0 * 8.0 * E.n;
    if (sweep) bytes += 8.0 * nb2 * L.nrow;
    cudaStream_t s = S->s;
    HZB_TRY(vzero<double>(E.n, E.x, s));
    auto launch = [&]() -> int {
        if (which == HZB_K_BSR_RES) {
            bsr_residual(L, E.b, E.x, E.w, s);
            HZB_LAUNCH_CHECK();
            return SUCCESS;
        }
        if (which == HZB_K_BSR_JAC) {
            with_nb(L.nb, [&](auto c) {
                constexpr int NB = decltype(c)::value;
                k_bsr_jacobi<NB><<<grid_for(L.nrow, 128), 128, 0, s>>>(L.nrow, L.ia, L.ja, L.val,
                                                                       L.dinv, E.b, E.x, E.t);
            });
            count_launch();
            HZB_LAUNCH_CHECK();
            return SUCCESS;
        }
        return bsr_smooth(S, L, 1, 1);
    };
    HZB_TRY(launch());
    HZB_CUDA(cudaEventRecord(S->e0, s));
    for (int r = 0; r < reps; ++r) HZB_TRY(launch());
    HZB_CUDA(cudaEventRecord(S->e1, s));
    HZB_CUDA(cudaEventSynchronize(S->e1));
    float ms = 0.f;
    HZB_CUDA(cudaEventElapsedTime(&ms, S->e0, S->e1));
    *ms_per_launch = ms / reps;
    *bytes_per_launch = bytes;
    return SUCCESS;
}

// precond_dbsr_amg (precond.c:1311-1335): maxit cycles from zero
int bsr_precond(hzb_solver *S, const double *r, double *z) {
    BsrHier &H = *S->bsr;
    Level &E = H.lv[0].s;
    double *sx = E.x;
    HZB_TRY(vcopy<double>(E.n, r, E.b, S->s));   // the residual is an input
    E.x = z;
    int rc = vzero<double>(E.n, z, S->s);
    for (int i = 0; rc == SUCCESS && i < S->bsr_cyc.maxit; ++i) rc = bsr_cycle(S, S->bsr_cyc);
    E.x = sx;
    return rc;
}

}  // namespace hzb
