// hzb_kernels.cuh -- host launchers of the sparse / vector / smoother kernels.
//
// Arithmetic contract of the FP64 kernels: this translation unit set is
// compiled with -fmad=false, every row sum runs in one thread in CSR order
// starting from 0.0 (or from b_i for the smoothers), so each value is
// rounded exactly as the reference's sequential C loops round it.
#pragma once
#include "hzb_common.cuh"

namespace hzb {

// FP32 sliced-ELL copy of a level's matrix (hzb_sell.cu): slot r of a
// 256-row window holds row row[r] (-1: none) of len[r] entries, stored at
// col/val[ptr[r / 32] + 32 u + r % 32]; npad = 0: none.
struct SellView {
    int npad = 0;
    const int *ptr = nullptr, *row = nullptr, *len = nullptr, *col = nullptr;
    const float *val = nullptr;
};
struct SellArrays {
    int npad = 0;
    int *ptr = nullptr, *row = nullptr, *len = nullptr, *col = nullptr;
    float *val = nullptr;
    SellView view() const {
        SellView v;
        v.npad = npad; v.ptr = ptr; v.row = row; v.len = len; v.col = col; v.val = val;
        return v;
    }
    void release();
};

// A CSR matrix resident in device memory (int32 pattern).
template <typename T>
struct DCsr {
    int n = 0, nnz = 0;
    const int *ia = nullptr, *ja = nullptr;
    const T *val = nullptr;
    int bundle_cap = 0;   // max entries in any bundle of bundle_rows rows (0: none)
    int bundle_rows = 128;   // rows per CTA of the staged kernels: 64, 128 or 256
    // FP32 only: lanes per row of the vector-CSR kernels (2..16), 0 for the
    // staged bundles, SELL_LANES for the sliced-ELL copy in `sell`.  A row's
    // partial sums are combined across its lanes, so the lanes kernels do
    // not give the sequential CSR-order sum of the FP64 kernels.
    int vec_lanes = 0;
    SellView sell;
    // Optional activity of 256-row blocks (ACT_ROWS): kernels skip the rows
    // of a block whose byte is 0 (batched solves skip converged systems).
    const unsigned char *act = nullptr;
};
constexpr int ACT_ROWS = 256;
constexpr int SELL_LANES = -1;

constexpr int SPMV_ROWS = 128;          // rows per CTA in the row-bundle SpMV
constexpr int SPMV_SMEM_MAX = 160 * 1024;

enum SpmvMode { SPMV_Y = 0, SPMV_RES = 1, SPMV_AXPY = 2, SPMV_Y_DOT = 3 };

// Largest number of stored entries in any SPMV_ROWS-row (rows-row) bundle.
int bundle_capacity(int n, const int *ia, cudaStream_t s, int *cap);
int bundle_capacity_rows(int n, int rows, const int *ia, cudaStream_t s, int *cap);
// Picks the bundle size (64/128/256 rows) of A by timing its SpMV on x -> y.
int autotune_bundle(DCsr<double> &A, const double *x, double *y, cudaStream_t s);
// Picks the FP32 schedule (staged bundles or 4/8/16 lanes per row) by timing
// the l1-Jacobi sweep of A on b, x -> xn.
int autotune_fp32(DCsr<float> &A, const float *b, const float *x, float *xn, cudaStream_t s);
// the FP32 schedule an earlier autotune_fp32 picked for a level of this
// shape, if any
bool fp32_schedule_known(int n, int nnz, int *lanes);

// Sliced-ELL copy of an FP32 CSR matrix (hzb_sell.cu); *out stays empty
// (npad 0) when its slice offsets would overflow int.  Sweep and SpMV on it
// (no activity array, no SPMV_Y_DOT).
int sell_build(int n, const int *ia, const int *ja, const float *a, SellArrays *out,
               cudaStream_t s);
int sell_l1_sweep(const DCsr<float> &A, const float *b, const float *x, float *xn,
                  const float *omega, cudaStream_t s);
int sell_spmv(const DCsr<float> &A, int mode, const float *x, const float *b, float *y,
              float alpha, cudaStream_t s);
int spmv_blocks_rows(int n, int rows);

// y = A x (SPMV_Y); y = b - A x (SPMV_RES); y += alpha A x with the
// reference's +-1 special cases (SPMV_AXPY); y = A x and partial dot(y, x)
// into part[blockIdx] (SPMV_Y_DOT, part sized by spmv_blocks()).
template <typename T>
int spmv(const DCsr<T> &A, int mode, const T *x, const T *b, T *y, T alpha,
         T *part, cudaStream_t s);
int spmv_blocks(int n);

// b_c[c] = sum over R row c of w (R rows list fine indices ascending).
template <typename T>
int restrict_agg(int nc, const int *ria, const int *rja, const T *w, T *bc,
                 cudaStream_t s, const unsigned char *act_c = nullptr);
// x_i (+/-)= alpha * x_c[agg_i] as dcsr_aAxpy_agg does for unit P.
template <typename T>
int prolong_agg(int n, const int *agg, const T *xc, T *x, T alpha,
                cudaStream_t s, const unsigned char *act = nullptr);
// fused: x_i += x_c[agg_i] (alpha = 1), then the first l1-Jacobi sweep
// reads the updated x -- kept separate in parity mode.

// Jacobi (w = 1) sweep reading x, writing xn (reference smoother.c:35-100).
int jacobi_sweep(const DCsr<double> &A, const double *dj, const double *b,
                 const double *x, double *xn, cudaStream_t s);
// l1-Jacobi sweep: xn = x + omega * (b - A x) / l1 (omega == nullptr: 1).
template <typename T>
int l1_sweep(const DCsr<T> &A, const T *b, const T *x, T *xn,
             const float *omega, cudaStream_t s);
// l1 row norms d_i = sum_j |a_ij| (CSR order), and the first l1-Jacobi sweep
// from x = 0, which needs no matrix: xn_i = omega_i * (b_i / d_i).
template <typename T>
int l1_norms(const DCsr<T> &A, T *d, cudaStream_t s);
template <typename T>
int l1_first_sweep(int n, const T *b, const T *d, T *xn, const float *omega,
                   cudaStream_t s, const unsigned char *act = nullptr);
// Gauss-Seidel family on a list of independent rows (one level set / colour).
//   kind 0: x_i = t * d_i            (GS, d_i = 1/a_ii)
//   kind 1: x_i = w (t/d_i) + (1-w) x_i  if |d_i| > 1e-20   (SOR)
//   kind 2: x_i = t / d_i               if |d_i| > 1e-20   (SGS)
//   | GS_SKIP_LAST: leave row n-1 untouched (SGS backward sweep)
constexpr int GS_SKIP_LAST = 16;
template <typename T>
int gs_rows(const DCsr<T> &A, int kind, const int *rows, int cnt,
            const T *d, T w, const T *b, T *x, cudaStream_t s);
// Grid barrier of the cooperative level-set sweeps: an arrival counter and a
// generation word (bar[0], bar[1]; the last CTA to arrive resets the counter
// and bumps the generation).  Its wait is bounded: after GRID_SPIN_LIMIT
// polls (about half a second) the CTA raises *err and returns false, and a
// CTA that sees *err raised returns false too, so a missing CTA ends the
// sweep with an error that the host reads, never with a hang.  Cooperative
// launch guarantees the CTAs are co-resident.  The host zeroes bar before
// every launch.
constexpr unsigned GRID_SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned nblocks, int *err) {
    __shared__ int s_bad;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = bar + 1;
        volatile int *verr = err;
        const unsigned g = *gen;
        int bad = 0;
        __threadfence();
        if (atomicAdd(bar, 1u) == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            for (unsigned spin = 0; *gen == g; ++spin) {
                if (*verr) { bad = 1; break; }
                if (spin > GRID_SPIN_LIMIT) {
                    atomicExch(err, 1);
                    bad = 1;
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        if (*verr) bad = 1;
        s_bad = bad;
    }
    __syncthreads();
    return !s_bad;
}

// consecutive level sets [first, last) of up to max_set rows each in one
// cooperative launch with a bounded grid barrier between sets (bar: 2
// device words, zero at first use; err: raised if a barrier wait ran out)
template <typename T>
int gs_sets_grid(const DCsr<T> &A, int kind, const int *rows, const int *set_ptr, int first,
                 int last, int max_set, const T *d, T w, const T *b, T *x, unsigned *bar,
                 int *err, cudaStream_t s);
// One CTA runs level sets [first, last) back to back, __syncthreads between
// sets: at most GS_RUN_SETS sets of at most GS_SMALL_SET rows each (max_set:
// the run's largest set), else ERROR_INPUT_PAR.  x lives in shared memory
// for the run when the level fits GS_SMEM_MAX.
constexpr int GS_SMALL_SET = 1024;
constexpr int GS_RUN_SETS = 4096;
constexpr size_t GS_SMEM_MAX = 220 * 1024;
__host__ __device__ constexpr size_t gs_sp_bytes(int nsets) {
    return (sizeof(int) * (size_t)(nsets + 1) + 15) / 16 * 16;
}
template <typename T>
int gs_run(const DCsr<T> &A, int kind, const int *rows, const int *set_ptr,
           int first, int last, int max_set, const T *d, T w, const T *b, T *x,
           cudaStream_t s);

// Deterministic reductions: partial sums per block, then an ordered final
// sum into out[0].
int reduce_final(const double *part, int nparts, double *out, cudaStream_t s);
int reduce_final_max(const double *part, int nparts, double *out,
                     cudaStream_t s);
int dot_partial(int n, const double *x, const double *y, double *part,
                cudaStream_t s);
int dot(int n, const double *x, const double *y, double *part, double *out,
        cudaStream_t s);
int reduce_blocks(int n);

// PCG update (krylov.c:198-224 + norms of checks I/II): alpha = num/den
// (device scalars); u += alpha p; r += (-alpha) t; per-block partials of
// (r,r), max|u|, (u,u), (p,p) into part4 (4 x reduce_blocks(n)).
int pcg_update(int n, const double *num, const double *den, double *u,
               double *r, const double *p, const double *t, double *part4,
               cudaStream_t s);
// p = 1.0 * z + beta * p with beta = num/den computed on device.
int pcg_axpby(int n, const double *num, const double *den, const double *z,
              double *p, cudaStream_t s);
// y = x (copy), y = 0
template <typename T>
int vcopy(int n, const T *x, T *y, cudaStream_t s);
template <typename T>
int vzero(int n, T *y, cudaStream_t s);
// precision conversions
int d2f(int n, const double *x, float *y, cudaStream_t s, const unsigned char *act = nullptr);
int f2d(int n, const float *x, double *y, cudaStream_t s, const unsigned char *act = nullptr);
int csr_val_d2f(int nnz, const double *x, float *y, cudaStream_t s);
// entries != 0 per row, and the FP32 copy of those entries (row pointer ia32
// from a scan of the counts)
int csr_nonzero_count(int n, const int *ia, const double *a, int *cnt, cudaStream_t s);
int csr_nonzero_fill64(int n, const int *ia, const double *a, const int *ia32, double *a64,
                       cudaStream_t s);
int csr_nonzero_fill(int n, const int *ia, const int *ja, const double *a, const int *ia32,
                     int *ja32, float *a32, cudaStream_t s);

// Dense coarse solve y = Ainv x (row-major n x n FP64 inverse).
template <typename TI>
int dense_gemv(int n, const double *Ainv, const TI *x, TI *y, cudaStream_t s);

}  // namespace hzb
