// hzb_sell.cu -- the FP32 cycle's sliced-ELL schedule.
//
// A level's FP32 matrix is also kept as 32-row slices stored column-major:
// entry u of the row in slot r of slice s sits at col/val[ptr[s] + 32 u +
// (r mod 32)], so the 32 threads of a warp, one row each, read entry u of
// their 32 rows as one coalesced 128-byte line -- no shared-memory staging
// (full occupancy) and no lanes to combine.  A slice is as wide as its
// longest row; rows are ordered by length (descending, ties by index)
// inside each 256-row window, so the rows of a slice have nearly equal
// lengths, and a thread stops at its own row's length, so the padding is
// never read.  Each row's entries keep their CSR order and one thread sums
// them in that order.  For the FP32 cycle, where it competes with the staged
// bundles and the lanes-per-row kernels in the per-level autotuner.
#include "hzb_setup.cuh"
#include <climits>

namespace hzb {

namespace {
constexpr int SELL_WIN = 256;   // rows sorted together (one CTA)
constexpr int SELL_C = 32;      // rows per slice

// One CTA per window: slot of each row by its rank (longer first, then by
// index), the slice widths (the first slot of a slice holds its longest
// row), and the slot -> row map (-1 past n).
__global__ void __launch_bounds__(SELL_WIN)
k_sell_order(int n, const int *__restrict__ ia, int *srow, int *slen, int *width32,
             unsigned long long *total) {
    __shared__ int len[SELL_WIN];
    const int t = threadIdx.x;
    const int i = blockIdx.x * SELL_WIN + t;
    const int li = i < n ? ia[i + 1] - ia[i] : -1;
    len[t] = li;
    __syncthreads();
    int rank = 0;
    for (int q = 0; q < SELL_WIN; ++q) {
        const int lq = len[q];
        rank += lq > li || (lq == li && q < t);
    }
    const int slot = blockIdx.x * SELL_WIN + rank;
    srow[slot] = i < n ? i : -1;
    slen[slot] = li > 0 ? li : 0;
    if (rank % SELL_C == 0) {
        width32[slot / SELL_C] = (li > 0 ? li : 0) * SELL_C;
        atomicAdd(total, (unsigned long long)(li > 0 ? li : 0) * SELL_C);
    }
}

__global__ void k_sell_fill(int npad, const int *__restrict__ ptr, const int *__restrict__ srow,
                            const int *__restrict__ slen, const int *__restrict__ ia,
                            const int *__restrict__ ja, const float *__restrict__ a, int *col,
                            float *val) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < npad; r += gridDim.x * blockDim.x) {
        const int s = r / SELL_C, lane = r % SELL_C;
        const int w = (ptr[s + 1] - ptr[s]) / SELL_C;
        const int i = srow[r], len = slen[r];
        const int k0 = i >= 0 ? ia[i] : 0;
        for (int u = 0; u < w; ++u) {
            const size_t q = (size_t)ptr[s] + (size_t)u * SELL_C + lane;
            col[q] = u < len ? ja[k0 + u] : 0;
            val[q] = u < len ? a[k0 + u] : 0.f;
        }
    }
}

// Row sum of slot r's row in CSR order, eight entries' loads and gathers in
// flight at a time.  L1: t -= v x and d += |v| (t starts at b_i); else
// t += v x.
template <bool L1>
__device__ __forceinline__ void sell_row(int base, int len, const int *__restrict__ col,
                                         const float *__restrict__ val,
                                         const float *__restrict__ x, float &t, float &d) {
    constexpr int G = 8;
    for (int u0 = 0; u0 < len; u0 += G) {
        int c[G];
        float v[G], xv[G];
#pragma unroll
        for (int q = 0; q < G; ++q) {
            c[q] = 0;
            v[q] = 0.f;
            if (u0 + q < len) {
                const int k = base + (u0 + q) * SELL_C;
                c[q] = __ldcs(col + k);
                v[q] = __ldcs(val + k);
            }
        }
#pragma unroll
        for (int q = 0; q < G; ++q) xv[q] = u0 + q < len ? __ldg(x + c[q]) : 0.f;
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if (u0 + q < len) {
                if (L1) {
                    t -= v[q] * xv[q];
                    d += fabsf(v[q]);
                } else {
                    t += v[q] * xv[q];
                }
            }
        }
    }
}

__global__ void __launch_bounds__(SELL_WIN)
k_l1_sell(int npad, const int *__restrict__ ptr, const int *__restrict__ srow,
          const int *__restrict__ slen, const int *__restrict__ col,
          const float *__restrict__ val, const float *__restrict__ b,
          const float *__restrict__ x, float *__restrict__ xn, const float *__restrict__ omega) {
    const int r = blockIdx.x * SELL_WIN + threadIdx.x;
    if (r >= npad) return;
    const int i = srow[r];
    if (i < 0) return;
    float t = b[i], d = 0.f;
    sell_row<true>(ptr[r / SELL_C] + r % SELL_C, slen[r], col, val, x, t, d);
    float xi = x[i];
    if (fabsf(d) > float(SMALLREAL)) xi += omega ? omega[i] * (t / d) : t / d;
    xn[i] = xi;
}

template <int MODE>
__global__ void __launch_bounds__(SELL_WIN)
k_spmv_sell(int npad, const int *__restrict__ ptr, const int *__restrict__ srow,
            const int *__restrict__ slen, const int *__restrict__ col,
            const float *__restrict__ val, const float *__restrict__ x,
            const float *__restrict__ b, float *__restrict__ y, float alpha) {
    const int r = blockIdx.x * SELL_WIN + threadIdx.x;
    if (r >= npad) return;
    const int i = srow[r];
    if (i < 0) return;
    float t = 0.f, d = 0.f;
    sell_row<false>(ptr[r / SELL_C] + r % SELL_C, slen[r], col, val, x, t, d);
    if (MODE == SPMV_RES) {
        y[i] = b[i] - t;
    } else if (MODE == SPMV_AXPY) {
        if (alpha == 1.f) y[i] += t;
        else if (alpha == -1.f) y[i] -= t;
        else y[i] += t * alpha;
    } else {
        y[i] = t;
    }
}
}  // namespace

int sell_pad_rows(int n) { return (n + SELL_WIN - 1) / SELL_WIN * SELL_WIN; }

int sell_build(int n, const int *ia, const int *ja, const float *a, SellArrays *out,
               cudaStream_t s) {
    *out = SellArrays();
    if (n <= 0) return SUCCESS;
    const int npad = sell_pad_rows(n), nsl = npad / SELL_C;
    int *w32 = nullptr, *tmp = nullptr;
    unsigned long long *dtot = nullptr, htot = 0;
    SellArrays S;
    S.npad = npad;
    int rc = SUCCESS;
    if ((rc = dalloc(&S.row, npad)) || (rc = dalloc(&S.len, npad)) ||
        (rc = dalloc(&S.ptr, nsl + 1)) || (rc = dalloc(&w32, nsl)) ||
        (rc = dalloc(&tmp, scan_tmp_size(nsl + 1))) || (rc = dalloc(&dtot, 1)))
        goto fail;
    if (cudaMemsetAsync(dtot, 0, sizeof(unsigned long long), s) != cudaSuccess) {
        rc = ERROR_SOLVER_MISC;
        goto fail;
    }
    k_sell_order<<<npad / SELL_WIN, SELL_WIN, 0, s>>>(n, ia, S.row, S.len, w32, dtot);
    count_launch();
    if (cudaMemcpyAsync(&htot, dtot, sizeof(htot), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        rc = ERROR_SOLVER_MISC;
        goto fail;
    }
    // the slice offsets are int: a level whose padded slices would not fit
    // gets no copy (the bundles and lanes kernels serve it)
    if (htot > (unsigned long long)(INT_MAX / 2)) goto fail;
    if ((rc = scan_exclusive(w32, S.ptr, nsl, tmp, s))) goto fail;
    if ((rc = dalloc(&S.col, htot > 0 ? htot : 1)) || (rc = dalloc(&S.val, htot > 0 ? htot : 1)))
        goto fail;
    k_sell_fill<<<grid_for(npad), 256, 0, s>>>(npad, S.ptr, S.row, S.len, ia, ja, a, S.col,
                                               S.val);
    count_launch();
    HZB_LAUNCH_CHECK();
    dfree(w32);
    dfree(tmp);
    dfree(dtot);
    *out = S;
    return SUCCESS;
fail:
    dfree(w32);
    dfree(tmp);
    dfree(dtot);
    S.release();
    return rc;
}

void SellArrays::release() {
    dfree(ptr);
    dfree(row);
    dfree(len);
    dfree(col);
    dfree(val);
    npad = 0;
}

int sell_l1_sweep(const DCsr<float> &A, const float *b, const float *x, float *xn,
                  const float *omega, cudaStream_t s) {
    const SellView &V = A.sell;
    k_l1_sell<<<V.npad / SELL_WIN, SELL_WIN, 0, s>>>(V.npad, V.ptr, V.row, V.len, V.col, V.val,
                                                     b, x, xn, omega);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

int sell_spmv(const DCsr<float> &A, int mode, const float *x, const float *b, float *y,
              float alpha, cudaStream_t s) {
    const SellView &V = A.sell;
    const int g = V.npad / SELL_WIN;
    switch (mode) {
    case SPMV_RES:
        k_spmv_sell<SPMV_RES><<<g, SELL_WIN, 0, s>>>(V.npad, V.ptr, V.row, V.len, V.col, V.val,
                                                     x, b, y, alpha);
        break;
    case SPMV_AXPY:
        k_spmv_sell<SPMV_AXPY><<<g, SELL_WIN, 0, s>>>(V.npad, V.ptr, V.row, V.len, V.col, V.val,
                                                      x, b, y, alpha);
        break;
    default:
        k_spmv_sell<SPMV_Y><<<g, SELL_WIN, 0, s>>>(V.npad, V.ptr, V.row, V.len, V.col, V.val, x,
                                                   b, y, alpha);
        break;
    }
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

}  // namespace hzb
