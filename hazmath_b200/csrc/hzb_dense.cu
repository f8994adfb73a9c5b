// hzb_dense.cu -- coarsest-level dense factorisation (FP64).
//
// The coarsest matrix (<= coarse_dof rows, ~1-2k) is expanded to a dense
// lower triangle, factored A = L L^T with a blocked right-looking Cholesky
// (32-wide panels: diagonal block in shared memory, panel solve, tiled
// trailing update), L is inverted block row by block row (tiled product with
// the rows already inverted, then a 32-row triangular solve per column), and
// A^{-1} = L^{-T} L^{-1} is formed once, so that every V-cycle applies the
// coarse solve as one dense matrix-vector product (n^2 FP64 reads from L2)
// instead of two dependent triangular sweeps.  About 5 n/32 launches.
// This file may contract a*b+c into FMA: the coarse solve is a direct
// solve that agrees with the reference's sparse LDL^T only to rounding.
#include <algorithm>
#include "hzb_setup.cuh"

namespace hzb {

constexpr int NB = 32;

__global__ void k_dense_from_csr(int n, const int *__restrict__ ia,
                                 const int *__restrict__ ja,
                                 const double *__restrict__ a, double *D) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        for (int k = ia[i]; k < ia[i + 1]; ++k) D[(size_t)i * n + ja[k]] += a[k];
}

// Cholesky of the jb x jb diagonal block at (j0, j0), in shared memory.
// blockDim = (32, 32).
__global__ void k_potrf_diag(int n, int j0, int jb, double *D, int *bad) {
    __shared__ double T[NB][NB + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    T[ty][tx] = (tx < jb && ty < jb) ? D[(size_t)(j0 + ty) * n + j0 + tx] : 0.0;
    __syncthreads();
    for (int j = 0; j < jb; ++j) {
        const double piv = T[j][j];
        if (!(piv > 0.0)) {
            if (tx == 0 && ty == 0) *bad = 1;
            return;   // uniform: every thread read the same pivot
        }
        const double l = sqrt(piv);
        __syncthreads();
        if (ty == 0 && tx == j) T[j][j] = l;
        if (ty == 0 && tx > j && tx < jb) T[tx][j] /= l;
        __syncthreads();
        if (ty > j && tx > j && tx <= ty && ty < jb) T[ty][tx] -= T[ty][j] * T[tx][j];
        __syncthreads();
    }
    if (tx < jb && ty < jb && tx <= ty) D[(size_t)(j0 + ty) * n + j0 + tx] = T[ty][tx];
}

// L[i, j0:j0+jb] = A[i, j0:j0+jb] L_JJ^{-T} for the rows below the block
__global__ void k_trsm_panel(int n, int j0, int jb, double *D, const int *bad) {
    __shared__ double Ljj[NB][NB + 1];
    if (*bad) return;
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        const int r = t / NB, c = t % NB;
        Ljj[r][c] = (r < jb && c < jb) ? D[(size_t)(j0 + r) * n + j0 + c] : 0.0;
    }
    __syncthreads();
    const int i = j0 + jb + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x[NB];
    double *row = D + (size_t)i * n + j0;
#pragma unroll
    for (int c = 0; c < NB; ++c) x[c] = c < jb ? row[c] : 0.0;
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        if (c < jb) {
            double v = x[c];
            for (int k = 0; k < c; ++k) v -= x[k] * Ljj[c][k];
            x[c] = v / Ljj[c][c];
        }
    }
#pragma unroll
    for (int c = 0; c < NB; ++c)
        if (c < jb) row[c] = x[c];
}

// trailing update D[i][k] -= sum_t L[i][j0+t] L[k][j0+t], r0 <= k <= i < n,
// r0 = j0 + jb; 32 x 32 output tiles of the lower triangle.
__global__ void k_syrk_update(int n, int j0, int jb, double *D, const int *bad) {
    __shared__ double Li[NB][NB + 1], Lk[NB][NB + 1];
    if (*bad) return;
    const int r0 = j0 + jb;
    const int bi = blockIdx.y, bk = blockIdx.x;
    if (bk > bi) return;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = r0 + bi * NB + ty, k = r0 + bk * NB + tx;
    const int ii = r0 + bi * NB + tx;   // loader indices
    const int kk = r0 + bk * NB + tx;
    // load panel rows: Li[row][t] = L[r0 + bi*NB + row][j0 + t]
    for (int row = ty; row < NB; row += blockDim.y) {
        const int gi = r0 + bi * NB + row, gk = r0 + bk * NB + row;
        Li[row][tx] = (gi < n && tx < jb) ? D[(size_t)gi * n + j0 + tx] : 0.0;
        Lk[row][tx] = (gk < n && tx < jb) ? D[(size_t)gk * n + j0 + tx] : 0.0;
    }
    (void)ii; (void)kk;
    __syncthreads();
    if (i >= n || k >= n || k > i) return;
    double acc = 0.0;
#pragma unroll 8
    for (int t = 0; t < NB; ++t) acc += Li[ty][t] * Lk[tx][t];
    D[(size_t)i * n + k] -= acc;
}

// Inverse of L, block row I (rows i0..i0+ib): first
//   X[I, c] = -sum_{k=c..i0-1} L[I][k] X[k][c]   for columns c < i0
// (32 x 32 output tiles), then the diagonal solve below.
__global__ void k_trinv_gemm(int n, int i0, int ib, const double *__restrict__ L,
                             double *X) {
    __shared__ double Ls[NB][NB + 1], Xs[NB][NB + 1];
    const int c0 = blockIdx.x * NB;
    if (c0 >= i0) return;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int r = i0 + ty, c = c0 + tx;
    double acc = 0.0;
    for (int k0 = c0; k0 < i0; k0 += NB) {
        const int lk = k0 + tx, xk = k0 + ty;
        Ls[ty][tx] = (ty < ib && lk < i0) ? L[(size_t)r * n + lk] : 0.0;
        Xs[ty][tx] = (xk < i0 && c < n) ? X[(size_t)xk * n + c] : 0.0;
        __syncthreads();
#pragma unroll 8
        for (int t = 0; t < NB; ++t) acc += Ls[ty][t] * Xs[t][tx];
        __syncthreads();
    }
    if (ty < ib && c < i0) X[(size_t)r * n + c] = -acc;
}

// X[I, c] = L_II^{-1} rhs(c) for every column c < i0 + ib, where rhs is the
// tile product above (c < i0) or the identity (c >= i0).
__global__ void k_trinv_diag(int n, int i0, int ib, const double *__restrict__ L,
                             double *X) {
    __shared__ double Lii[NB][NB + 1];
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        const int rr = t / NB, cc = t % NB;
        Lii[rr][cc] = (rr < ib && cc < ib) ? L[(size_t)(i0 + rr) * n + i0 + cc] : 0.0;
    }
    __syncthreads();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= i0 + ib) return;
    double x[NB];
#pragma unroll
    for (int rr = 0; rr < NB; ++rr) {
        if (rr < ib) {
            double v = (c < i0) ? X[(size_t)(i0 + rr) * n + c] : (c == i0 + rr ? 1.0 : 0.0);
            for (int t = 0; t < rr; ++t) v -= Lii[rr][t] * x[t];
            x[rr] = v / Lii[rr][rr];
        } else {
            x[rr] = 0.0;
        }
    }
#pragma unroll
    for (int rr = 0; rr < NB; ++rr)
        if (rr < ib) X[(size_t)(i0 + rr) * n + c] = x[rr];
}

// Ainv = X^T X (16 x 16 tiles; X lower triangular)
__global__ void k_xtx(int n, const double *__restrict__ X, double *Ainv) {
    __shared__ double ta[16][17], tb[16][17];
    const int a = blockIdx.y * 16 + threadIdx.y;   // output row
    const int b = blockIdx.x * 16 + threadIdx.x;   // output column
    const int i0 = max(blockIdx.y, blockIdx.x) * 16;   // X[i][a] = 0 for i < a
    double acc = 0.0;
    for (int it = i0; it < n; it += 16) {
        const int ir = it + threadIdx.y;
        const int ca = blockIdx.y * 16 + threadIdx.x;
        const int cb = blockIdx.x * 16 + threadIdx.x;
        ta[threadIdx.y][threadIdx.x] = (ir < n && ca < n) ? X[(size_t)ir * n + ca] : 0.0;
        tb[threadIdx.y][threadIdx.x] = (ir < n && cb < n) ? X[(size_t)ir * n + cb] : 0.0;
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16; ++q) acc += ta[q][threadIdx.y] * tb[q][threadIdx.x];
        __syncthreads();
    }
    if (a < n && b < n) Ainv[(size_t)a * n + b] = acc;
}

int dense_inverse(const DCsr<double> &A, double **Ainv_out, cudaStream_t s) {
    const int n = A.n;
    *Ainv_out = nullptr;
    double *D = nullptr, *X = nullptr, *Ainv = nullptr;
    int *bad = nullptr;
    const size_t nn = (size_t)n * n;
    int rc = SUCCESS, hbad = 0;
    cudaError_t e;
    if ((rc = dalloc(&D, nn))) goto done;
    if ((rc = dalloc(&X, nn))) goto done;
    if ((rc = dalloc(&Ainv, nn))) goto done;
    if ((rc = dalloc(&bad, 1))) goto done;
    cudaMemsetAsync(D, 0, nn * sizeof(double), s);
    cudaMemsetAsync(X, 0, nn * sizeof(double), s);
    cudaMemsetAsync(bad, 0, sizeof(int), s);
    k_dense_from_csr<<<grid_for(n), 256, 0, s>>>(n, A.ia, A.ja, A.val, D);
    count_launch();
    for (int j0 = 0; j0 < n; j0 += NB) {
        const int jb = std::min(NB, n - j0);
        const int rest = n - j0 - jb;
        k_potrf_diag<<<1, dim3(NB, NB), 0, s>>>(n, j0, jb, D, bad);
        count_launch();
        if (rest > 0) {
            k_trsm_panel<<<div_up(rest, 128), 128, 0, s>>>(n, j0, jb, D, bad);
            const int nt = div_up(rest, NB);
            k_syrk_update<<<dim3(nt, nt), dim3(NB, NB), 0, s>>>(n, j0, jb, D, bad);
            count_launch(2);
        }
    }
    e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
    if (hbad) { set_error_msg("coarse matrix is not positive definite"); rc = ERROR_DATA_ZERODIAG; goto done; }
    for (int i0 = 0; i0 < n; i0 += NB) {
        const int ib = std::min(NB, n - i0);
        if (i0 > 0) {
            k_trinv_gemm<<<div_up(i0, NB), dim3(NB, NB), 0, s>>>(n, i0, ib, D, X);
            count_launch();
        }
        k_trinv_diag<<<div_up(i0 + ib, 128), 128, 0, s>>>(n, i0, ib, D, X);
        count_launch();
    }
    {
        dim3 blk(16, 16), grd(div_up(n, 16), div_up(n, 16));
        k_xtx<<<grd, blk, 0, s>>>(n, X, Ainv);
        count_launch();
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
    *Ainv_out = Ainv;
    Ainv = nullptr;
done:
    dfree(D); dfree(X); dfree(Ainv); dfree(bad);
    return rc;
}

}  // namespace hzb
