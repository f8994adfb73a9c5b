// hzb_dense.cu -- coarsest-level dense factorisation (FP64).
//
// The coarsest matrix (<= coarse_dof rows, ~1-2k) is expanded to a dense
// lower triangle, factored A = L L^T column by column (right-looking), and
// its inverse A^{-1} = L^{-T} L^{-1} is formed once, so that every V-cycle
// applies the coarse solve as one dense matrix-vector product (n^2 FP64
// reads from L2) instead of two dependent triangular sweeps.
// This file may contract a*b+c into FMA: the coarse solve is a direct
// solve that agrees with the reference's sparse LDL^T only to rounding.
#include "hzb_setup.cuh"

namespace hzb {

__global__ void k_dense_from_csr(int n, const int *__restrict__ ia,
                                 const int *__restrict__ ja,
                                 const double *__restrict__ a, double *D) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        for (int k = ia[i]; k < ia[i + 1]; ++k) D[(size_t)i * n + ja[k]] += a[k];
}

__global__ void k_chol_pivot(int n, int j, double *D, int *bad) {
    // single block: every thread reads the pivot before thread 0 replaces it
    const double piv = D[(size_t)j * n + j];
    if (!(piv > 0.0)) {
        if (threadIdx.x == 0) *bad = 1;
        return;
    }
    const double l = sqrt(piv);
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x)
        D[(size_t)i * n + j] /= l;
    __syncthreads();
    if (threadIdx.x == 0) D[(size_t)j * n + j] = l;
}

// trailing update of the lower triangle: D[i][k] -= L[i][j] L[k][j], j < k <= i
__global__ void k_chol_update(int n, int j, double *D, const int *bad) {
    if (*bad) return;
    const int k = j + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int i = j + 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (k >= n || i >= n || k > i) return;
    D[(size_t)i * n + k] -= D[(size_t)i * n + j] * D[(size_t)k * n + j];
}

// X = L^{-1}, one thread per column (X lower triangular)
__global__ void k_tri_inv(int n, const double *__restrict__ L, double *X) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += gridDim.x * blockDim.x) {
        X[(size_t)c * n + c] = 1.0 / L[(size_t)c * n + c];
        for (int i = c + 1; i < n; ++i) {
            double t = 0.0;
            for (int k = c; k < i; ++k) t += L[(size_t)i * n + k] * X[(size_t)k * n + c];
            X[(size_t)i * n + c] = -t / L[(size_t)i * n + i];
        }
    }
}

// Ainv = X^T X (16 x 16 tiles)
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
    for (int j = 0; j < n; ++j) {
        const int m = n - j - 1;
        k_chol_pivot<<<1, 256, 0, s>>>(n, j, D, bad);
        if (m > 0) {
            dim3 blk(32, 8), grd(div_up(m, 32), div_up(m, 8));
            k_chol_update<<<grd, blk, 0, s>>>(n, j, D, bad);
        }
        count_launch(2);
    }
    e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
    if (hbad) { set_error_msg("coarse matrix is not positive definite"); rc = ERROR_DATA_ZERODIAG; goto done; }
    k_tri_inv<<<div_up(n, 64), 64, 0, s>>>(n, D, X);
    {
        dim3 blk(16, 16), grd(div_up(n, 16), div_up(n, 16));
        k_xtx<<<grd, blk, 0, s>>>(n, X, Ainv);
    }
    count_launch(2);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
    *Ainv_out = Ainv;
    Ainv = nullptr;
done:
    dfree(D); dfree(X); dfree(Ainv); dfree(bad);
    return rc;
}

}  // namespace hzb
