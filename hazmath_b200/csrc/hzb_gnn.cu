// hzb_gnn.cu -- message-passing network that predicts per-row l1-Jacobi
// weights omega_i in (0, 2) from the fine-level matrix, with its forward and
// backward kernels (BF16 weights and activations, FP32 accumulation).
//
// Features (scale-invariant): node i: [a_ii/l1_i, sum_{j!=i} a_ij / l1_i,
// max_{j!=i} |a_ij| / l1_i, 1]; edge (i,j), j != i: [a_ij / sqrt(a_ii a_jj),
// clamp(0.5 log(a_jj / a_ii), -4, 4)].  Width H = 32, three layers:
//     h0 = relu(W_in x + b_in)
//     P_l = h_{l-1} U_l^T                              (tensor cores)
//     M_l,i = mean_{j != i} relu(P_l,j + V_l e_ij + c_l)
//     y_l = [h_{l-1}, M_l] W_l^T + b_l                 (tensor cores)
//     h_l = relu(y_l) + h_{l-1}
//     omega_i = 2 sigmoid(w_o . h_3,i + b_o)
// The output layer starts at zero, so an untrained network returns omega = 1,
// the reference's l1-Jacobi.  Dense layers use mma.sync m16n8k16 BF16 tiles
// (FP32 accumulate); they are memory-bound (K, N <= 64), so the legacy warp
// MMA already saturates HBM for them.  Weight gradients are FP32 block
// reductions.
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "hzb_solver.cuh"

namespace hzb {

constexpr int H = 32;
constexpr int OFF_WIN = 0, OFF_BIN = 128;
constexpr int LAYER = 32 * 32 + 32 * 2 + 32 + 32 * 64 + 32;   // 3200
constexpr int L_U = 0, L_V = 1024, L_C = 1088, L_W = 1120, L_B = 3168;
constexpr int OFF_L0 = 160;
constexpr int OFF_WO = OFF_L0 + 3 * LAYER;   // 9760
constexpr int OFF_BO = OFF_WO + 32;          // 9792
constexpr int NPARAM = OFF_BO + 1;           // 9793

typedef __nv_bfloat16 bf16;

}  // namespace hzb

struct hzb_gnn {
    float *params = nullptr, *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
    hzb::bf16 *Ubf[3] = {nullptr}, *UTbf[3] = {nullptr}, *Wbf[3] = {nullptr},
              *WTbf[3] = {nullptr};
    int step = 0;
    // activations for the last forward (n rows)
    int n = 0;
    float *feats = nullptr, *omega = nullptr;
    double *diag = nullptr;
    hzb::bf16 *h[4] = {nullptr}, *P[3] = {nullptr}, *M[3] = {nullptr}, *y[3] = {nullptr};
    float *dH = nullptr, *dY = nullptr, *dP = nullptr, *dM = nullptr;
    cudaStream_t s = nullptr;
};

namespace hzb {

// ---------------------------------------------------------------------------
// warp-level BF16 MMA tile: 16 rows x N columns, K deep
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<unsigned *>(&v);
}
__device__ __forceinline__ unsigned pair_bf16(const bf16 *p) {
    return *reinterpret_cast<const unsigned *>(p);
}

__device__ __forceinline__ void mma16816(float *c, const unsigned *a, unsigned b0,
                                         unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc[nt][4] += A(16 x K) * B(K x N), Bt (N x K, row-major) in shared memory.
// afetch(r, c) returns the packed BF16 pair A[r][c], A[r][c+1] of the tile.
template <int K, int N, typename AF>
__device__ __forceinline__ void warp_tile(AF afetch, const bf16 *Bt, float acc[N / 8][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int kk = 0; kk < K / 16; ++kk) {
        const int c0 = kk * 16 + tg * 2;
        unsigned a[4];
        a[0] = afetch(g, c0);
        a[1] = afetch(g + 8, c0);
        a[2] = afetch(g, c0 + 8);
        a[3] = afetch(g + 8, c0 + 8);
#pragma unroll
        for (int nt = 0; nt < N / 8; ++nt) {
            const bf16 *brow = Bt + (nt * 8 + g) * K + c0;
            mma16816(acc[nt], a, pair_bf16(brow), pair_bf16(brow + 8));
        }
    }
}

template <int K, int N>
__device__ __forceinline__ void stage_bt(const bf16 *Bt, bf16 *sB) {
    for (int t = threadIdx.x; t < K * N; t += blockDim.x) sB[t] = Bt[t];
    __syncthreads();
}

// P = h U^T  (K = 32, N = 32), stored BF16
__global__ void k_gemm_P(int n, const bf16 *__restrict__ h, const bf16 *__restrict__ Ubf,
                         bf16 *__restrict__ P) {
    __shared__ __align__(16) bf16 sB[32 * 32];
    stage_bt<32, 32>(Ubf, sB);
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row0 = warp * 16;
    if (row0 >= n) return;
    auto af = [&](int r, int c) -> unsigned {
        const int rr = row0 + r;
        return rr < n ? pair_bf16(h + (size_t)rr * 32 + c) : 0u;
    };
    float acc[4][4] = {};
    warp_tile<32, 32>(af, sB, acc);
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const int col = nt * 8 + tg * 2;
        const int r0 = row0 + g, r1 = row0 + g + 8;
        if (r0 < n) *reinterpret_cast<unsigned *>(P + (size_t)r0 * 32 + col) = pack_bf16(acc[nt][0], acc[nt][1]);
        if (r1 < n) *reinterpret_cast<unsigned *>(P + (size_t)r1 * 32 + col) = pack_bf16(acc[nt][2], acc[nt][3]);
    }
}

// y = [h, M] W^T + b; h_new = relu(y) + h   (K = 64, N = 32)
__global__ void k_gemm_Y(int n, const bf16 *__restrict__ h, const bf16 *__restrict__ M,
                         const bf16 *__restrict__ Wbf, const float *__restrict__ b,
                         bf16 *__restrict__ y, bf16 *__restrict__ hn) {
    __shared__ __align__(16) bf16 sB[32 * 64];
    stage_bt<64, 32>(Wbf, sB);
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row0 = warp * 16;
    if (row0 >= n) return;
    auto af = [&](int r, int c) -> unsigned {
        const int rr = row0 + r;
        if (rr >= n) return 0u;
        return c < 32 ? pair_bf16(h + (size_t)rr * 32 + c) : pair_bf16(M + (size_t)rr * 32 + c - 32);
    };
    float acc[4][4] = {};
    warp_tile<64, 32>(af, sB, acc);
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const int col = nt * 8 + tg * 2;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int r = row0 + g + half * 8;
            if (r >= n) continue;
            const float y0 = acc[nt][2 * half] + b[col], y1 = acc[nt][2 * half + 1] + b[col + 1];
            const float h0 = __bfloat162float(h[(size_t)r * 32 + col]);
            const float h1 = __bfloat162float(h[(size_t)r * 32 + col + 1]);
            *reinterpret_cast<unsigned *>(y + (size_t)r * 32 + col) = pack_bf16(y0, y1);
            *reinterpret_cast<unsigned *>(hn + (size_t)r * 32 + col) =
                pack_bf16(fmaxf(y0, 0.f) + h0, fmaxf(y1, 0.f) + h1);
        }
    }
}

// dX = bf16(dY) W (K = 32, N = 64): dH += dX[:, :32], dM = dX[:, 32:]
__global__ void k_gemm_dX(int n, const float *__restrict__ dY, const bf16 *__restrict__ WT,
                          float *__restrict__ dH, float *__restrict__ dM) {
    __shared__ __align__(16) bf16 sB[64 * 32];
    stage_bt<32, 64>(WT, sB);
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row0 = warp * 16;
    if (row0 >= n) return;
    auto af = [&](int r, int c) -> unsigned {
        const int rr = row0 + r;
        return rr < n ? pack_bf16(dY[(size_t)rr * 32 + c], dY[(size_t)rr * 32 + c + 1]) : 0u;
    };
    float acc[8][4] = {};
    warp_tile<32, 64>(af, sB, acc);
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + tg * 2;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int r = row0 + g + half * 8;
            if (r >= n) continue;
            if (col < 32) {
                dH[(size_t)r * 32 + col] += acc[nt][2 * half];
                dH[(size_t)r * 32 + col + 1] += acc[nt][2 * half + 1];
            } else {
                dM[(size_t)r * 32 + col - 32] = acc[nt][2 * half];
                dM[(size_t)r * 32 + col - 31] = acc[nt][2 * half + 1];
            }
        }
    }
}

// dH += bf16(dP) U  (K = 32, N = 32)
__global__ void k_gemm_dH(int n, const float *__restrict__ dP, const bf16 *__restrict__ UT,
                          float *__restrict__ dH) {
    __shared__ __align__(16) bf16 sB[32 * 32];
    stage_bt<32, 32>(UT, sB);
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row0 = warp * 16;
    if (row0 >= n) return;
    auto af = [&](int r, int c) -> unsigned {
        const int rr = row0 + r;
        return rr < n ? pack_bf16(dP[(size_t)rr * 32 + c], dP[(size_t)rr * 32 + c + 1]) : 0u;
    };
    float acc[4][4] = {};
    warp_tile<32, 32>(af, sB, acc);
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const int col = nt * 8 + tg * 2;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int r = row0 + g + half * 8;
            if (r >= n) continue;
            dH[(size_t)r * 32 + col] += acc[nt][2 * half];
            dH[(size_t)r * 32 + col + 1] += acc[nt][2 * half + 1];
        }
    }
}

// ---------------------------------------------------------------------------
// features, input layer, messages, output (warp per row, lane = feature)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void edge_feat(double aij, double aii, double ajj, float &e0,
                                          float &e1) {
    e0 = (float)(aij / sqrt(fabs(aii * ajj)));
    float l = (float)(0.5 * log(fabs(ajj / aii)));
    e1 = fminf(4.f, fmaxf(-4.f, l));
}

__global__ void k_gnn_diag(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                           const double *__restrict__ a, double *diag, float *feats) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        double d = 0.0, l1 = 0.0, off = 0.0, mx = 0.0;
        bool got = false;
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            const double v = a[k];
            l1 += fabs(v);
            if (ja[k] == i) { if (!got) { d = v; got = true; } }
            else { off += v; mx = fmax(mx, fabs(v)); }
        }
        diag[i] = d;
        const double il = l1 > 0 ? 1.0 / l1 : 0.0;
        feats[4 * i + 0] = (float)(d * il);
        feats[4 * i + 1] = (float)(off * il);
        feats[4 * i + 2] = (float)(mx * il);
        feats[4 * i + 3] = 1.0f;
    }
}

__global__ void k_gnn_input(int n, const float *__restrict__ feats,
                            const float *__restrict__ prm, bf16 *h0) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float *W = prm + OFF_WIN, *b = prm + OFF_BIN;
    for (int i = warp; i < n; i += nw) {
        float v = b[lane];
#pragma unroll
        for (int k = 0; k < 4; ++k) v += W[lane * 4 + k] * feats[4 * i + k];
        h0[(size_t)i * 32 + lane] = __float2bfloat16_rn(fmaxf(v, 0.f));
    }
}

// Warp per row, lane = channel.  The row's edges are loaded one per lane
// (features computed once per edge), then broadcast four at a time so four
// neighbour rows of P are gathered together; the sum runs in CSR order.
__global__ void k_gnn_message(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                              const double *__restrict__ a, const double *__restrict__ diag,
                              const bf16 *__restrict__ P, const float *__restrict__ lay,
                              bf16 *M) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float v0 = lay[L_V + 2 * lane], v1 = lay[L_V + 2 * lane + 1], c = lay[L_C + lane];
    for (int i = warp; i < n; i += nw) {
        float s = 0.f;
        int deg = 0;
        const double aii = diag[i];
        const int b1 = ia[i + 1];
        for (int base = ia[i]; base < b1; base += 32) {
            const int k = base + lane;
            int j = -1;
            float e0 = 0.f, e1 = 0.f;
            if (k < b1) {
                j = ja[k];
                if (j != i) edge_feat(a[k], aii, diag[j], e0, e1);
                else j = -1;
            }
            unsigned m = __ballot_sync(0xffffffffu, j >= 0);
            deg += __popc(m);
            while (m) {
                int src[4], jj[4];
                int cnt = 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    src[u] = m ? __ffs(m) - 1 : 0;
                    cnt += m != 0u;
                    m &= m - 1u;
                }
                float q[4], f0[4], f1[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    jj[u] = __shfl_sync(0xffffffffu, j, src[u]);
                    f0[u] = __shfl_sync(0xffffffffu, e0, src[u]);
                    f1[u] = __shfl_sync(0xffffffffu, e1, src[u]);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    q[u] = u < cnt ? __bfloat162float(P[(size_t)jj[u] * 32 + lane]) : 0.f;
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (u < cnt) s += fmaxf(q[u] + v0 * f0[u] + v1 * f1[u] + c, 0.f);
            }
        }
        M[(size_t)i * 32 + lane] = __float2bfloat16_rn(deg ? s / deg : 0.f);
    }
}

__global__ void k_gnn_output(int n, const bf16 *__restrict__ h3, const float *__restrict__ prm,
                             float *omega) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float wo = prm[OFF_WO + lane], bo = prm[OFF_BO];
    for (int i = warp; i < n; i += nw) {
        float z = warp_sum(wo * __bfloat162float(h3[(size_t)i * 32 + lane])) + bo;
        z = fminf(12.f, fmaxf(-12.f, z));   // omega stays strictly inside (0, 2)
        if (lane == 0) omega[i] = 2.0f / (1.0f + expf(-z));
    }
}

// ---------------------------------------------------------------------------
// backward kernels
// ---------------------------------------------------------------------------
// per-lane partials of a warp-per-row kernel, reduced over the block's warps
// and added to the gradient
__device__ __forceinline__ void block_add(float v, float *sh, float *dst) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    sh[wid * 32 + lane] = v;
    __syncthreads();
    if (wid == 0) {
        float s = 0.f;
        for (int w = 0; w < nw; ++w) s += sh[w * 32 + lane];
        atomicAdd(dst + lane, s);
    }
    __syncthreads();
}

// dz = domega * omega (1 - omega / 2); dH3 = dz w_o; grads of w_o, b_o
__global__ void k_gnn_output_bwd(int n, const float *__restrict__ domega,
                                 const float *__restrict__ omega, const bf16 *__restrict__ h3,
                                 const float *__restrict__ prm, float *dH, float *grad) {
    __shared__ float sh[8 * 32];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float wo = prm[OFF_WO + lane];
    float gw = 0.f, gb = 0.f;
    for (int i = warp; i < n; i += nw) {
        const float om = omega[i];
        const float dz = domega[i] * om * (1.f - 0.5f * om);
        dH[(size_t)i * 32 + lane] = dz * wo;
        gw += dz * __bfloat162float(h3[(size_t)i * 32 + lane]);
        if (lane == 0) gb += dz;
    }
    block_add(gw, sh, grad + OFF_WO);
    gb = warp_sum(gb);
    if ((threadIdx.x & 31) == 0) atomicAdd(grad + OFF_BO, gb);
}

// dY = dH * [y > 0]; grad b += sum dY
__global__ void k_gnn_relu_bwd(int n, const float *__restrict__ dH, const bf16 *__restrict__ y,
                               float *dY, float *gradb) {
    __shared__ float sh[8 * 32];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    float gb = 0.f;
    for (int i = warp; i < n; i += nw) {
        const size_t q = (size_t)i * 32 + lane;
        const float d = __bfloat162float(y[q]) > 0.f ? dH[q] : 0.f;
        dY[q] = d;
        gb += d;
    }
    block_add(gb, sh, gradb);
}

// grad[o][k] += sum_i dY[i][o] X[i][k]; X = [X0, X1] (BF16, 32 columns each),
// K = 32 or 64.  Block: 256 threads, 64-row tiles.
template <int K>
__global__ void k_gnn_wgrad(int n, const float *__restrict__ dY, const bf16 *__restrict__ X0,
                            const bf16 *__restrict__ X1, float *grad) {
    __shared__ float sY[64][33];
    __shared__ float sX[64][K + 1];
    constexpr int OUT = 32 * K, PER = OUT / 256;
    float acc[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) acc[q] = 0.f;
    for (int r0 = blockIdx.x * 64; r0 < n; r0 += gridDim.x * 64) {
        for (int t = threadIdx.x; t < 64 * 32; t += 256) {
            const int r = t / 32, c = t % 32, i = r0 + r;
            sY[r][c] = i < n ? dY[(size_t)i * 32 + c] : 0.f;
        }
        for (int t = threadIdx.x; t < 64 * K; t += 256) {
            const int r = t / K, c = t % K, i = r0 + r;
            float v = 0.f;
            if (i < n) v = __bfloat162float(c < 32 ? X0[(size_t)i * 32 + c] : X1[(size_t)i * 32 + c - 32]);
            sX[r][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int o = (threadIdx.x + q * 256) / K, k = (threadIdx.x + q * 256) % K;
            float s = 0.f;
            for (int r = 0; r < 64; ++r) s += sY[r][o] * sX[r][k];
            acc[q] += s;
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) atomicAdd(grad + threadIdx.x + q * 256, acc[q]);
}

// message backward: dm_ij = dM_i / deg_i * [q_ij > 0]; dP_j += dm_ij;
// grads of V, c
__global__ void k_gnn_message_bwd(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                  const double *__restrict__ a, const double *__restrict__ diag,
                                  const bf16 *__restrict__ P, const float *__restrict__ lay,
                                  const float *__restrict__ dM, float *dP, float *glay) {
    __shared__ float sh[8 * 32];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float v0 = lay[L_V + 2 * lane], v1 = lay[L_V + 2 * lane + 1], c = lay[L_C + lane];
    float g0 = 0.f, g1 = 0.f, gc = 0.f;
    for (int i = warp; i < n; i += nw) {
        int deg = 0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) deg += ja[k] != i;
        if (!deg) continue;
        const float gm = dM[(size_t)i * 32 + lane] / deg;
        const double aii = diag[i];
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            const int j = ja[k];
            if (j == i) continue;
            float e0, e1;
            edge_feat(a[k], aii, diag[j], e0, e1);
            const float q = __bfloat162float(P[(size_t)j * 32 + lane]) + v0 * e0 + v1 * e1 + c;
            if (q > 0.f) {
                atomicAdd(dP + (size_t)j * 32 + lane, gm);
                g0 += gm * e0;
                g1 += gm * e1;
                gc += gm;
            }
        }
    }
    // V is stored [lane][2]: reduce the two components separately
    const int wid = threadIdx.x >> 5, nwb = blockDim.x >> 5;
    sh[wid * 32 + lane] = g0;
    __syncthreads();
    if (wid == 0) {
        float s = 0.f;
        for (int w = 0; w < nwb; ++w) s += sh[w * 32 + lane];
        atomicAdd(glay + L_V + 2 * lane, s);
    }
    __syncthreads();
    sh[wid * 32 + lane] = g1;
    __syncthreads();
    if (wid == 0) {
        float s = 0.f;
        for (int w = 0; w < nwb; ++w) s += sh[w * 32 + lane];
        atomicAdd(glay + L_V + 2 * lane + 1, s);
    }
    __syncthreads();
    block_add(gc, sh, glay + L_C);
}

// input layer backward: dY0 = dH0 [h0 > 0]; grads of W_in, b_in
__global__ void k_gnn_input_bwd(int n, const float *__restrict__ feats,
                                const bf16 *__restrict__ h0, const float *__restrict__ dH,
                                float *grad) {
    __shared__ float sh[8 * 32];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    float gw[4] = {0.f, 0.f, 0.f, 0.f}, gb = 0.f;
    for (int i = warp; i < n; i += nw) {
        const size_t q = (size_t)i * 32 + lane;
        const float d = __bfloat162float(h0[q]) > 0.f ? dH[q] : 0.f;
        gb += d;
#pragma unroll
        for (int k = 0; k < 4; ++k) gw[k] += d * feats[4 * i + k];
    }
    block_add(gb, sh, grad + OFF_BIN);
    // W_in is [lane][4]
    for (int k = 0; k < 4; ++k) {
        const int wid = threadIdx.x >> 5, nwb = blockDim.x >> 5;
        sh[wid * 32 + lane] = gw[k];
        __syncthreads();
        if (wid == 0) {
            float s = 0.f;
            for (int w = 0; w < nwb; ++w) s += sh[w * 32 + lane];
            atomicAdd(grad + OFF_WIN + lane * 4 + k, s);
        }
        __syncthreads();
    }
}

// weights -> BF16 copies (U, U^T, W, W^T per layer)
__global__ void k_gnn_cast(const float *__restrict__ prm, bf16 *U0, bf16 *UT0, bf16 *W0,
                           bf16 *WT0, int l) {
    const float *lay = prm + OFF_L0 + l * LAYER;
    for (int t = threadIdx.x + blockIdx.x * blockDim.x; t < 32 * 64;
         t += blockDim.x * gridDim.x) {
        if (t < 32 * 32) {
            const int r = t / 32, c = t % 32;
            U0[t] = __float2bfloat16_rn(lay[L_U + t]);
            UT0[c * 32 + r] = __float2bfloat16_rn(lay[L_U + t]);
        }
        const int r = t / 64, c = t % 64;
        W0[t] = __float2bfloat16_rn(lay[L_W + t]);
        WT0[c * 32 + r] = __float2bfloat16_rn(lay[L_W + t]);
    }
}

__global__ void k_adam(int np, float *p, const float *g, float *m1, float *m2, float lr,
                       float b1t, float b2t) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
         i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float a = b1 * m1[i] + (1.f - b1) * gi;
        const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
        m1[i] = a;
        m2[i] = b;
        p[i] -= lr * (a / (1.f - b1t)) / (sqrtf(b / (1.f - b2t)) + eps);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int gnn_refresh_bf16(hzb_gnn *G) {
    for (int l = 0; l < 3; ++l) {
        k_gnn_cast<<<8, 256, 0, G->s>>>(G->params, G->Ubf[l], G->UTbf[l], G->Wbf[l],
                                       G->WTbf[l], l);
        count_launch();
    }
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

static void gnn_free_acts(hzb_gnn *G) {
    dfree(G->feats); dfree(G->omega); dfree(G->diag);
    for (auto &p : G->h) dfree(p);
    for (int l = 0; l < 3; ++l) { dfree(G->P[l]); dfree(G->M[l]); dfree(G->y[l]); }
    dfree(G->dH); dfree(G->dY); dfree(G->dP); dfree(G->dM);
    G->n = 0;
}

static int gnn_acts(hzb_gnn *G, int n) {
    if (G->n == n) return SUCCESS;
    gnn_free_acts(G);
    HZB_TRY(dalloc(&G->feats, (size_t)4 * n));
    HZB_TRY(dalloc(&G->omega, n));
    HZB_TRY(dalloc(&G->diag, n));
    for (auto &p : G->h) HZB_TRY(dalloc(&p, (size_t)32 * n));
    for (int l = 0; l < 3; ++l) {
        HZB_TRY(dalloc(&G->P[l], (size_t)32 * n));
        HZB_TRY(dalloc(&G->M[l], (size_t)32 * n));
        HZB_TRY(dalloc(&G->y[l], (size_t)32 * n));
    }
    HZB_TRY(dalloc(&G->dH, (size_t)32 * n));
    HZB_TRY(dalloc(&G->dY, (size_t)32 * n));
    HZB_TRY(dalloc(&G->dP, (size_t)32 * n));
    HZB_TRY(dalloc(&G->dM, (size_t)32 * n));
    G->n = n;
    return SUCCESS;
}

static int warp_grid(int n) { return grid_for((long long)n * 32, 256); }
static int tile_grid(int n) { return div_up(div_up(n, 16), 4); }   // 4 warps / block

int gnn_forward(hzb_gnn *G, const Level &L0, float *omega_out) {
    const int n = L0.n;
    HZB_TRY(gnn_acts(G, n));
    cudaStream_t s = G->s;
    k_gnn_diag<<<grid_for(n), 256, 0, s>>>(n, L0.ia, L0.ja, L0.val, G->diag, G->feats);
    k_gnn_input<<<warp_grid(n), 256, 0, s>>>(n, G->feats, G->params, G->h[0]);
    count_launch(2);
    for (int l = 0; l < 3; ++l) {
        const float *lay = G->params + OFF_L0 + l * LAYER;
        k_gemm_P<<<tile_grid(n), 128, 0, s>>>(n, G->h[l], G->Ubf[l], G->P[l]);
        k_gnn_message<<<warp_grid(n), 256, 0, s>>>(n, L0.ia, L0.ja, L0.val, G->diag, G->P[l],
                                                   lay, G->M[l]);
        k_gemm_Y<<<tile_grid(n), 128, 0, s>>>(n, G->h[l], G->M[l], G->Wbf[l], lay + L_B,
                                              G->y[l], G->h[l + 1]);
        count_launch(3);
    }
    k_gnn_output<<<warp_grid(n), 256, 0, s>>>(n, G->h[3], G->params, G->omega);
    count_launch();
    if (omega_out)
        HZB_CUDA(cudaMemcpyAsync(omega_out, G->omega, sizeof(float) * n,
                                 cudaMemcpyDeviceToDevice, s));
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

int gnn_backward(hzb_gnn *G, const Level &L0, const float *domega) {
    const int n = L0.n;
    if (G->n != n) { set_error_msg("hzb_gnn_backward: run the forward pass first"); return ERROR_INPUT_PAR; }
    cudaStream_t s = G->s;
    const int wg = warp_grid(n), tg = tile_grid(n);
    const int gw = std::max(1, std::min(div_up(n, 64), sm_count() * 4));
    k_gnn_output_bwd<<<wg, 256, 0, s>>>(n, domega, G->omega, G->h[3], G->params, G->dH, G->grads);
    count_launch();
    for (int l = 2; l >= 0; --l) {
        const float *lay = G->params + OFF_L0 + l * LAYER;
        float *glay = G->grads + OFF_L0 + l * LAYER;
        // h_{l+1} = relu(y) + h_l
        k_gnn_relu_bwd<<<wg, 256, 0, s>>>(n, G->dH, G->y[l], G->dY, glay + L_B);
        k_gnn_wgrad<64><<<gw, 256, 0, s>>>(n, G->dY, G->h[l], G->M[l], glay + L_W);
        k_gemm_dX<<<tg, 128, 0, s>>>(n, G->dY, G->WTbf[l], G->dH, G->dM);   // dH: residual + dX
        // messages
        HZB_CUDA(cudaMemsetAsync(G->dP, 0, sizeof(float) * 32 * (size_t)n, s));
        k_gnn_message_bwd<<<wg, 256, 0, s>>>(n, L0.ia, L0.ja, L0.val, G->diag, G->P[l], lay,
                                             G->dM, G->dP, glay);
        // P = h U^T
        k_gnn_wgrad<32><<<gw, 256, 0, s>>>(n, G->dP, G->h[l], nullptr, glay + L_U);
        k_gemm_dH<<<tg, 128, 0, s>>>(n, G->dP, G->UTbf[l], G->dH);
        count_launch(6);
    }
    k_gnn_input_bwd<<<wg, 256, 0, s>>>(n, G->feats, G->h[0], G->dH, G->grads);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

static void init_params(std::vector<float> &p, unsigned long long seed) {
    p.assign(NPARAM, 0.f);
    unsigned long long x = seed * 0x9E3779B97F4A7C15ull + 12345;
    auto uni = [&]() {
        x ^= x >> 12; x ^= x << 25; x ^= x >> 27;
        return (double)((x * 0x2545F4914F6CDD1Dull) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    const double a_in = std::sqrt(6.0 / (4 + 32)), a_u = std::sqrt(6.0 / 64.0);
    const double a_v = std::sqrt(6.0 / 34.0), a_w = 0.5 * std::sqrt(6.0 / 96.0);
    for (int i = 0; i < 128; ++i) p[OFF_WIN + i] = (float)(a_in * uni());
    for (int l = 0; l < 3; ++l) {
        float *lay = p.data() + OFF_L0 + l * LAYER;
        for (int i = 0; i < 1024; ++i) lay[L_U + i] = (float)(a_u * uni());
        for (int i = 0; i < 64; ++i) lay[L_V + i] = (float)(a_v * uni());
        for (int i = 0; i < 2048; ++i) lay[L_W + i] = (float)(a_w * uni());
    }
    // w_o = 0, b_o = 0: omega = 1 until trained
}

}  // namespace hzb

using namespace hzb;

extern "C" INT hzb_gnn_num_params(void) { return NPARAM; }

extern "C" INT hzb_gnn_create(hzb_gnn **out, unsigned long long seed, INT device) {
    *out = nullptr;
    hzb_gnn *G = new (std::nothrow) hzb_gnn();
    if (!G) return ERROR_ALLOC_MEM;
    cudaSetDevice(device);
    if (cudaStreamCreateWithFlags(&G->s, cudaStreamNonBlocking) != cudaSuccess) {
        delete G;
        return ERROR_SOLVER_MISC;
    }
    StreamScope scope_(G->s);
    int rc = SUCCESS;
    std::vector<float> p;
    init_params(p, seed);
    if (!rc) rc = dalloc(&G->params, NPARAM);
    if (!rc) rc = dalloc(&G->grads, NPARAM);
    if (!rc) rc = dalloc(&G->m1, NPARAM);
    if (!rc) rc = dalloc(&G->m2, NPARAM);
    for (int l = 0; l < 3 && !rc; ++l) {
        rc = dalloc(&G->Ubf[l], 1024);
        if (!rc) rc = dalloc(&G->UTbf[l], 1024);
        if (!rc) rc = dalloc(&G->Wbf[l], 2048);
        if (!rc) rc = dalloc(&G->WTbf[l], 2048);
    }
    if (!rc && cudaMemcpyAsync(G->params, p.data(), sizeof(float) * NPARAM,
                               cudaMemcpyHostToDevice, G->s) != cudaSuccess) rc = ERROR_SOLVER_MISC;
    if (!rc) {
        cudaMemsetAsync(G->grads, 0, sizeof(float) * NPARAM, G->s);
        cudaMemsetAsync(G->m1, 0, sizeof(float) * NPARAM, G->s);
        cudaMemsetAsync(G->m2, 0, sizeof(float) * NPARAM, G->s);
        rc = gnn_refresh_bf16(G);
    }
    if (!rc && cudaStreamSynchronize(G->s) != cudaSuccess) rc = ERROR_SOLVER_MISC;
    if (rc) { hzb_gnn_destroy(G); return rc; }
    *out = G;
    return SUCCESS;
}

extern "C" void hzb_gnn_destroy(hzb_gnn *G) {
    if (!G) return;
    {
        StreamScope scope_(G->s);
        cudaStreamSynchronize(G->s);
        gnn_free_acts(G);
        dfree(G->params); dfree(G->grads); dfree(G->m1); dfree(G->m2);
        for (int l = 0; l < 3; ++l) {
            dfree(G->Ubf[l]); dfree(G->UTbf[l]); dfree(G->Wbf[l]); dfree(G->WTbf[l]);
        }
        cudaStreamSynchronize(G->s);
    }
    cudaStreamDestroy(G->s);
    delete G;
}

extern "C" INT hzb_gnn_get_params(const hzb_gnn *G, float *host) {
    HZB_CUDA(cudaMemcpy(host, G->params, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    return SUCCESS;
}
extern "C" INT hzb_gnn_get_grads(const hzb_gnn *G, float *host) {
    HZB_CUDA(cudaStreamSynchronize(G->s));
    HZB_CUDA(cudaMemcpy(host, G->grads, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    return SUCCESS;
}
extern "C" INT hzb_gnn_set_params(hzb_gnn *G, const float *host) {
    StreamScope scope_(G->s);
    HZB_CUDA(cudaMemcpyAsync(G->params, host, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, G->s));
    HZB_TRY(gnn_refresh_bf16(G));
    HZB_CUDA(cudaStreamSynchronize(G->s));
    return SUCCESS;
}
extern "C" INT hzb_gnn_zero_grad(hzb_gnn *G) {
    HZB_CUDA(cudaMemsetAsync(G->grads, 0, sizeof(float) * NPARAM, G->s));
    return SUCCESS;
}
extern "C" INT hzb_gnn_adam_step(hzb_gnn *G, REAL lr) {
    StreamScope scope_(G->s);
    G->step += 1;
    const float b1t = powf(0.9f, (float)G->step), b2t = powf(0.999f, (float)G->step);
    k_adam<<<div_up(NPARAM, 256), 256, 0, G->s>>>(NPARAM, G->params, G->grads, G->m1, G->m2,
                                                  (float)lr, b1t, b2t);
    count_launch();
    HZB_TRY(gnn_refresh_bf16(G));
    HZB_CUDA(cudaStreamSynchronize(G->s));
    return SUCCESS;
}

// omega (device, n) = network(level-0 matrix of s); also left in the network
extern "C" INT hzb_gnn_infer(hzb_gnn *G, hzb_solver *S, float *d_omega) {
    if (!G || !S || S->nl < 1) return ERROR_INPUT_PAR;
    // the solver's stream waits for nothing of ours: run on the network's
    // stream, then make the solver's stream wait on it
    StreamScope scope_(G->s);
    HZB_CUDA(cudaStreamSynchronize(S->s));
    HZB_TRY(gnn_forward(G, S->lv[0], d_omega));
    HZB_CUDA(cudaStreamSynchronize(G->s));
    return SUCCESS;
}

extern "C" INT hzb_gnn_backward(hzb_gnn *G, hzb_solver *S, const float *d_domega) {
    if (!G || !S || S->nl < 1) return ERROR_INPUT_PAR;
    StreamScope scope_(G->s);
    HZB_TRY(gnn_backward(G, S->lv[0], d_domega));
    HZB_CUDA(cudaStreamSynchronize(G->s));
    return SUCCESS;
}

extern "C" INT hzb_learn_errors(hzb_solver *S, INT ns, unsigned long long seed, REAL *d_E,
                                const float *d_omega, INT ncycles) {
    if (!S) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    return learn_errors(S, ns, seed, d_E, d_omega, ncycles);
}

extern "C" INT hzb_learn_loss_grad(hzb_solver *S, const float *d_omega, INT ns,
                                   const REAL *d_E, INT ncycles, REAL *loss,
                                   float *d_domega) {
    if (!S) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    return learn_loss_grad(S, d_omega, ns, d_E, ncycles, loss, d_domega);
}

// Infer omega for the solver's fine level, measure the two-cycle contraction
// of the solve's own cycle with and without it on ns method-generated error
// vectors, and keep the learned weights only if they contract better (plain
// l1-Jacobi otherwise).  Contractions are reported per cycle:
// (||E^2 e||_A / ||e||_A)^(1/2).
extern "C" INT hzb_learn_select_omega(hzb_solver *S, hzb_gnn *G, INT ns,
                                      unsigned long long seed, REAL *rho_plain,
                                      REAL *rho_learned) {
    if (!S || !G || S->nl < 2 || ns < 1) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const int n = S->lv[0].n;
    if (!S->omega) HZB_TRY(dalloc(&S->omega, n));
    HZB_CUDA(cudaStreamSynchronize(S->s));
    {
        StreamScope gs(G->s);
        HZB_TRY(gnn_forward(G, S->lv[0], S->omega));
        HZB_CUDA(cudaStreamSynchronize(G->s));
    }
    // each cycle -- the one the solve runs -- is measured on the errors it
    // leaves itself (its slowest modes), from the same seeded vectors
    double lp = 0.0, ll = 0.0;
    S->omega_active = false;
    HZB_TRY(cycle_contraction(S, ns, seed, &lp));
    S->omega_active = true;
    HZB_TRY(cycle_contraction(S, ns, seed, &ll));
    const double rp = std::pow(std::max(lp, 0.0), 0.25), rl = std::pow(std::max(ll, 0.0), 0.25);
    S->omega_active = rl < rp;
    S->st.omega_contraction[0] = rp;
    S->st.omega_contraction[1] = rl;
    S->st.omega_used = S->omega_active ? 1 : 0;
    if (rho_plain) *rho_plain = rp;
    if (rho_learned) *rho_learned = rl;
    return SUCCESS;
}
