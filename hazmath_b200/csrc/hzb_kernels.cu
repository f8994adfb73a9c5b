// hzb_kernels.cu -- sparse, vector and smoother kernels (FP64 parity + FP32).
//
// Compiled with -fmad=false: a*b+c is rounded twice, as in the reference's
// C loops built without FMA.  Row sums run sequentially in CSR order inside
// one thread; coalescing comes from staging each row bundle's entries in
// shared memory (the CSR-stream schedule), not from splitting rows.
#include "hzb_kernels.cuh"
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <utility>

namespace hzb {

// ---------------------------------------------------------------------------
// bookkeeping
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
static thread_local long long g_launches = 0;

void set_error(cudaError_t e, const char *file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s (%s:%d)", cudaGetErrorString(e), file, line);
    g_err = buf;
}
void set_error_msg(const std::string &m) { g_err = m; }
const char *last_error() { return g_err.c_str(); }
void count_launch(int k) { g_launches += k; }
long long launch_count() { return g_launches; }

cudaStream_t &cur_stream() {
    static thread_local cudaStream_t s = 0;
    return s;
}

void ensure_pool() {
    static std::mutex mu;
    static bool done[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;   // process-local pool attribute
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done[dev] = true;
}

int sm_count() {
    static int cached = 0;
    if (!cached) {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cached = v > 0 ? v : 148;
    }
    return cached;
}

// ---------------------------------------------------------------------------
// SpMV: row bundles staged in shared memory
//
// A CTA owns ROWS consecutive rows (ROWS = 64, 128 or 256, picked per level
// by autotune_bundle).  Their entries form one contiguous range of val/ja;
// it is copied to shared memory with 16-byte streaming loads (ld.global.cs:
// the matrix is read once per pass and should not evict x from L2), then
// every thread sums its own row sequentially in CSR order, gathering x
// through the read-only path.
// ---------------------------------------------------------------------------
__global__ void k_bundle_cap(int n, int rows, const int *__restrict__ ia, int *cap) {
    __shared__ int sh[32];
    int best = 0;
    const int nb = (n + rows - 1) / rows;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb;
         b += gridDim.x * blockDim.x) {
        int r0 = b * rows, r1 = min(r0 + rows, n);
        best = max(best, ia[r1] - ia[r0]);
    }
    best = block_max(best, sh);
    if (threadIdx.x == 0) atomicMax(cap, best);
}

int bundle_capacity_rows(int n, int rows, const int *ia, cudaStream_t s, int *cap) {
    int *d = nullptr;
    HZB_TRY(dalloc(&d, 1));
    cudaMemsetAsync(d, 0, sizeof(int), s);
    const int nb = div_up(n, rows);
    k_bundle_cap<<<grid_for(nb), 256, 0, s>>>(n, rows, ia, d);
    count_launch();
    cudaError_t e = cudaMemcpyAsync(cap, d, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dfree(d);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
    return SUCCESS;
}

int bundle_capacity(int n, const int *ia, cudaStream_t s, int *cap) {
    return bundle_capacity_rows(n, SPMV_ROWS, ia, s, cap);
}

// shared-memory words needed for a bundle of cap entries (4 elements of
// alignment slack in front, one vector of slack at the end)
template <typename T>
__host__ __device__ inline size_t bundle_sc_offset(int cap) {
    return (((size_t)cap + 8) * sizeof(T) + 15) & ~(size_t)15;   // 16-byte aligned
}
template <typename T>
__host__ __device__ inline size_t bundle_smem(int cap) {
    return bundle_sc_offset<T>(cap) + ((size_t)cap + 8) * sizeof(int);
}
// the staged kernels load val/ja with 16-byte vectors: both bases must be
// 16-byte aligned (device allocations are; arbitrary caller views may not be)
template <typename T>
inline bool bundle_aligned(const DCsr<T> &A) {
    return ((reinterpret_cast<uintptr_t>(A.val) | reinterpret_cast<uintptr_t>(A.ja)) & 15) == 0;
}

// One bundle's shared-memory stage: values, column indices and row pointers.
template <typename T>
__host__ __device__ inline size_t bundle_stage_bytes(int cap, int rows) {
    return (bundle_smem<T>(cap) + ((size_t)rows + 4) * sizeof(int) + 15) & ~(size_t)15;
}

__device__ __forceinline__ void cp_async16(unsigned dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
template <int BYTES>
__device__ __forceinline__ void cp_async_small(unsigned dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(src), "n"(BYTES)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issue (without waiting) the copies of a bundle of rows [r0, r1) with
// entries [s, e) into a stage: values/columns at offsets k - s0, s0 = s
// rounded down to 4 entries (16 bytes for both), and ia[r0..r1].  The
// 16-byte body goes as 16-byte copies, the ragged end element by element, so
// nothing outside the arrays is read (their bases are 16-byte aligned).
template <typename T, int NT>
__device__ __forceinline__ int issue_bundle(const int *__restrict__ ia, const T *__restrict__ val,
                                            const int *__restrict__ ja, int r0, int r1, int s,
                                            int e, T *sv, int *sc, int *sia) {
    const int s0 = s & ~3;
    const int ev = e & ~3;
    const int nvec = ev > s0 ? (ev - s0) >> 2 : 0;
    const unsigned dv = (unsigned)__cvta_generic_to_shared(sv);
    const unsigned dc = (unsigned)__cvta_generic_to_shared(sc);
    const unsigned di = (unsigned)__cvta_generic_to_shared(sia);
    const int nv = sizeof(T) == 8 ? 2 * nvec : nvec;
    const char *gv = reinterpret_cast<const char *>(val + s0);
    const char *gc = reinterpret_cast<const char *>(ja + s0);
    for (int q = threadIdx.x; q < nv; q += NT) cp_async16(dv + 16u * q, gv + 16 * (size_t)q);
    for (int q = threadIdx.x; q < nvec; q += NT) cp_async16(dc + 16u * q, gc + 16 * (size_t)q);
    for (int k = max(ev, s0) + threadIdx.x; k < e; k += NT) {
        cp_async_small<sizeof(T)>(dv + (unsigned)((k - s0) * sizeof(T)), val + k);
        cp_async_small<4>(dc + 4u * (k - s0), ja + k);
    }
    for (int q = threadIdx.x; q <= r1 - r0; q += NT) cp_async_small<4>(di + 4u * q, ia + r0 + q);
    return s0;
}

// Persistent bundle loop: CTA c works on bundles c, c + grid, ...; while it
// computes one bundle the copies of its next are in flight (two stages).
// body(bundle, r0, r1, s0, sv, sc, sia) runs between two __syncthreads.
template <typename T, int ROWS, bool ACT, typename F>
__device__ __forceinline__ void bundle_pipeline(int n, const int *__restrict__ ia,
                                                const T *__restrict__ val,
                                                const int *__restrict__ ja, int cap,
                                                const unsigned char *__restrict__ act,
                                                unsigned char *smem, F body) {
    static_assert(ACT_ROWS % ROWS == 0, "bundles tile the activity blocks");
    const int nb = (n + ROWS - 1) / ROWS;
    // ACT: the next bundle of this CTA at or after b that is active
    auto next_active = [&](int b) {
        if constexpr (ACT)
            while (b < nb && !act[(b * ROWS) / ACT_ROWS]) b += gridDim.x;
        return b;
    };
    const size_t stage = bundle_stage_bytes<T>(cap, ROWS);
    const size_t off_c = bundle_sc_offset<T>(cap), off_i = bundle_smem<T>(cap);
    auto SV = [&](int k) { return reinterpret_cast<T *>(smem + k * stage); };
    auto SC = [&](int k) { return reinterpret_cast<int *>(smem + k * stage + off_c); };
    auto SI = [&](int k) { return reinterpret_cast<int *>(smem + k * stage + off_i); };
    int bid = next_active(blockIdx.x);
    if (bid >= nb) return;
    int r0 = bid * ROWS, r1 = min(r0 + ROWS, n);
    int s0 = issue_bundle<T, ROWS>(ia, val, ja, r0, r1, __ldg(ia + r0), __ldg(ia + r1), SV(0),
                                   SC(0), SI(0));
    cp_async_commit();
    // entry range of the next bundle, loaded one bundle ahead
    int nxt = next_active(bid + gridDim.x);
    int ns = 0, ne = 0;
    if (nxt < nb) {
        ns = __ldg(ia + nxt * ROWS);
        ne = __ldg(ia + min(nxt * ROWS + ROWS, n));
    }
    for (int it = 0; bid < nb; ++it) {
        const int st = it & 1;
        int s0n = 0, r0n = 0, r1n = 0;
        if (nxt < nb) {
            r0n = nxt * ROWS;
            r1n = min(r0n + ROWS, n);
            s0n = issue_bundle<T, ROWS>(ia, val, ja, r0n, r1n, ns, ne, SV(st ^ 1), SC(st ^ 1),
                                        SI(st ^ 1));
        }
        cp_async_commit();
        const int after = ACT ? (nxt < nb ? next_active(nxt + gridDim.x) : nb)
                              : nxt + gridDim.x;
        if (after < nb) {
            ns = __ldg(ia + after * ROWS);
            ne = __ldg(ia + min(after * ROWS + ROWS, n));
        }
        cp_async_wait<1>();   // this bundle's copies have landed
        __syncthreads();
        body(bid, r0, r1, s0, SV(st), SC(st), SI(st));
        __syncthreads();      // the stage is free for the bundle after next
        bid = nxt;
        nxt = after;
        r0 = r0n;
        r1 = r1n;
        s0 = s0n;
    }
    cp_async_wait<0>();
}

template <typename T, int MODE>
__device__ __forceinline__ void spmv_store(int row, T t, const T *b, T *y, T alpha) {
    if (MODE == SPMV_Y || MODE == SPMV_Y_DOT) {
        y[row] = t;
    } else if (MODE == SPMV_RES) {
        y[row] = b[row] - t;
    } else {
        if (alpha == T(1)) y[row] += t;
        else if (alpha == T(-1)) y[row] -= t;
        else y[row] += t * alpha;
    }
}

// Sum over one staged row in CSR order.  The x gathers of a group of entries
// are issued before any of them is used: they are independent, and on the
// coarse levels, whose columns scatter, their latency is what bounds the
// sweep.  The sum itself keeps the reference's order, so the result is the
// same as the plain loop's bit for bit.  L1: t -= v x and d += |v| (the
// l1-Jacobi sweep); otherwise t += v x.
// eight gathers in flight per thread (sixteen were measured slower on the
// fine level of the 256^3 case: 0.62 against 0.75 of HBM for its l1 sweep)
template <typename T, bool L1>
__device__ __forceinline__ void staged_row_sum(const T *__restrict__ sv,
                                               const int *__restrict__ sc, int b0, int b1,
                                               const T *__restrict__ x, T &t, T &d) {
    constexpr int GATHER = 8;
    for (int k0 = b0; k0 < b1; k0 += GATHER) {
        T xv[GATHER];
#pragma unroll
        for (int u = 0; u < GATHER; ++u)
            xv[u] = k0 + u < b1 ? __ldg(x + sc[k0 + u]) : T(0);
#pragma unroll
        for (int u = 0; u < GATHER; ++u) {
            if (k0 + u < b1) {
                const T v = sv[k0 + u];
                if (L1) {
                    t -= v * xv[u];
                    d += fabs(v);
                } else {
                    t += v * xv[u];
                }
            }
        }
    }
}

template <typename T, int MODE, int ROWS, bool ACT>
__global__ void __launch_bounds__(ROWS)
k_spmv_bundle(int n, const int *__restrict__ ia, const int *__restrict__ ja,
              const T *__restrict__ val, const T *__restrict__ x,
              const T *__restrict__ b, T *__restrict__ y, T alpha,
              T *__restrict__ part, int cap, const unsigned char *__restrict__ act) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T sh[32];
    bundle_pipeline<T, ROWS, ACT>(n, ia, val, ja, cap, act, smem_raw,
                             [&](int bundle, int r0, int r1, int s0, const T *sv, const int *sc,
                                 const int *sia) {
        const int row = r0 + threadIdx.x;
        T t = T(0), prod = T(0);
        if (row < r1) {
            const int b0 = sia[threadIdx.x] - s0, b1 = sia[threadIdx.x + 1] - s0;
            T unused = T(0);
            staged_row_sum<T, false>(sv, sc, b0, b1, x, t, unused);
            spmv_store<T, MODE>(row, t, b, y, alpha);
            if (MODE == SPMV_Y_DOT) prod = t * __ldg(x + row);
        }
        if (MODE == SPMV_Y_DOT) {
            prod = block_sum(prod, sh);
            if (threadIdx.x == 0) part[bundle] = prod;
        }
    });
}

// Rows too long for the staged bundle: one thread per row from global memory.
template <typename T, int MODE, int ROWS>
__global__ void __launch_bounds__(ROWS)
k_spmv_rows(int n, const int *__restrict__ ia, const int *__restrict__ ja,
            const T *__restrict__ val, const T *__restrict__ x,
            const T *__restrict__ b, T *__restrict__ y, T alpha,
            T *__restrict__ part, const unsigned char *__restrict__ act) {
    const int row = blockIdx.x * ROWS + threadIdx.x;
    T t = T(0), prod = T(0);
    if (row < n && (!act || act[row / ACT_ROWS])) {
        const int b0 = ia[row], b1 = ia[row + 1];
        for (int k = b0; k < b1; ++k) t += val[k] * __ldg(x + ja[k]);
        spmv_store<T, MODE>(row, t, b, y, alpha);
        if (MODE == SPMV_Y_DOT) prod = t * x[row];
    }
    if (MODE == SPMV_Y_DOT) {
        __shared__ T sh[32];
        prod = block_sum(prod, sh);
        if (threadIdx.x == 0) part[blockIdx.x] = prod;
    }
}

int spmv_blocks(int n) { return div_up(n > 0 ? n : 1, SPMV_ROWS); }
int spmv_blocks_rows(int n, int rows) { return div_up(n > 0 ? n : 1, rows > 0 ? rows : SPMV_ROWS); }

// Grid of a persistent bundle kernel: as many CTAs as fit on all SMs at
// once (at most one per bundle).
template <typename K>
static int persistent_grid(K kernel, int threads, size_t smem, int nbundles) {
    static thread_local std::map<std::pair<const void *, size_t>, int> cache;
    const auto key = std::make_pair(reinterpret_cast<const void *>(kernel), smem);
    auto it = cache.find(key);
    int per_sm = 0;
    if (it != cache.end()) {
        per_sm = it->second;
    } else {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
            cudaSuccess || per_sm < 1)
            per_sm = 1;
        cache[key] = per_sm;
    }
    return std::max(1, std::min(nbundles, per_sm * sm_count()));
}

template <typename T>
static bool staged_ok(const DCsr<T> &A, int rows, size_t *smem) {
    *smem = 2 * bundle_stage_bytes<T>(A.bundle_cap, rows);
    return A.bundle_cap > 0 && *smem <= SPMV_SMEM_MAX && bundle_aligned(A);
}

template <typename T, int MODE, int ROWS>
static int spmv_launch(const DCsr<T> &A, const T *x, const T *b, T *y, T alpha, T *part,
                       cudaStream_t s) {
    const int nb = div_up(A.n, ROWS);
    size_t smem = 0;
    if (staged_ok(A, ROWS, &smem)) {
        static bool done = false;   // per instantiation: raise the limit once
        if (!done) {
            cudaFuncSetAttribute(k_spmv_bundle<T, MODE, ROWS, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, SPMV_SMEM_MAX);
            cudaFuncSetAttribute(k_spmv_bundle<T, MODE, ROWS, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, SPMV_SMEM_MAX);
            done = true;
        }
        // the activity check is a separate instantiation: ordinary solves
        // run the kernel without it
        if (A.act) {
            const int grid = persistent_grid(k_spmv_bundle<T, MODE, ROWS, true>, ROWS, smem, nb);
            k_spmv_bundle<T, MODE, ROWS, true><<<grid, ROWS, smem, s>>>(
                A.n, A.ia, A.ja, A.val, x, b, y, alpha, part, A.bundle_cap, A.act);
        } else {
            const int grid = persistent_grid(k_spmv_bundle<T, MODE, ROWS, false>, ROWS, smem, nb);
            k_spmv_bundle<T, MODE, ROWS, false><<<grid, ROWS, smem, s>>>(
                A.n, A.ia, A.ja, A.val, x, b, y, alpha, part, A.bundle_cap, nullptr);
        }
    } else {
        const int grid = nb;
        k_spmv_rows<T, MODE, ROWS><<<grid, ROWS, 0, s>>>(A.n, A.ia, A.ja, A.val, x, b, y,
                                                         alpha, part, A.act);
    }
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// FP32 vector CSR: LPR lanes per row read the row's entries with coalesced
// loads (no staging), partial sums combined by shuffles.  For the FP32 cycle,
// whose arithmetic is judged by convergence, not by the reference's order.
template <int LPR>
__device__ __forceinline__ float lanes_sum(float v) {
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, LPR);
    return v;
}

// Without an activity array (ACT false) a thread group handles one row of a
// flat grid.  With one, a CTA takes 256-row blocks in turn, skips inactive
// blocks, and its 256 / LPR groups cover a block in LPR passes.
template <int MODE, int LPR, bool ACT>
__global__ void __launch_bounds__(256)
k_spmv_vec(int n, const int *__restrict__ ia, const int *__restrict__ ja,
           const float *__restrict__ val, const float *__restrict__ x,
           const float *__restrict__ b, float *__restrict__ y, float alpha,
           const unsigned char *__restrict__ act) {
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR;
    auto one_row = [&](int g) {
        const int row = g < n ? g : n - 1;   // whole groups stay in the shuffles
        float t = 0.f;
        for (int k = __ldg(ia + row) + lane; k < __ldg(ia + row + 1); k += LPR)
            t += __ldcs(val + k) * __ldg(x + __ldcs(ja + k));
        t = lanes_sum<LPR>(t);
        if (lane == 0 && g < n) spmv_store<float, MODE>(row, t, b, y, alpha);
    };
    if constexpr (!ACT) {
        one_row((blockIdx.x * blockDim.x + threadIdx.x) / LPR);
    } else {
        const int nblk = (n + ACT_ROWS - 1) / ACT_ROWS;
        for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
            if (!act[blk]) continue;
            for (int pass = 0; pass < LPR; ++pass)
                one_row(blk * ACT_ROWS + pass * (256 / LPR) + grp);
        }
    }
}

template <int LPR, bool ACT>
__global__ void __launch_bounds__(256)
k_l1_vec(int n, const int *__restrict__ ia, const int *__restrict__ ja,
         const float *__restrict__ a, const float *__restrict__ b,
         const float *__restrict__ x, float *__restrict__ xn, const float *__restrict__ omega,
         const unsigned char *__restrict__ act) {
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR;
    auto one_row = [&](int g) {
        const int row = g < n ? g : n - 1;
        float t = 0.f, d = 0.f;
        for (int k = __ldg(ia + row) + lane; k < __ldg(ia + row + 1); k += LPR) {
            const float v = __ldcs(a + k);
            t += v * __ldg(x + __ldcs(ja + k));
            d += fabsf(v);
        }
        t = lanes_sum<LPR>(t);
        d = lanes_sum<LPR>(d);
        if (lane == 0 && g < n) {
            float xi = x[row];
            if (fabsf(d) > float(SMALLREAL)) {
                const float r = b[row] - t;
                xi += omega ? omega[row] * (r / d) : r / d;
            }
            xn[row] = xi;
        }
    };
    if constexpr (!ACT) {
        one_row((blockIdx.x * blockDim.x + threadIdx.x) / LPR);
    } else {
        const int nblk = (n + ACT_ROWS - 1) / ACT_ROWS;
        for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
            if (!act[blk]) continue;
            for (int pass = 0; pass < LPR; ++pass)
                one_row(blk * ACT_ROWS + pass * (256 / LPR) + grp);
        }
    }
}

// grid of the lane kernels: one row per group, or (with an activity array)
// the 256-row blocks shared by at most 16 CTAs per SM
static int vec_grid(int n, int lanes, bool act) {
    if (!act) return div_up(n, 256 / lanes);
    return std::max(1, std::min((n + ACT_ROWS - 1) / ACT_ROWS, 16 * sm_count()));
}

template <int MODE>
static int spmv_vec_launch(const DCsr<float> &A, const float *x, const float *b, float *y,
                           float alpha, cudaStream_t s) {
    const int L = A.vec_lanes;
    const bool act = A.act != nullptr;
    const int grid = vec_grid(A.n, L, act);
    auto go = [&](auto kernel) {
        kernel<<<grid, 256, 0, s>>>(A.n, A.ia, A.ja, A.val, x, b, y, alpha, A.act);
    };
    switch (L) {
    case 2: act ? go(k_spmv_vec<MODE, 2, true>) : go(k_spmv_vec<MODE, 2, false>); break;
    case 4: act ? go(k_spmv_vec<MODE, 4, true>) : go(k_spmv_vec<MODE, 4, false>); break;
    case 8: act ? go(k_spmv_vec<MODE, 8, true>) : go(k_spmv_vec<MODE, 8, false>); break;
    default: act ? go(k_spmv_vec<MODE, 16, true>) : go(k_spmv_vec<MODE, 16, false>); break;
    }
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

template <typename T, int MODE>
static int spmv_mode(const DCsr<T> &A, const T *x, const T *b, T *y, T alpha, T *part,
                     cudaStream_t s) {
    if (A.n <= 0) return SUCCESS;
    if constexpr (sizeof(T) == 4 && MODE != SPMV_Y_DOT) {
        if (A.vec_lanes == SELL_LANES && A.sell.npad > 0 && !A.act)
            return sell_spmv(A, MODE, x, b, y, alpha, s);
        if (A.vec_lanes > 0) return spmv_vec_launch<MODE>(A, x, b, y, alpha, s);
    }
    switch (A.bundle_rows) {
    case 64: return spmv_launch<T, MODE, 64>(A, x, b, y, alpha, part, s);
    case 256: return spmv_launch<T, MODE, 256>(A, x, b, y, alpha, part, s);
    default: return spmv_launch<T, MODE, 128>(A, x, b, y, alpha, part, s);
    }
}

template <typename T>
int spmv(const DCsr<T> &A, int mode, const T *x, const T *b, T *y, T alpha,
         T *part, cudaStream_t s) {
    switch (mode) {
    case SPMV_Y: return spmv_mode<T, SPMV_Y>(A, x, b, y, alpha, part, s);
    case SPMV_RES: return spmv_mode<T, SPMV_RES>(A, x, b, y, alpha, part, s);
    case SPMV_AXPY: return spmv_mode<T, SPMV_AXPY>(A, x, b, y, alpha, part, s);
    case SPMV_Y_DOT: return spmv_mode<T, SPMV_Y_DOT>(A, x, b, y, alpha, part, s);
    }
    return ERROR_INPUT_PAR;
}
template int spmv<double>(const DCsr<double> &, int, const double *, const double *,
                          double *, double, double *, cudaStream_t);
template int spmv<float>(const DCsr<float> &, int, const float *, const float *,
                         float *, float, float *, cudaStream_t);

// Decisions of the autotuners, kept per level shape (rows, stored entries)
// for the life of the process: a later setup of a level of the same shape
// reuses them instead of timing the candidates again.
namespace {
std::mutex tune_mu;
std::map<std::pair<int, int>, int> tune_bundle_rows, tune_fp32_lanes;
bool tune_lookup(std::map<std::pair<int, int>, int> &m, int n, int nnz, int *v) {
    std::lock_guard<std::mutex> g(tune_mu);
    auto it = m.find({n, nnz});
    if (it == m.end()) return false;
    *v = it->second;
    return true;
}
void tune_store(std::map<std::pair<int, int>, int> &m, int n, int nnz, int v) {
    std::lock_guard<std::mutex> g(tune_mu);
    m[{n, nnz}] = v;
}
}  // namespace

// Autotuner of the bundle size: times each candidate on this level's SpMV
// (y = A x with the level's own buffers) and keeps the fastest.
int autotune_bundle(DCsr<double> &A, const double *x, double *y, cudaStream_t s) {
    int known = 0;
    if (tune_lookup(tune_bundle_rows, A.n, A.nnz, &known)) {
        A.bundle_rows = known;
        return bundle_capacity_rows(A.n, known, A.ia, s, &A.bundle_cap);
    }
    const int cands[3] = {64, 128, 256};
    cudaEvent_t e0, e1;
    HZB_CUDA(cudaEventCreate(&e0));
    HZB_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_rows = SPMV_ROWS, best_cap = A.bundle_cap;
    for (int c : cands) {
        DCsr<double> B = A;
        B.bundle_rows = c;
        HZB_TRY(bundle_capacity_rows(A.n, c, A.ia, s, &B.bundle_cap));
        if (2 * bundle_stage_bytes<double>(B.bundle_cap, c) > SPMV_SMEM_MAX) continue;
        HZB_TRY(spmv<double>(B, SPMV_Y, x, nullptr, y, 1.0, nullptr, s));   // warm
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; ++r) HZB_TRY(spmv<double>(B, SPMV_Y, x, nullptr, y, 1.0, nullptr, s));
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; best_rows = c; best_cap = B.bundle_cap; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    A.bundle_rows = best_rows;
    A.bundle_cap = best_cap;
    tune_store(tune_bundle_rows, A.n, A.nnz, best_rows);
    return SUCCESS;
}

bool fp32_schedule_known(int n, int nnz, int *lanes) {
    return tune_lookup(tune_fp32_lanes, n, nnz, lanes);
}

// FP32 schedule of a level: the staged bundles (vec_lanes 0), 4/8/16 lanes
// per row or the sliced-ELL copy (when A.sell holds one), whichever runs
// this level's l1-Jacobi sweep fastest.
int autotune_fp32(DCsr<float> &A, const float *b, const float *x, float *xn, cudaStream_t s) {
    int known = 0;
    if (tune_lookup(tune_fp32_lanes, A.n, A.nnz, &known)) {
        A.vec_lanes = known;
        return SUCCESS;
    }
    const int cands[5] = {0, 4, 8, 16, SELL_LANES};
    cudaEvent_t e0, e1;
    HZB_CUDA(cudaEventCreate(&e0));
    HZB_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int pick = 0;
    for (int c : cands) {
        if (c == SELL_LANES && A.sell.npad == 0) continue;
        DCsr<float> B = A;
        B.vec_lanes = c;
        HZB_TRY(l1_sweep<float>(B, b, x, xn, nullptr, s));   // warm
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; ++r) HZB_TRY(l1_sweep<float>(B, b, x, xn, nullptr, s));
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; pick = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    A.vec_lanes = pick;
    tune_store(tune_fp32_lanes, A.n, A.nnz, pick);
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// Transfers (P = aggregate map, R = P^T with ascending fine rows)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_restrict(int nc, const int *__restrict__ ria,
                           const int *__restrict__ rja, const T *__restrict__ w,
                           T *__restrict__ bc, const unsigned char *__restrict__ act) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc;
         c += gridDim.x * blockDim.x) {
        if (act && !act[c / ACT_ROWS]) continue;
        T t = T(0);
        for (int k = ria[c]; k < ria[c + 1]; ++k) t += w[rja[k]];
        bc[c] = t;
    }
}

template <typename T>
int restrict_agg(int nc, const int *ria, const int *rja, const T *w, T *bc,
                 cudaStream_t s, const unsigned char *act_c) {
    if (nc <= 0) return SUCCESS;
    k_restrict<T><<<grid_for(nc), 256, 0, s>>>(nc, ria, rja, w, bc, act_c);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
template int restrict_agg<double>(int, const int *, const int *, const double *,
                                  double *, cudaStream_t, const unsigned char *);
template int restrict_agg<float>(int, const int *, const int *, const float *,
                                 float *, cudaStream_t, const unsigned char *);

template <typename T>
__global__ void k_prolong(int n, const int *__restrict__ agg,
                          const T *__restrict__ xc, T *__restrict__ x, T alpha,
                          const unsigned char *__restrict__ act) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        if (act && !act[i / ACT_ROWS]) continue;
        T t = T(0);
        const int c = agg[i];
        if (c >= 0) t += xc[c];
        if (alpha == T(1)) x[i] += t;
        else if (alpha == T(-1)) x[i] -= t;
        else x[i] += t * alpha;
    }
}

template <typename T>
int prolong_agg(int n, const int *agg, const T *xc, T *x, T alpha,
                cudaStream_t s, const unsigned char *act) {
    if (n <= 0) return SUCCESS;
    k_prolong<T><<<grid_for(n), 256, 0, s>>>(n, agg, xc, x, alpha, act);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
template int prolong_agg<double>(int, const int *, const double *, double *,
                                 double, cudaStream_t, const unsigned char *);
template int prolong_agg<float>(int, const int *, const float *, float *, float,
                                cudaStream_t, const unsigned char *);

// ---------------------------------------------------------------------------
// Point smoothers
// ---------------------------------------------------------------------------
// Jacobi, w = 1: t = b_i - sum_{j != i} a_ij x_j;  x_i = (1-w) x_i + w t / d_i
__global__ void k_jacobi(int n, const int *__restrict__ ia,
                         const int *__restrict__ ja, const double *__restrict__ a,
                         const double *__restrict__ dj, const double *__restrict__ b,
                         const double *__restrict__ x, double *__restrict__ xn) {
    const double w = 1.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        double t = b[i];
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (ja[k] != i) t -= a[k] * x[ja[k]];
        const double d = dj[i];
        xn[i] = (fabs(d) > SMALLREAL) ? (1 - w) * x[i] + w * t / d : x[i];
    }
}

int jacobi_sweep(const DCsr<double> &A, const double *dj, const double *b,
                 const double *x, double *xn, cudaStream_t s) {
    if (A.n <= 0) return SUCCESS;
    k_jacobi<<<grid_for(A.n), 256, 0, s>>>(A.n, A.ia, A.ja, A.val, dj, b, x, xn);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

// l1-Jacobi: t = b_i - sum_j a_ij x_j, d = sum_j |a_ij| (both in CSR order);
// x_i += omega_i * (t / d).  Rows are staged per bundle like the SpMV.
template <typename T>
__device__ __forceinline__ T l1_update(int i, T t, T d, const T *__restrict__ x,
                                      const float *__restrict__ omega) {
    T xi = x[i];
    if (fabs(d) > T(SMALLREAL)) {
        if (omega) xi += T(omega[i]) * (t / d);
        else xi += t / d;
    }
    return xi;
}

template <typename T, int ROWS, bool ACT>
__global__ void __launch_bounds__(ROWS)
k_l1_bundle(int n, const int *__restrict__ ia, const int *__restrict__ ja,
            const T *__restrict__ a, const T *__restrict__ b,
            const T *__restrict__ x, T *__restrict__ xn,
            const float *__restrict__ omega, int cap, const unsigned char *__restrict__ act) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bundle_pipeline<T, ROWS, ACT>(n, ia, a, ja, cap, act, smem_raw,
                             [&](int, int r0, int r1, int s0, const T *sv, const int *sc,
                                 const int *sia) {
        const int i = r0 + threadIdx.x;
        if (i >= r1) return;
        T t = b[i], d = T(0);
        const int b0 = sia[threadIdx.x] - s0, b1 = sia[threadIdx.x + 1] - s0;
        staged_row_sum<T, true>(sv, sc, b0, b1, x, t, d);
        xn[i] = l1_update(i, t, d, x, omega);
    });
}

// Rows too long for a staged bundle: one thread per row from global memory.
template <typename T, int ROWS>
__global__ void __launch_bounds__(ROWS)
k_l1_rows(int n, const int *__restrict__ ia, const int *__restrict__ ja,
          const T *__restrict__ a, const T *__restrict__ b, const T *__restrict__ x,
          T *__restrict__ xn, const float *__restrict__ omega,
          const unsigned char *__restrict__ act) {
    const int i = blockIdx.x * ROWS + threadIdx.x;
    if (i >= n || (act && !act[i / ACT_ROWS])) return;
    T t = b[i], d = T(0);
    for (int k = ia[i]; k < ia[i + 1]; ++k) {
        const T v = a[k];
        t -= v * __ldg(x + ja[k]);
        d += fabs(v);
    }
    xn[i] = l1_update(i, t, d, x, omega);
}

template <typename T, int ROWS>
static int l1_launch(const DCsr<T> &A, const T *b, const T *x, T *xn, const float *omega,
                     cudaStream_t s) {
    const int nb = div_up(A.n, ROWS);
    size_t smem = 0;
    if (staged_ok(A, ROWS, &smem)) {
        static bool done = false;
        if (!done) {
            cudaFuncSetAttribute(k_l1_bundle<T, ROWS, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, SPMV_SMEM_MAX);
            cudaFuncSetAttribute(k_l1_bundle<T, ROWS, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, SPMV_SMEM_MAX);
            done = true;
        }
        if (A.act) {
            const int grid = persistent_grid(k_l1_bundle<T, ROWS, true>, ROWS, smem, nb);
            k_l1_bundle<T, ROWS, true><<<grid, ROWS, smem, s>>>(A.n, A.ia, A.ja, A.val, b, x,
                                                                xn, omega, A.bundle_cap, A.act);
        } else {
            const int grid = persistent_grid(k_l1_bundle<T, ROWS, false>, ROWS, smem, nb);
            k_l1_bundle<T, ROWS, false><<<grid, ROWS, smem, s>>>(A.n, A.ia, A.ja, A.val, b, x,
                                                                 xn, omega, A.bundle_cap,
                                                                 nullptr);
        }
    } else {
        k_l1_rows<T, ROWS><<<nb, ROWS, 0, s>>>(A.n, A.ia, A.ja, A.val, b, x, xn, omega, A.act);
    }
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

static int l1_vec_launch(const DCsr<float> &A, const float *b, const float *x, float *xn,
                         const float *omega, cudaStream_t s) {
    const int L = A.vec_lanes;
    const bool act = A.act != nullptr;
    const int grid = vec_grid(A.n, L, act);
    auto go = [&](auto kernel) {
        kernel<<<grid, 256, 0, s>>>(A.n, A.ia, A.ja, A.val, b, x, xn, omega, A.act);
    };
    switch (L) {
    case 2: act ? go(k_l1_vec<2, true>) : go(k_l1_vec<2, false>); break;
    case 4: act ? go(k_l1_vec<4, true>) : go(k_l1_vec<4, false>); break;
    case 8: act ? go(k_l1_vec<8, true>) : go(k_l1_vec<8, false>); break;
    default: act ? go(k_l1_vec<16, true>) : go(k_l1_vec<16, false>); break;
    }
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

template <typename T>
int l1_sweep(const DCsr<T> &A, const T *b, const T *x, T *xn,
             const float *omega, cudaStream_t s) {
    if (A.n <= 0) return SUCCESS;
    if constexpr (sizeof(T) == 4) {
        if (A.vec_lanes == SELL_LANES && A.sell.npad > 0 && !A.act)
            return sell_l1_sweep(A, b, x, xn, omega, s);
        if (A.vec_lanes > 0) return l1_vec_launch(A, b, x, xn, omega, s);
    }
    switch (A.bundle_rows) {
    case 64: return l1_launch<T, 64>(A, b, x, xn, omega, s);
    case 256: return l1_launch<T, 256>(A, b, x, xn, omega, s);
    default: return l1_launch<T, 128>(A, b, x, xn, omega, s);
    }
}
template int l1_sweep<double>(const DCsr<double> &, const double *, const double *,
                              double *, const float *, cudaStream_t);
template int l1_sweep<float>(const DCsr<float> &, const float *, const float *,
                             float *, const float *, cudaStream_t);

template <typename T>
__global__ void k_l1_norms(int n, const int *__restrict__ ia, const T *__restrict__ a,
                           T *__restrict__ d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        T s = T(0);
        for (int k = ia[i]; k < ia[i + 1]; ++k) s += fabs(a[k]);
        d[i] = s;
    }
}

template <typename T>
__global__ void k_l1_first(int n, const T *__restrict__ b, const T *__restrict__ d,
                           T *__restrict__ xn, const float *__restrict__ omega,
                           const unsigned char *__restrict__ act) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        if (act && !act[i / ACT_ROWS]) continue;
        const T di = d[i];
        T xi = T(0);
        if (fabs(di) > T(SMALLREAL)) xi += (omega ? T(omega[i]) : T(1)) * (b[i] / di);
        xn[i] = xi;
    }
}

template <typename T>
int l1_norms(const DCsr<T> &A, T *d, cudaStream_t s) {
    if (A.n <= 0) return SUCCESS;
    k_l1_norms<T><<<grid_for(A.n), 256, 0, s>>>(A.n, A.ia, A.val, d);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
template <typename T>
int l1_first_sweep(int n, const T *b, const T *d, T *xn, const float *omega,
                   cudaStream_t s, const unsigned char *act) {
    if (n <= 0) return SUCCESS;
    k_l1_first<T><<<grid_for(n), 256, 0, s>>>(n, b, d, xn, omega, act);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
template int l1_norms<float>(const DCsr<float> &, float *, cudaStream_t);
template int l1_norms<double>(const DCsr<double> &, double *, cudaStream_t);
template int l1_first_sweep<float>(int, const float *, const float *, float *,
                                   const float *, cudaStream_t, const unsigned char *);
template int l1_first_sweep<double>(int, const double *, const double *, double *,
                                    const float *, cudaStream_t, const unsigned char *);

// Gauss-Seidel family on independent rows.  x is read with plain loads:
// in gs_run earlier sets of the same CTA wrote it.
// Row `skip` is left untouched: the backward sweep of smoother_dcsr_sgs starts
// at row n-2 (smoother.c:225); the host passes kind | GS_SKIP_LAST for it.
template <typename T>
__device__ __forceinline__ void gs_row(int i, int kind, const int *ia,
                                       const int *ja, const T *a, const T *d,
                                       T w, const T *b, T *x, int skip) {
    if (i == skip) return;
    T t = b[i];
    const int k1 = ia[i + 1];
    for (int k = ia[i]; k < k1; ++k) {
        const int j = ja[k];
        if (j != i) t -= a[k] * x[j];
    }
    const T di = d[i];
    if (kind == 0) {
        x[i] = t * di;
    } else if (kind == 1) {
        if (fabs(di) > T(SMALLREAL)) x[i] = w * (t / di) + (1 - w) * x[i];
    } else {
        if (fabs(di) > T(SMALLREAL)) x[i] = t / di;
    }
}

template <typename T>
__global__ void k_gs_rows(int cnt, const int *__restrict__ rows,
                          const int *__restrict__ ia, const int *__restrict__ ja,
                          const T *__restrict__ a, const T *__restrict__ d,
                          int kind, T w, const T *__restrict__ b, T *x,
                          int skip) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt;
         q += gridDim.x * blockDim.x)
        gs_row<T>(rows[q], kind, ia, ja, a, d, w, b, x, skip);
}

// Row data of one thread's row in a level set: its index, bounds, the first
// P column indices and values, b_i and d_i -- all independent of the sweep,
// so a kernel loads them for its next set before the barrier that ends the
// current one.
template <typename T, int P>
struct GsRowData {
    int i = -1, k0 = 0, k1 = 0;
    int col[P];
    T val[P];
    T bi = T(0), di = T(0);
};
template <typename T, int P>
__device__ __forceinline__ void gs_row_load(GsRowData<T, P> &r, const int *__restrict__ rows,
                                            int q, int q1, const int *__restrict__ ia,
                                            const int *__restrict__ ja,
                                            const T *__restrict__ a,
                                            const T *__restrict__ d,
                                            const T *__restrict__ b) {
    r.i = q < q1 ? rows[q] : -1;
    if (r.i < 0) return;
    r.k0 = ia[r.i];
    r.k1 = ia[r.i + 1];
#pragma unroll
    for (int u = 0; u < P; ++u) {
        if (r.k0 + u < r.k1) {
            r.col[u] = ja[r.k0 + u];
            r.val[u] = a[r.k0 + u];
        }
    }
    r.bi = b[r.i];
    r.di = d[r.i];
}
// A run of small level sets (at most NT rows each, so a thread has at most
// one row per set) in one CTA of NT threads, the sets separated by
// __syncthreads.  Everything a row needs except x is independent of the
// sweep and is loaded ahead in a three-deep pipeline: while set s is swept,
// a thread loads its row index in set s+3, the bounds, b_i and d_i of its
// row in set s+2 and the first P column indices and values of its row in
// set s+1, each from values that arrived during the previous set, so the
// chain set pointer -> row -> row bounds -> entries costs no barrier period
// of its own.  The four sets in flight live in four register stages whose
// roles rotate through an unrolled loop: a stage is never copied, so no
// instruction waits on a load issued for a later set.  Only the x gathers
// remain between barriers.  The run's set pointers sit in shared memory, and
// so does x when the level fits (XS): the run then reads x once, sweeps in
// shared memory and writes x back.  The row sum runs in CSR order from b_i
// with the diagonal skipped, as gs_row's.
template <typename T, int P>
struct GsStage {
    int i, k0, k1;
    T bi, di;
    int c[P];
    T v[P];
};

template <typename T, int NT, int P, bool XS>
__global__ void __launch_bounds__(NT)
k_gs_pipe(const int *__restrict__ rows, const int *__restrict__ set_ptr, int first, int last,
          int n, const int *__restrict__ ia, const int *__restrict__ ja,
          const T *__restrict__ a, const T *__restrict__ d, int kind, T w,
          const T *__restrict__ b, T *xg, int skip) {
    extern __shared__ __align__(16) unsigned char gs_smem[];
    const int ns = last - first;
    int *sp = reinterpret_cast<int *>(gs_smem);
    T *xs = reinterpret_cast<T *>(gs_smem + gs_sp_bytes(ns));
    for (int k = threadIdx.x; k <= ns; k += NT) sp[k] = set_ptr[first + k];
    if (XS) {
#pragma unroll 4
        for (int k = threadIdx.x; k < n; k += NT) xs[k] = xg[k];
    }
    __syncthreads();
    T *x = XS ? xs : xg;
    const int t = threadIdx.x;
    using St = GsStage<T, P>;
    auto row_of = [&](St &S, int r) {   // this thread's row in set r of the run, or -1
        S.i = -1;
        if (r < ns) {
            const int q = sp[r] + t;
            if (q < sp[r + 1]) S.i = __ldg(rows + q);
        }
    };
    auto bounds = [&](St &S) {
        S.k0 = S.k1 = 0;
        S.bi = S.di = T(0);
        if (S.i >= 0) {
            S.k0 = __ldg(ia + S.i);
            S.k1 = __ldg(ia + S.i + 1);
            S.bi = __ldg(b + S.i);
            S.di = __ldg(d + S.i);
        }
    };
    auto entries = [&](St &S) {
#pragma unroll
        for (int u = 0; u < P; ++u) {
            S.c[u] = 0;
            S.v[u] = T(0);
            if (S.k0 + u < S.k1) {
                S.c[u] = __ldg(ja + S.k0 + u);
                S.v[u] = __ldg(a + S.k0 + u);
            }
        }
    };
    auto apply = [&](const St &S) {
        const int i = S.i;
        if (i < 0 || i == skip) return;
        T xv[P];
#pragma unroll
        for (int u = 0; u < P; ++u) xv[u] = S.k0 + u < S.k1 ? x[S.c[u]] : T(0);
        T tv = S.bi;
#pragma unroll
        for (int u = 0; u < P; ++u)
            if (S.k0 + u < S.k1 && S.c[u] != i) tv -= S.v[u] * xv[u];
        for (int k = S.k0 + P; k < S.k1; ++k) {
            const int j = __ldg(ja + k);
            if (j != i) tv -= __ldg(a + k) * x[j];
        }
        const T di = S.di;
        if (kind == 0) {
            x[i] = tv * di;
        } else if (kind == 1) {
            if (fabs(di) > T(SMALLREAL)) x[i] = w * (tv / di) + (1 - w) * x[i];
        } else {
            if (fabs(di) > T(SMALLREAL)) x[i] = tv / di;
        }
    };
    // set s+3 (row), s+2 (bounds), s+1 (entries) loaded; set s swept
    auto step = [&](int s, St &A3, St &B2, St &C1, const St &D0) {
        entries(C1);
        bounds(B2);
        row_of(A3, s + 3);
        apply(D0);
        __syncthreads();
    };
    St S0, S1, S2, S3;
    row_of(S0, 0);
    row_of(S1, 1);
    row_of(S2, 2);
    bounds(S0);
    bounds(S1);
    entries(S0);
    for (int s = 0; s < ns; s += 4) {
        step(s, S3, S2, S1, S0);
        if (s + 1 >= ns) break;
        step(s + 1, S0, S3, S2, S1);
        if (s + 2 >= ns) break;
        step(s + 2, S1, S0, S3, S2);
        if (s + 3 >= ns) break;
        step(s + 3, S2, S1, S0, S3);
    }
    if (XS) {
#pragma unroll 4
        for (int k = threadIdx.x; k < n; k += NT) xg[k] = xs[k];
    }
}

// The same sweep for runs of sets of at most 256 rows with the pipeline
// twice as deep: a thread loads its row index in set s+6, the bounds of its
// row in set s+4 and the entries of its row in set s+2, so every load has
// two barrier periods to arrive before anything uses it.  Seven register
// stages rotate through a seven-fold unrolled loop.  x lives in the CTA's
// shared memory when the level fits (XS), else in global memory.  (Holding
// x in the distributed shared memory of a cluster of 2-8 CTAs instead, with
// a cluster barrier between sets, measured slower on the 2D 255^2 levels:
// 854 against 612 us for the 509 sets of level 0.)
template <typename T, int NT, int P, bool XS>
__global__ void __launch_bounds__(NT)
k_gs_deep(const int *__restrict__ rows, const int *__restrict__ set_ptr, int first, int last,
          int n, const int *__restrict__ ia, const int *__restrict__ ja,
          const T *__restrict__ a, const T *__restrict__ d, int kind, T w,
          const T *__restrict__ b, T *xg, int skip) {
    extern __shared__ __align__(16) unsigned char gs_smem[];
    const int ns = last - first;
    int *sp = reinterpret_cast<int *>(gs_smem);
    T *xs = reinterpret_cast<T *>(gs_smem + gs_sp_bytes(ns));
    for (int k = threadIdx.x; k <= ns; k += NT) sp[k] = set_ptr[first + k];
    if (XS) {
#pragma unroll 4
        for (int k = threadIdx.x; k < n; k += NT) xs[k] = xg[k];
    }
    __syncthreads();
    auto xat = [&](int j) -> T * { return XS ? xs + j : xg + j; };
    const int t = threadIdx.x;
    using St = GsStage<T, P>;
    auto row_of = [&](St &S, int r) {
        S.i = -1;
        if (r < ns) {
            const int q = sp[r] + t;
            if (q < sp[r + 1]) S.i = __ldg(rows + q);
        }
    };
    auto bounds = [&](St &S) {
        S.k0 = S.k1 = 0;
        S.bi = S.di = T(0);
        if (S.i >= 0) {
            S.k0 = __ldg(ia + S.i);
            S.k1 = __ldg(ia + S.i + 1);
            S.bi = __ldg(b + S.i);
            S.di = __ldg(d + S.i);
        }
    };
    auto entries = [&](St &S) {
#pragma unroll
        for (int u = 0; u < P; ++u) {
            S.c[u] = 0;
            S.v[u] = T(0);
            if (S.k0 + u < S.k1) {
                S.c[u] = __ldg(ja + S.k0 + u);
                S.v[u] = __ldg(a + S.k0 + u);
            }
        }
    };
    auto apply = [&](const St &S) {
        const int i = S.i;
        if (i < 0 || i == skip) return;
        T xv[P];
#pragma unroll
        for (int u = 0; u < P; ++u) xv[u] = S.k0 + u < S.k1 ? *xat(S.c[u]) : T(0);
        T tv = S.bi;
#pragma unroll
        for (int u = 0; u < P; ++u)
            if (S.k0 + u < S.k1 && S.c[u] != i) tv -= S.v[u] * xv[u];
        for (int k = S.k0 + P; k < S.k1; ++k) {
            const int j = __ldg(ja + k);
            if (j != i) tv -= __ldg(a + k) * *xat(j);
        }
        const T di = S.di;
        T *xi = xat(i);
        if (kind == 0) {
            *xi = tv * di;
        } else if (kind == 1) {
            if (fabs(di) > T(SMALLREAL)) *xi = w * (tv / di) + (1 - w) * *xi;
        } else {
            if (fabs(di) > T(SMALLREAL)) *xi = tv / di;
        }
    };
    auto step = [&](int s, St &R6, St &B4, St &E2, const St &D0) {
        entries(E2);
        bounds(B4);
        row_of(R6, s + 6);
        apply(D0);
        __syncthreads();
    };
    St S0, S1, S2, S3, S4, S5, S6;
    row_of(S0, 0);
    row_of(S1, 1);
    row_of(S2, 2);
    row_of(S3, 3);
    row_of(S4, 4);
    row_of(S5, 5);
    bounds(S0);
    bounds(S1);
    bounds(S2);
    bounds(S3);
    entries(S0);
    entries(S1);
    for (int s = 0; s < ns; s += 7) {
        step(s, S6, S4, S2, S0);
        if (s + 1 >= ns) break;
        step(s + 1, S0, S5, S3, S1);
        if (s + 2 >= ns) break;
        step(s + 2, S1, S6, S4, S2);
        if (s + 3 >= ns) break;
        step(s + 3, S2, S0, S5, S3);
        if (s + 4 >= ns) break;
        step(s + 4, S3, S1, S6, S4);
        if (s + 5 >= ns) break;
        step(s + 5, S4, S2, S0, S5);
        if (s + 6 >= ns) break;
        step(s + 6, S5, S3, S1, S6);
    }
    if (XS) {
#pragma unroll 4
        for (int k = threadIdx.x; k < n; k += NT) xg[k] = xs[k];
    }
}

template <typename T>
int gs_rows(const DCsr<T> &A, int kind, const int *rows, int cnt, const T *d,
            T w, const T *b, T *x, cudaStream_t s) {
    if (cnt <= 0) return SUCCESS;
    const int skip = (kind & GS_SKIP_LAST) ? A.n - 1 : -1;
    k_gs_rows<T><<<grid_for(cnt), 256, 0, s>>>(cnt, rows, A.ia, A.ja, A.val, d,
                                               kind & 15, w, b, x, skip);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
// raise a kernel's dynamic shared memory limit once per process
template <typename K>
static void gs_smem_limit(K kernel, bool &done) {
    if (!done) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)GS_SMEM_MAX);
        done = true;
    }
}

// the four-stage run kernel (any thread count): x in shared memory when the
// level fits, else in global memory
template <typename T, int NT, int P>
static int gs_pipe_launch(const DCsr<T> &A, int kd, const int *rows, const int *set_ptr,
                          int first, int last, const T *d, T w, const T *b, T *x, int skip,
                          cudaStream_t s) {
    const size_t spb = gs_sp_bytes(last - first);
    const size_t xsb = sizeof(T) * (size_t)A.n;
    if (spb + xsb <= GS_SMEM_MAX) {
        static bool done = false;
        gs_smem_limit(k_gs_pipe<T, NT, P, true>, done);
        k_gs_pipe<T, NT, P, true><<<1, NT, spb + xsb, s>>>(rows, set_ptr, first, last, A.n,
                                                           A.ia, A.ja, A.val, d, kd, w, b, x,
                                                           skip);
    } else {
        k_gs_pipe<T, NT, P, false><<<1, NT, spb, s>>>(rows, set_ptr, first, last, A.n, A.ia,
                                                      A.ja, A.val, d, kd, w, b, x, skip);
    }
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

// the deep run kernel (at most 256 threads): x in shared memory when the
// level fits, else in global memory
template <typename T, int NT, int P>
static int gs_deep_launch(const DCsr<T> &A, int kd, const int *rows, const int *set_ptr,
                          int first, int last, const T *d, T w, const T *b, T *x, int skip,
                          cudaStream_t s) {
    const size_t spb = gs_sp_bytes(last - first);
    const size_t xsb = sizeof(T) * (size_t)A.n;
    if (spb + xsb <= GS_SMEM_MAX) {
        static bool done = false;
        gs_smem_limit(k_gs_deep<T, NT, P, true>, done);
        k_gs_deep<T, NT, P, true><<<1, NT, spb + xsb, s>>>(rows, set_ptr, first, last, A.n,
                                                           A.ia, A.ja, A.val, d, kd, w, b, x,
                                                           skip);
    } else {
        k_gs_deep<T, NT, P, false><<<1, NT, spb, s>>>(rows, set_ptr, first, last, A.n, A.ia,
                                                      A.ja, A.val, d, kd, w, b, x, skip);
    }
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

template <typename T>
int gs_run(const DCsr<T> &A, int kind, const int *rows, const int *set_ptr,
           int first, int last, int max_set, const T *d, T w, const T *b, T *x,
           cudaStream_t s) {
    if (last <= first) return SUCCESS;
    if (last - first > GS_RUN_SETS || max_set > GS_SMALL_SET) return ERROR_INPUT_PAR;
    const int skip = (kind & GS_SKIP_LAST) ? A.n - 1 : -1;
    const int kd = kind & 15;
    // up to 256 rows a set: the deep pipeline (HZB_GS_DEEP=0: the four-stage
    // one; same results); larger sets: four stages, 8 entries per row held
    // ahead up to 512 threads, fewer at 1024 (64 registers a thread)
    constexpr int P1024 = sizeof(T) == 8 ? 2 : 4;
    static const bool deep = [] {
        const char *e = getenv("HZB_GS_DEEP");
        return !(e && e[0] == '0');
    }();
    if (max_set <= 128)
        return deep ? gs_deep_launch<T, 128, 8>(A, kd, rows, set_ptr, first, last, d, w, b, x,
                                                skip, s)
                    : gs_pipe_launch<T, 128, 8>(A, kd, rows, set_ptr, first, last, d, w, b, x,
                                                skip, s);
    if (max_set <= 256)
        return deep ? gs_deep_launch<T, 256, 8>(A, kd, rows, set_ptr, first, last, d, w, b, x,
                                                skip, s)
                    : gs_pipe_launch<T, 256, 8>(A, kd, rows, set_ptr, first, last, d, w, b, x,
                                                skip, s);
    if (max_set <= 512)
        return gs_pipe_launch<T, 512, 8>(A, kd, rows, set_ptr, first, last, d, w, b, x, skip,
                                         s);
    return gs_pipe_launch<T, 1024, P1024>(A, kd, rows, set_ptr, first, last, d, w, b, x, skip,
                                          s);
}
// ---------------------------------------------------------------------------
// Consecutive large level sets in one cooperative launch, the sets separated
// by grid_barrier (hzb_kernels.cuh).  x is read and written at L2
// (ld/st.global.cg): the CTAs of other SMs wrote it.
// ---------------------------------------------------------------------------
// One row per thread per set when the grid covers the largest set (the
// launch sizes it so): the row data of the next set is loaded before each
// barrier, as in k_gs_run; rows beyond the grid (a set larger than the
// co-resident threads) are swept with plain loads.
template <typename T>
__global__ void __launch_bounds__(256)
k_gs_sets_grid(const int *__restrict__ rows, const int *__restrict__ set_ptr, int first,
               int last, const int *__restrict__ ia, const int *__restrict__ ja,
               const T *__restrict__ a, const T *__restrict__ d, int kind, T w,
               const T *__restrict__ b, T *x, int skip, unsigned *bar, int *err) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthr = gridDim.x * blockDim.x;
    constexpr int P = 16;
    GsRowData<T, P> cur, nxt;
    int q0 = set_ptr[first], q1 = set_ptr[first + 1];
    gs_row_load(cur, rows, q0 + gtid, q1, ia, ja, a, d, b);
    for (int sidx = first; sidx < last; ++sidx) {
        const int i = cur.i;
        if (i >= 0 && i != skip) {
            T t = cur.bi;
            T xv[P];
#pragma unroll
            for (int u = 0; u < P; ++u)
                xv[u] = cur.k0 + u < cur.k1 ? __ldcg(x + cur.col[u]) : T(0);
#pragma unroll
            for (int u = 0; u < P; ++u)
                if (cur.k0 + u < cur.k1 && cur.col[u] != i) t -= cur.val[u] * xv[u];
            for (int k = cur.k0 + P; k < cur.k1; ++k) {
                const int j = ja[k];
                if (j != i) t -= a[k] * __ldcg(x + j);
            }
            const T di = cur.di;
            if (kind == 0) {
                __stcg(x + i, t * di);
            } else if (kind == 1) {
                if (fabs(di) > T(SMALLREAL)) __stcg(x + i, w * (t / di) + (1 - w) * __ldcg(x + i));
            } else {
                if (fabs(di) > T(SMALLREAL)) __stcg(x + i, t / di);
            }
        }
        for (int q = q0 + gtid + nthr; q < q1; q += nthr) {   // beyond one row per thread
            const int r = rows[q];
            if (r == skip) continue;
            T t = b[r];
            for (int k = ia[r]; k < ia[r + 1]; ++k) {
                const int j = ja[k];
                if (j != r) t -= a[k] * __ldcg(x + j);
            }
            const T di = d[r];
            if (kind == 0) {
                __stcg(x + r, t * di);
            } else if (kind == 1) {
                if (fabs(di) > T(SMALLREAL)) __stcg(x + r, w * (t / di) + (1 - w) * __ldcg(x + r));
            } else {
                if (fabs(di) > T(SMALLREAL)) __stcg(x + r, t / di);
            }
        }
        if (sidx + 1 < last) {
            q0 = q1;
            q1 = set_ptr[sidx + 2];
            gs_row_load(nxt, rows, q0 + gtid, q1, ia, ja, a, d, b);
            if (!grid_barrier(bar, gridDim.x, err)) return;
            cur = nxt;
        }
    }
}

template <typename T>
int gs_sets_grid(const DCsr<T> &A, int kind, const int *rows, const int *set_ptr, int first,
                 int last, int max_set, const T *d, T w, const T *b, T *x, unsigned *bar,
                 int *err, cudaStream_t s) {
    if (last <= first) return SUCCESS;
    static int per_sm = 0;
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs_sets_grid<T>, 256, 0) !=
                cudaSuccess || per_sm < 1)
            per_sm = 1;
    }
    const int grid = std::max(1, std::min(per_sm * sm_count(), div_up(max_set, 256)));
    const int skip = (kind & GS_SKIP_LAST) ? A.n - 1 : -1;
    const int kd = kind & 15;
    // every launch starts its barrier from zero (a wait that ran out may
    // have left an arrival counted)
    HZB_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HZB_CUDA(cudaLaunchKernelEx(&cfg, k_gs_sets_grid<T>, rows, set_ptr, first, last, A.ia,
                                A.ja, A.val, d, kd, w, b, x, skip, bar, err));
    count_launch();
    return SUCCESS;
}
template int gs_sets_grid<double>(const DCsr<double> &, int, const int *, const int *, int,
                                  int, int, const double *, double, const double *, double *,
                                  unsigned *, int *, cudaStream_t);

template int gs_rows<double>(const DCsr<double> &, int, const int *, int,
                             const double *, double, const double *, double *,
                             cudaStream_t);
template int gs_rows<float>(const DCsr<float> &, int, const int *, int,
                            const float *, float, const float *, float *,
                            cudaStream_t);
template int gs_run<double>(const DCsr<double> &, int, const int *, const int *,
                            int, int, int, const double *, double, const double *,
                            double *, cudaStream_t);
template int gs_run<float>(const DCsr<float> &, int, const int *, const int *,
                           int, int, int, const float *, float, const float *,
                           float *, cudaStream_t);

// ---------------------------------------------------------------------------
// Reductions (deterministic: fixed grid for a given n, ordered final sum)
// ---------------------------------------------------------------------------
constexpr int RED_BLOCK = 256;
int reduce_blocks(int n) {
    int g = div_up(n > 0 ? n : 1, RED_BLOCK * 4);
    int cap = sm_count() * 4;
    return g < cap ? g : cap;
}

__global__ void k_reduce_final(const double *__restrict__ part, int np,
                               double *out, int is_max) {
    __shared__ double sh[32];
    double v = 0.0;
    // each thread folds a contiguous slice in order
    const int per = (np + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per, b1 = min(b0 + per, np);
    for (int k = b0; k < b1; ++k) v = is_max ? fmax(v, part[k]) : v + part[k];
    v = is_max ? block_max(v, sh) : block_sum(v, sh);
    if (threadIdx.x == 0) out[0] = v;
}

int reduce_final(const double *part, int np, double *out, cudaStream_t s) {
    k_reduce_final<<<1, 256, 0, s>>>(part, np, out, 0);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
int reduce_final_max(const double *part, int np, double *out, cudaStream_t s) {
    k_reduce_final<<<1, 256, 0, s>>>(part, np, out, 1);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

__global__ void k_dot_partial(int n, const double *__restrict__ x,
                              const double *__restrict__ y, double *part) {
    __shared__ double sh[32];
    double v = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        v += x[i] * y[i];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
}

int dot_partial(int n, const double *x, const double *y, double *part,
                cudaStream_t s) {
    k_dot_partial<<<reduce_blocks(n), RED_BLOCK, 0, s>>>(n, x, y, part);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
int dot(int n, const double *x, const double *y, double *part, double *out,
        cudaStream_t s) {
    HZB_TRY(dot_partial(n, x, y, part, s));
    return reduce_final(part, reduce_blocks(n), out, s);
}

// part4 layout: [0..G) (r,r)  [G..2G) max|u|  [2G..3G) (u,u)  [3G..4G) (p,p)
__global__ void k_pcg_update(int n, const double *__restrict__ num,
                             const double *__restrict__ den, double *u,
                             double *r, const double *__restrict__ p,
                             const double *__restrict__ t, double *part4) {
    __shared__ double sh[32];
    const double alpha = num[0] / den[0];
    double rr = 0.0, um = 0.0, uu = 0.0, pp = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const double pi = p[i];
        double ui = u[i];
        if (alpha == 1.0) ui += pi;
        else if (alpha == -1.0) ui -= pi;
        else ui += alpha * pi;
        const double ma = -alpha;
        double ri = r[i];
        const double ti = t[i];
        if (ma == 1.0) ri += ti;
        else if (ma == -1.0) ri -= ti;
        else ri += ma * ti;
        u[i] = ui;
        r[i] = ri;
        rr += ri * ri;
        um = fmax(um, fabs(ui));
        uu += ui * ui;
        pp += pi * pi;
    }
    const int G = gridDim.x;
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) part4[blockIdx.x] = rr;
    um = block_max(um, sh);
    if (threadIdx.x == 0) part4[G + blockIdx.x] = um;
    uu = block_sum(uu, sh);
    if (threadIdx.x == 0) part4[2 * G + blockIdx.x] = uu;
    pp = block_sum(pp, sh);
    if (threadIdx.x == 0) part4[3 * G + blockIdx.x] = pp;
}

int pcg_update(int n, const double *num, const double *den, double *u,
               double *r, const double *p, const double *t, double *part4,
               cudaStream_t s) {
    k_pcg_update<<<reduce_blocks(n), RED_BLOCK, 0, s>>>(n, num, den, u, r, p, t,
                                                        part4);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

__global__ void k_pcg_axpby(int n, const double *__restrict__ num,
                            const double *__restrict__ den,
                            const double *__restrict__ z, double *p) {
    const double beta = num[0] / den[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        p[i] = 1.0 * z[i] + beta * p[i];
}

int pcg_axpby(int n, const double *num, const double *den, const double *z,
              double *p, cudaStream_t s) {
    k_pcg_axpby<<<grid_for(n), 256, 0, s>>>(n, num, den, z, p);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

template <typename T>
__global__ void k_copy(int n, const T *__restrict__ x, T *__restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        y[i] = x[i];
}
template <typename T>
__global__ void k_zero(int n, T *__restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        y[i] = T(0);
}
template <typename T>
int vcopy(int n, const T *x, T *y, cudaStream_t s) {
    if (n <= 0) return SUCCESS;
    k_copy<T><<<grid_for(n), 256, 0, s>>>(n, x, y);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
template <typename T>
int vzero(int n, T *y, cudaStream_t s) {
    if (n <= 0) return SUCCESS;
    k_zero<T><<<grid_for(n), 256, 0, s>>>(n, y);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
template int vcopy<double>(int, const double *, double *, cudaStream_t);
template int vcopy<float>(int, const float *, float *, cudaStream_t);
template int vcopy<int>(int, const int *, int *, cudaStream_t);
template int vzero<double>(int, double *, cudaStream_t);
template int vzero<float>(int, float *, cudaStream_t);

__global__ void k_d2f(int n, const double *__restrict__ x, float *__restrict__ y,
                      const unsigned char *__restrict__ act) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        if (!act || act[i / ACT_ROWS]) y[i] = (float)x[i];
}
__global__ void k_f2d(int n, const float *__restrict__ x, double *__restrict__ y,
                      const unsigned char *__restrict__ act) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        if (!act || act[i / ACT_ROWS]) y[i] = (double)x[i];
}
int d2f(int n, const double *x, float *y, cudaStream_t s, const unsigned char *act) {
    if (n <= 0) return SUCCESS;
    k_d2f<<<grid_for(n), 256, 0, s>>>(n, x, y, act);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
int f2d(int n, const float *x, double *y, cudaStream_t s, const unsigned char *act) {
    if (n <= 0) return SUCCESS;
    k_f2d<<<grid_for(n), 256, 0, s>>>(n, x, y, act);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
// FP32 copy of a CSR matrix without its exactly-zero entries (row order kept)
__global__ void k_nz_count(int n, const int *__restrict__ ia, const double *__restrict__ a,
                           int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        int c = 0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) c += a[k] != 0.0;
        cnt[i] = c;
    }
}
__global__ void k_nz_fill(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                          const double *__restrict__ a, const int *__restrict__ ia32,
                          int *ja32, float *a32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        int p = ia32[i];
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (a[k] != 0.0) { ja32[p] = ja[k]; a32[p] = (float)a[k]; ++p; }
    }
}
int csr_nonzero_count(int n, const int *ia, const double *a, int *cnt, cudaStream_t s) {
    k_nz_count<<<grid_for(n), 256, 0, s>>>(n, ia, a, cnt);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
int csr_nonzero_fill(int n, const int *ia, const int *ja, const double *a, const int *ia32,
                     int *ja32, float *a32, cudaStream_t s) {
    k_nz_fill<<<grid_for(n), 256, 0, s>>>(n, ia, ja, a, ia32, ja32, a32);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

// the FP64 values of the same entries (the FP32 copy's pattern)
__global__ void k_nz_fill64(int n, const int *__restrict__ ia, const double *__restrict__ a,
                            const int *__restrict__ ia32, double *a64) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        int p = ia32[i];
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (a[k] != 0.0) a64[p++] = a[k];
    }
}
int csr_nonzero_fill64(int n, const int *ia, const double *a, const int *ia32, double *a64,
                       cudaStream_t s) {
    k_nz_fill64<<<grid_for(n), 256, 0, s>>>(n, ia, a, ia32, a64);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

int csr_val_d2f(int nnz, const double *x, float *y, cudaStream_t s) {
    return d2f(nnz, x, y, s);
}

// ---------------------------------------------------------------------------
// Coarse level: y = Ainv x, one warp per row, FP64 accumulation
// ---------------------------------------------------------------------------
template <typename TI>
__global__ void k_gemv(int n, const double *__restrict__ M,
                       const TI *__restrict__ x, TI *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < n; r += nwarps) {
        const double *row = M + (size_t)r * n;
        double t = 0.0;
        for (int c = lane; c < n; c += 32) t += row[c] * (double)x[c];
        t = warp_sum(t);
        if (lane == 0) y[r] = (TI)t;
    }
}

template <typename TI>
int dense_gemv(int n, const double *Ainv, const TI *x, TI *y, cudaStream_t s) {
    if (n <= 0) return SUCCESS;
    const int grid = div_up((long long)n * 32, 256);
    k_gemv<TI><<<grid, 256, 0, s>>>(n, Ainv, x, y);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}
template int dense_gemv<double>(int, const double *, const double *, double *,
                                cudaStream_t);
template int dense_gemv<float>(int, const double *, const float *, float *,
                               cudaStream_t);

}  // namespace hzb
