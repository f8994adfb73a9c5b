// hzb_common.cuh -- shared device helpers of the B200 UA-AMG library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include "../../include/hazmath_b200.h"

namespace hzb {

// Error reporting: the last CUDA failure of this thread, as text.
void set_error(cudaError_t e, const char *file, int line);
void set_error_msg(const std::string &msg);
const char *last_error();

#define HZB_CUDA(call)                                                     \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) {                                           \
            ::hzb::set_error(e_, __FILE__, __LINE__);                      \
            return ERROR_SOLVER_MISC;                                      \
        }                                                                  \
    } while (0)

#define HZB_LAUNCH_CHECK() HZB_CUDA(cudaGetLastError())

#define HZB_TRY(expr)                                                      \
    do {                                                                   \
        int rc_ = (expr);                                                  \
        if (rc_ < 0) return rc_;                                           \
    } while (0)

// Number of SMs of the current device (148 on B200), cached.
int sm_count();

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// Grid for a grid-stride elementwise kernel: at most 8 resident 256-thread
// blocks per SM.
inline int grid_for(long long n, int block = 256) {
    long long g = (n + block - 1) / block;
    long long cap = (long long)sm_count() * 8;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// Device allocations are stream-ordered (cudaMallocAsync / cudaFreeAsync on
// the calling solver's stream, from the device's default pool with its
// release threshold raised so freed blocks stay cached): rebuilding a
// hierarchy does not pay cudaMalloc/cudaFree and their device-wide syncs.
// The stream is a thread-local set by StreamScope at each entry point
// (legacy default stream otherwise).
cudaStream_t &cur_stream();
void ensure_pool();
struct StreamScope {
    cudaStream_t prev;
    explicit StreamScope(cudaStream_t s) : prev(cur_stream()) { cur_stream() = s; ensure_pool(); }
    ~StreamScope() { cur_stream() = prev; }
};

// Device allocation helpers (return ERROR_ALLOC_MEM on failure).
template <typename T>
int dalloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocAsync((void **)p, count * sizeof(T), cur_stream());
    if (e != cudaSuccess) {
        set_error(e, __FILE__, __LINE__);
        *p = nullptr;
        return ERROR_ALLOC_MEM;
    }
    return SUCCESS;
}
template <typename T>
void dfree(T *&p) {
    if (p) cudaFreeAsync((void *)p, cur_stream());
    p = nullptr;
}

// Warp-level sum in a fixed butterfly order (deterministic).
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = v > w ? v : w;
    }
    return v;
}

// Block sum over blockDim.x threads (multiple of 32, <= 1024); result valid
// in thread 0.  Fixed order: warp butterflies, then warp 0 over warp sums.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T *sh /* >= 32 */) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : T(0);
    if (wid == 0) v = warp_sum(v);
    __syncthreads();
    return v;
}
template <typename T>
__device__ __forceinline__ T block_max(T v, T *sh) {
    v = warp_max(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : T(0);
    if (wid == 0) v = warp_max(v);
    __syncthreads();
    return v;
}

// Launch counter of the calling thread (kernels issued by this library).
void count_launch(int k = 1);
long long launch_count();

}  // namespace hzb
