// hzb_setup.cu -- setup-phase kernels of the UA-AMG hierarchy.
// Compiled with -fmad=false like the cycle kernels: the Galerkin sums are
// rounded in the reference's order.
#include "hzb_setup.cuh"
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace hzb {

// ---------------------------------------------------------------------------
// exclusive scan (int32)
// ---------------------------------------------------------------------------
constexpr int SCAN_BLOCK = 256, SCAN_ITEMS = 8, SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ int block_exscan(int v, int *sh, int *total) {
    // inclusive warp scan
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    if (wid == 0) {
        int w = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) sh[lane] = w;   // inclusive warp totals
    }
    __syncthreads();
    const int before = wid > 0 ? sh[wid - 1] : 0;
    *total = sh[nw - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void k_scan_tiles(const int *__restrict__ in, int n, int *tiles) {
    __shared__ int sh[32];
    const int base = blockIdx.x * SCAN_TILE;
    int v = 0;
    for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_BLOCK) {
        int i = base + k;
        if (i < n) v += in[i];
    }
    int tot;
    block_exscan(v, sh, &tot);
    if (threadIdx.x == 0) tiles[blockIdx.x] = tot;
}

__global__ void k_scan_tilesums(int *tiles, int nt) {
    __shared__ int sh[32];
    int carry = 0;
    for (int b = 0; b < nt; b += blockDim.x) {
        int i = b + threadIdx.x;
        int v = i < nt ? tiles[i] : 0;
        int tot;
        int ex = block_exscan(v, sh, &tot);
        if (i < nt) tiles[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) tiles[nt] = carry;
}

__global__ void k_scan_apply(const int *__restrict__ in, int *out, int n,
                             const int *__restrict__ tiles) {
    __shared__ int sh[32];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int i = base + k;
        v[k] = i < n ? in[i] : 0;
        sum += v[k];
    }
    int tot;
    int ex = block_exscan(sum, sh, &tot) + tiles[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = tiles[gridDim.x];
}

int scan_tmp_size(int n) { return div_up(n > 0 ? n : 1, SCAN_TILE) + 1; }

int scan_exclusive(const int *in, int *out, int n, int *tmp, cudaStream_t s) {
    if (n <= 0) {
        HZB_CUDA(cudaMemsetAsync(out, 0, sizeof(int), s));
        return SUCCESS;
    }
    const int nt = div_up(n, SCAN_TILE);
    k_scan_tiles<<<nt, SCAN_BLOCK, 0, s>>>(in, n, tmp);
    k_scan_tilesums<<<1, 1024, 0, s>>>(tmp, nt);
    k_scan_apply<<<nt, SCAN_BLOCK, 0, s>>>(in, out, n, tmp);
    count_launch(3);
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// strength graph
// ---------------------------------------------------------------------------
__global__ void k_first_diag(int n, const int *__restrict__ ia,
                             const int *__restrict__ ja, const double *__restrict__ a,
                             double *d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (ja[k] == i) { v = a[k]; break; }
        d[i] = v;
    }
}

__device__ __forceinline__ bool strong(int i, int j, double v, double th2,
                                       const double *d) {
    return j == i || ((v * v) >= th2 * fabs(d[i] * d[j]) && v < 0e0);
}

__global__ void k_strength_count(int n, const int *__restrict__ ia,
                                 const int *__restrict__ ja,
                                 const double *__restrict__ a,
                                 const double *__restrict__ d, double th2,
                                 int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        int c = 0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) c += strong(i, ja[k], a[k], th2, d);
        cnt[i] = c;
    }
}

__global__ void k_strength_fill(int n, const int *__restrict__ ia,
                                const int *__restrict__ ja,
                                const double *__restrict__ a,
                                const double *__restrict__ d, double th2,
                                const int *__restrict__ nia, int *nja,
                                double *nval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        int p = nia[i];
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (strong(i, ja[k], a[k], th2, d)) { nja[p] = ja[k]; nval[p] = a[k]; ++p; }
    }
}

int strength_graph(const DCsr<double> &A, double theta, int *nia, int *nja,
                   double *nval, int *nnnz, int *tmp, cudaStream_t s) {
    const int n = A.n;
    double *d = nullptr;
    int *cnt = nullptr;
    HZB_TRY(dalloc(&d, n));
    int rc = dalloc(&cnt, n);
    if (rc) { dfree(d); return rc; }
    const double th2 = theta * theta;
    const int g = grid_for(n);
    k_first_diag<<<g, 256, 0, s>>>(n, A.ia, A.ja, A.val, d);
    k_strength_count<<<g, 256, 0, s>>>(n, A.ia, A.ja, A.val, d, th2, cnt);
    count_launch(2);
    rc = scan_exclusive(cnt, nia, n, tmp, s);
    if (!rc) {
        k_strength_fill<<<g, 256, 0, s>>>(n, A.ia, A.ja, A.val, d, th2, nia, nja, nval);
        count_launch();
        cudaError_t e = cudaMemcpyAsync(nnnz, nia + n, sizeof(int),
                                        cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; }
    }
    dfree(d);
    dfree(cnt);
    return rc;
}

// ---------------------------------------------------------------------------
// heavy edge matching, reference order: one warp walks the vertices in
// ascending order; the 32 lanes examine a row's neighbours together.
// ---------------------------------------------------------------------------
// Candidate order of heavy_edg(w, id, iz-1, 0): the largest weight wins, and
// among equal weights the later position in the row (backward scan, strict >).
__device__ __forceinline__ void better_last(double &w, int &p, double w2, int p2) {
    if (p2 >= 0 && (p < 0 || w2 > w || (w2 == w && p2 > p))) { w = w2; p = p2; }
}
// heavy_edg(w, id, 0, iz-1): largest weight, among equals the earlier position.
__device__ __forceinline__ void better_first(double &w, int &p, double w2, int p2) {
    if (p2 >= 0 && (p < 0 || w2 > w || (w2 == w && p2 < p))) { w = w2; p = p2; }
}

__global__ void __launch_bounds__(32)
k_hem_seq(int n, const int *__restrict__ ia, const int *__restrict__ ja,
          const double *__restrict__ a, int *mask_, int *cnt_, int *out) {
    volatile int *mask = mask_;
    volatile int *cnt = cnt_;
    const int lane = threadIdx.x;
    for (int k = lane; k < n; k += 32) {
        mask[k] = (ia[k + 1] - ia[k] > 1) ? -1 : -2;   // pass 0
        cnt[k] = 0;
    }
    __syncwarp();
    int nc = 0;
    for (int k = 0; k < n; ++k) {                      // pass 1
        if (mask[k] != -1) continue;
        const int b0 = ia[k], b1 = ia[k + 1];
        double bw = 0.0;
        int bp = -1;
        for (int p = b0 + lane; p < b1; p += 32) {
            const int j = ja[p];
            if (j != k && mask[j] < 0) better_last(bw, bp, fabs(a[p]), p);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double w2 = __shfl_xor_sync(0xffffffffu, bw, o);
            int p2 = __shfl_xor_sync(0xffffffffu, bp, o);
            better_last(bw, bp, w2, p2);
        }
        if (bp >= 0) {
            if (lane == 0) {
                const int pick = ja[bp];
                mask[k] = nc;
                mask[pick] = nc;
                cnt[nc] = 2;
            }
            ++nc;
        }
        __syncwarp();
    }
    int status = 0;
    for (int k = 0; k < n; ++k) {                      // pass 2
        if (mask[k] != -1) continue;
        const int b0 = ia[k], b1 = ia[k + 1];
        double bw = 0.0;
        int bp = -1, bc = -1;
        for (int p = b0 + lane; p < b1; p += 32) {
            const int kc = mask[ja[p]];
            if (kc >= 0) {
                double w2 = (double)(-cnt[kc]);
                int oldp = bp;
                better_first(bw, bp, w2, p);
                if (bp != oldp) bc = kc;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double w2 = __shfl_xor_sync(0xffffffffu, bw, o);
            int p2 = __shfl_xor_sync(0xffffffffu, bp, o);
            int c2 = __shfl_xor_sync(0xffffffffu, bc, o);
            int oldp = bp;
            better_first(bw, bp, w2, p2);
            if (bp != oldp) bc = c2;
        }
        if (bp < 0) { status = -1; break; }
        if (lane == 0) {
            mask[k] = bc;
            cnt[bc] = cnt[bc] + 1;
        }
        __syncwarp();
    }
    __syncwarp();
    for (int k = lane; k < n; k += 32)                 // pass 3
        if (mask[k] < 0) mask[k] = UNPT;
    if (lane == 0) { out[0] = nc; out[1] = status; }
}

// --- the same matching with the pass-1 state in shared memory -------------
// Pass 1 only asks "is j already matched?".  While every neighbour index is
// within B of its row (B = the graph's bandwidth), the vertices in play at
// step k lie in [k - B, k + B], so one bit per vertex in a ring of RING bits
// (RING > 2B) indexed by v mod RING holds that state; the slot of vertex
// k + B is cleared when step k begins (its previous owner, k + B - RING,
// finished long ago).  Pass 2 then visits only the vertices left unmatched.
constexpr int HEM_RING_BITS = 1 << 20;                 // 128 KB of shared memory
constexpr int HEM_RING_WORDS = HEM_RING_BITS / 32;

// bw[0] = max |j - i| over the stored entries, bw[1] = longest row
__global__ void k_graph_bandwidth(int n, const int *__restrict__ ia,
                                  const int *__restrict__ ja, int *bw) {
    __shared__ int sh[32];
    int b = 0, len = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        for (int k = ia[i]; k < ia[i + 1]; ++k) b = max(b, abs(ja[k] - i));
        len = max(len, ia[i + 1] - ia[i]);
    }
    b = block_max(b, sh);
    len = block_max(len, sh);
    if (threadIdx.x == 0) { atomicMax(bw, b); atomicMax(bw + 1, len); }
}

__global__ void k_hem_init(int n, const int *__restrict__ ia, int *mask, int *cnt) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += gridDim.x * blockDim.x) {
        mask[k] = (ia[k + 1] - ia[k] > 1) ? -1 : -2;   // pass 0
        cnt[k] = 0;
    }
}

__global__ void __launch_bounds__(32)
k_hem_pass1_ring(int n, int bw, const int *__restrict__ ia, const int *__restrict__ ja,
                 const double *__restrict__ a, int *mask, int *cnt, int *out) {
    extern __shared__ unsigned ring[];
    const int lane = threadIdx.x;
    for (int w = lane; w < HEM_RING_WORDS; w += 32) ring[w] = 0u;
    __syncwarp();
    constexpr unsigned RM = HEM_RING_BITS - 1;
    int nc = 0;
    for (int k = 0; k < n; ++k) {
        if (lane == 0) {
            const unsigned v = (unsigned)(k + bw) & RM;   // entering the window
            ring[v >> 5] &= ~(1u << (v & 31));
        }
        __syncwarp();
        const unsigned vk = (unsigned)k & RM;
        const bool matched = (ring[vk >> 5] >> (vk & 31)) & 1u;
        const int b0 = __ldg(ia + k), b1 = __ldg(ia + k + 1);
        if (matched || b1 - b0 <= 1) continue;   // already paired / pass-0 isolated
        double bwgt = 0.0;
        int bp = -1;
        for (int p = b0 + lane; p < b1; p += 32) {
            const int j = __ldg(ja + p);
            const unsigned vj = (unsigned)j & RM;
            const bool mj = (ring[vj >> 5] >> (vj & 31)) & 1u;
            if (j != k && !mj) better_last(bwgt, bp, fabs(__ldg(a + p)), p);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double w2 = __shfl_xor_sync(0xffffffffu, bwgt, o);
            int p2 = __shfl_xor_sync(0xffffffffu, bp, o);
            better_last(bwgt, bp, w2, p2);
        }
        if (bp >= 0) {
            if (lane == 0) {
                const int pick = __ldg(ja + bp);
                const unsigned vp = (unsigned)pick & RM;
                ring[vk >> 5] |= 1u << (vk & 31);
                ring[vp >> 5] |= 1u << (vp & 31);
                mask[k] = nc;
                mask[pick] = nc;
                cnt[nc] = 2;
            }
            ++nc;
        }
        __syncwarp();
    }
    if (lane == 0) out[0] = nc;
}

// --- pass 1 with pre-ranked candidate lists ---------------------------------
// Pass 1 of vertex k takes, among the unmatched neighbours j != k, the entry
// of largest |a_kj|, ties to the later position.  That order does not depend
// on the matching state, so a parallel kernel first writes every row's
// neighbours in that order (self entries as -1 at the end), and the
// sequential walk only looks for the first unmatched entry of the list.
// The walk streams the lists through shared memory in tiles of 32 rows with
// cp.async, HEM_PIPE tiles ahead of the tile it works on, so no global load
// latency sits on its critical path.
constexpr int HEM_PIPE = 4;                 // tiles in flight ahead of the walk
constexpr int HEM_TILE_CAP = 3072;          // staged candidates per tile
constexpr int HEM_RANK_MAXLEN = 4096;       // longest row the ranking accepts
// slots: the tiles in flight plus the one being walked
constexpr int HEM_IA_SLOTS = 2 * HEM_PIPE + 2, HEM_IA_STRIDE = 36;
constexpr int HEM_C_SLOTS = HEM_PIPE + 2;
constexpr int HEM_MISC_WORDS = 32 * 2 + 32 + 2 * 32 + 2;   // info, Pm, picks, accepted
constexpr size_t HEM_STAGED_SMEM =
    (size_t)HEM_RING_WORDS * 4 + (size_t)HEM_C_SLOTS * HEM_TILE_CAP * 4 +
    (size_t)HEM_IA_SLOTS * HEM_IA_STRIDE * 4 + (size_t)HEM_MISC_WORDS * 4;

// one warp per row: rank of entry p = number of entries that come before it
__global__ void k_hem_rank(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                           const double *__restrict__ a, int *__restrict__ cand) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nw) {
        const int b0 = ia[k], b1 = ia[k + 1];
        int nself = 0;
        for (int p = b0 + lane; p < b1; p += 32) nself += ja[p] == k;
        for (int o = 16; o > 0; o >>= 1) nself += __shfl_xor_sync(0xffffffffu, nself, o);
        const int nother = b1 - b0 - nself;
        for (int p = b0 + lane; p < b1; p += 32) {
            const int j = ja[p];
            int r = 0;
            if (j != k) {
                const double w = fabs(a[p]);
                for (int q = b0; q < b1; ++q) {
                    if (ja[q] == k) continue;
                    const double w2 = fabs(a[q]);
                    r += (w2 > w) || (w2 == w && q > p);
                }
                cand[b0 + r] = j;
            } else {
                for (int q = b0; q < p; ++q) r += ja[q] == k;
                cand[b0 + nother + r] = -1;
            }
        }
    }
}

__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The matched state of the vertices in play lives in a ring of shared memory:
// one byte per vertex (BYTES, 2^17 vertices, plain stores) while the window
// fits, else one bit per vertex (2^20 vertices, atomicOr).  Both rings take
// 128 KB.  Ring size > 2 bw + 64: the 32 slots entering the window are
// cleared when a tile begins (vertices >= r0 + bw cannot be matched before
// tile r0 starts, and the slot's previous owner lies below r0 - bw).
template <bool BYTES>
struct HemRing {
    static constexpr unsigned SIZE = BYTES ? (1u << 17) : (1u << 20);
    static constexpr unsigned RM = SIZE - 1;
    void *mem;
    __device__ __forceinline__ bool get(int v) const {
        const unsigned u = (unsigned)v & RM;
        if (BYTES) return ((const volatile unsigned char *)mem)[u] != 0;
        return (((const volatile unsigned *)mem)[u >> 5] >> (u & 31)) & 1u;
    }
    __device__ __forceinline__ void set(int v) {
        const unsigned u = (unsigned)v & RM;
        if (BYTES) ((volatile unsigned char *)mem)[u] = 1;
        else atomicOr((unsigned *)mem + (u >> 5), 1u << (u & 31));
    }
    // vertices v0 .. v0 + 31, by the whole warp
    __device__ __forceinline__ void clear32(int v0, int lane) {
        if (BYTES) {
            ((unsigned char *)mem)[((unsigned)v0 + lane) & RM] = 0;
        } else {
            const unsigned u = (unsigned)v0 & RM, sh = u & 31u, w0 = u >> 5;
            unsigned *w = (unsigned *)mem;
            if (lane == 0) w[w0] &= ~(0xffffffffu << sh);
            if (lane == 1 && sh) w[(w0 + 1) & (SIZE / 32 - 1)] &= ~((1u << sh) - 1u);
        }
    }
};

// Two warps.  Warp 1 streams row pointers and ranked lists into shared
// memory (cp.async, HEM_PIPE tiles ahead) and writes the pairs of finished
// tiles to mask/cnt; warp 0 walks the tiles.  Within a tile of 32 rows every
// row first takes its best candidate unmatched when the tile starts; rows are
// then settled in order.  A row keeps that choice unless an earlier row of
// the tile took it or matched the row's choice (vertices only ever become
// matched, so the entries ranked above it stay ineligible); such a row scans
// its list again.  For a row that keeps its choice the effect on the rows
// after it is known in advance: the row it picks leaves the walk (rm) and the
// rows that wanted the same vertex or this row go stale (st).
template <bool BYTES>
__global__ void __launch_bounds__(64)
k_hem_pass1_staged(int n, int bw, const int *__restrict__ ia, const int *__restrict__ cand,
                   int *mask, int *cnt, int *out) {
    extern __shared__ unsigned hem_smem[];
    HemRing<BYTES> ring{hem_smem};
    int *cbuf = (int *)(hem_smem + HEM_RING_WORDS);
    int *iabuf = cbuf + HEM_C_SLOTS * HEM_TILE_CAP;
    uint2 *info = (uint2 *)(iabuf + HEM_IA_SLOTS * HEM_IA_STRIDE);
    unsigned *pm = (unsigned *)(info + 32);
    int *picks = (int *)(pm + 32);              // [2][32], by tile parity
    unsigned *accepted = (unsigned *)(picks + 64);   // [2]
    const int lane = threadIdx.x & 31;
    const int ntiles = (n + 31) >> 5;

    if (threadIdx.x >= 32) {   // ---- warp 1: staging and output
        int nc = 0;
        auto emit = [&](int u) {
            const unsigned acc = accepted[u & 1];
            if ((acc >> lane) & 1u) {
                const int id = nc + __popc(acc & ((1u << lane) - 1u));
                const int q = picks[(u & 1) * 32 + lane];
                mask[(u << 5) + lane] = id;
                mask[q] = id;
                cnt[id] = 2;
            }
            nc += __popc(acc);
        };
        for (int j = -2 * HEM_PIPE; j < ntiles; ++j) {
            if (j >= 2) emit(j - 2);
            const int ui = j + 2 * HEM_PIPE;   // row pointers of tile j + 2 PIPE
            if (ui < ntiles) {
                const int r0 = ui << 5, rows = min(32, n - r0);
                int *dst = iabuf + (ui % HEM_IA_SLOTS) * HEM_IA_STRIDE;
                cp_async4(dst + lane, ia + r0 + min(lane, rows));
                if (lane == 0) cp_async4(dst + 32, ia + r0 + rows);
            }
            cp_async_wait<HEM_PIPE - 1>();   // ia(j + PIPE) and cand(j) have landed
            __syncwarp();
            const int uc = j + HEM_PIPE;     // ranked lists of tile j + PIPE
            if (uc >= 0 && uc < ntiles) {
                const int *iu = iabuf + (uc % HEM_IA_SLOTS) * HEM_IA_STRIDE;
                const int rows = min(32, n - (uc << 5));
                const int e0 = iu[0], m = iu[rows] - e0;
                if (m <= HEM_TILE_CAP) {
                    int *dst = cbuf + (uc % HEM_C_SLOTS) * HEM_TILE_CAP;
                    for (int e = lane; e < m; e += 32) cp_async4(dst + e, cand + e0 + e);
                }
            }
            cp_async_commit();
            if (j >= 0) __syncthreads();   // tile j is ready; tile j - 1 is walked
        }
        cp_async_wait<0>();
        __syncthreads();                    // the last tile is walked
        if (ntiles >= 2) emit(ntiles - 2);
        if (ntiles >= 1) emit(ntiles - 1);
        if (lane == 0) out[0] = nc;
        return;
    }

    // ---- warp 0: the walk
    for (int w = lane; w < HEM_RING_WORDS; w += 32) hem_smem[w] = 0u;
    __syncthreads();
    for (int t = 0; t < ntiles; ++t) {
        const int r0 = t << 5, rows = min(32, n - r0);
        ring.clear32(r0 + bw, lane);
        __syncwarp();
        const int *it = iabuf + (t % HEM_IA_SLOTS) * HEM_IA_STRIDE;
        const int e0 = it[0];
        const bool staged = it[rows] - e0 <= HEM_TILE_CAP;
        const int *ct = staged ? cbuf + (t % HEM_C_SLOTS) * HEM_TILE_CAP : cand;
        const int off = staged ? e0 : 0;
        int *pk = picks + (t & 1) * 32;
        // rows of the tile still unmatched and not isolated (pass 0)
        const bool act = lane < rows && it[lane + 1] - it[lane] > 1 && !ring.get(r0 + lane);
        unsigned todo = __ballot_sync(0xffffffffu, act);
        int p = -1;
        if (act) {
            const int b1 = it[lane + 1];
            for (int e = it[lane]; e < b1; e += 2) {
                const int c0 = ct[e - off];
                const int c1 = e + 1 < b1 ? ct[e + 1 - off] : -1;
                const bool ok0 = c0 >= 0 && !ring.get(c0);
                const bool ok1 = c1 >= 0 && !ring.get(c1);
                if (ok0) { p = c0; break; }
                if (ok1) { p = c1; break; }
            }
        }
        const unsigned tl = (unsigned)(p - r0);   // < 32: the pick is a row of this tile
        pm[lane] = 0u;
        __syncwarp();
        if (p >= 0 && tl < 32u) atomicOr(pm + tl, 1u << lane);
        const unsigned same = __match_any_sync(0xffffffffu, p);
        const unsigned has = __ballot_sync(0xffffffffu, p >= 0);
        __syncwarp();
        if (p >= 0) info[lane] = make_uint2(tl < 32u ? 1u << tl : 0u, same | pm[lane]);
        else info[lane] = make_uint2(0u, 0u);
        pk[lane] = p;
        __syncwarp();
        unsigned stale = 0u, done = 0u, racc = 0u, written = 0u;
        while (todo) {
            const int i = __ffs(todo) - 1;
            todo &= todo - 1u;
            if ((stale >> i) & 1u) {
                // the ring takes every pick of the tile so far, then row i scans again
                const unsigned w = done & has & ~written;
                if ((w >> lane) & 1u) { ring.set(r0 + lane); ring.set(p); }
                written |= w;
                __syncwarp();
                const int b0 = it[i], b1 = it[i + 1];
                int q = -1;
                for (int e = b0; e < b1; e += 32) {
                    const int c = e + lane < b1 ? ct[e + lane - off] : -1;
                    const bool ok = c >= 0 && !ring.get(c);
                    const unsigned bal = __ballot_sync(0xffffffffu, ok);
                    if (bal) {
                        q = __shfl_sync(0xffffffffu, c, __ffs(bal) - 1);
                        break;
                    }
                }
                if (q >= 0) {
                    if (lane == 0) { ring.set(r0 + i); ring.set(q); pk[i] = q; }
                    racc |= 1u << i;
                    const unsigned d = (unsigned)(q - r0);
                    if (d < 32u) todo &= ~(1u << d);
                    stale |= __ballot_sync(0xffffffffu, p == q || p == r0 + i);
                }
                __syncwarp();
                continue;
            }
            const uint2 f = info[i];
            done |= 1u << i;
            todo &= ~f.x;
            stale |= f.y;
        }
        const unsigned acc = (done & has) | racc;
        const unsigned w = done & has & ~written;
        if ((w >> lane) & 1u) { ring.set(r0 + lane); ring.set(p); }
        if (lane == 0) accepted[t & 1] = acc;
        __syncthreads();   // tile t walked; tile t + 1 staged
    }
}

__global__ void k_flag_eq(int n, const int *__restrict__ v, int val, int *flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        flag[i] = v[i] == val;
}
__global__ void k_compact(int n, const int *__restrict__ flag, const int *__restrict__ pos,
                          int *list) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        if (flag[i]) list[pos[i]] = i;
}

// pass 2 over the leftover list (ascending), one warp, reference semantics
__global__ void __launch_bounds__(32)
k_hem_pass2_list(int m, const int *__restrict__ list, const int *__restrict__ ia,
                 const int *__restrict__ ja, int *mask_, int *cnt_, int *out) {
    volatile int *mask = mask_;
    volatile int *cnt = cnt_;
    const int lane = threadIdx.x;
    int status = 0;
    for (int q = 0; q < m; ++q) {
        const int k = list[q];
        const int b0 = ia[k], b1 = ia[k + 1];
        double bwgt = 0.0;
        int bp = -1, bc = -1;
        for (int p = b0 + lane; p < b1; p += 32) {
            const int kc = mask[ja[p]];
            if (kc >= 0) {
                double w2 = (double)(-cnt[kc]);
                int oldp = bp;
                better_first(bwgt, bp, w2, p);
                if (bp != oldp) bc = kc;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double w2 = __shfl_xor_sync(0xffffffffu, bwgt, o);
            int p2 = __shfl_xor_sync(0xffffffffu, bp, o);
            int c2 = __shfl_xor_sync(0xffffffffu, bc, o);
            int oldp = bp;
            better_first(bwgt, bp, w2, p2);
            if (bp != oldp) bc = c2;
        }
        if (bp < 0) { status = -1; break; }
        if (lane == 0) {
            mask[k] = bc;
            cnt[bc] = cnt[bc] + 1;
        }
        __syncwarp();
    }
    if (lane == 0) out[1] = status;
}

__global__ void k_hem_final(int n, int *mask) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += gridDim.x * blockDim.x)
        if (mask[k] < 0) mask[k] = UNPT;
}

int hem_exact(int n, const int *nia, const int *nja, const double *nval,
              int *agg, int *nagg, int *work_n, cudaStream_t s) {
    int *out = nullptr;
    HZB_TRY(dalloc(&out, 4));
    HZB_CUDA(cudaMemsetAsync(out, 0, 4 * sizeof(int), s));
    k_graph_bandwidth<<<grid_for(n), 256, 0, s>>>(n, nia, nja, out + 2);
    count_launch();
    int gb[3] = {0, 0, 0};
    HZB_CUDA(cudaMemcpyAsync(gb, out + 2, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaMemcpyAsync(gb + 2, nia + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    const int bw = gb[0], maxlen = gb[1], gnnz = gb[2];
    // Four implementations with the same decisions, the fastest that the
    // graph allows: 1 ranked lists + byte ring, 2 ranked lists + bit ring,
    // 3 bit ring over the raw rows, 4 state in global memory.  HZB_HEM_PATH
    // names one (if the graph allows it) for tests of the others.
    int path = 4;
    if (2 * bw + 64 < (int)HemRing<true>::SIZE && maxlen <= HEM_RANK_MAXLEN) path = 1;
    else if (2 * bw + 64 < HEM_RING_BITS && maxlen <= HEM_RANK_MAXLEN) path = 2;
    else if (2 * bw + 2 < HEM_RING_BITS) path = 3;
    if (const char *f = getenv("HZB_HEM_PATH")) {
        const int want = atoi(f);
        if (want >= path && want <= 4) path = want;
    }
    int rc = SUCCESS;
    if (path <= 3) {
        int *flag = nullptr, *pos = nullptr, *list = nullptr, *tmp = nullptr;
        const int g = grid_for(n);
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_hem_pass1_ring, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 HEM_RING_WORDS * 4);
            attr = true;
        }
        if ((rc = dalloc(&flag, n)) || (rc = dalloc(&pos, n + 1)) || (rc = dalloc(&list, n)) ||
            (rc = dalloc(&tmp, scan_tmp_size(n + 1)))) {
            dfree(flag); dfree(pos); dfree(list); dfree(tmp); dfree(out);
            return rc;
        }
        k_hem_init<<<g, 256, 0, s>>>(n, nia, agg, work_n);
        count_launch();
        int *cand = nullptr;
        if (path <= 2 && dalloc(&cand, std::max(1, gnnz)) == SUCCESS) {
            static bool attr2 = false;
            if (!attr2) {
                cudaFuncSetAttribute(k_hem_pass1_staged<true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)HEM_STAGED_SMEM);
                cudaFuncSetAttribute(k_hem_pass1_staged<false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)HEM_STAGED_SMEM);
                attr2 = true;
            }
            k_hem_rank<<<std::min(div_up(n, 8), 148 * 64), 256, 0, s>>>(n, nia, nja, nval, cand);
            if (path == 1)
                k_hem_pass1_staged<true><<<1, 64, HEM_STAGED_SMEM, s>>>(n, bw, nia, cand, agg,
                                                                        work_n, out);
            else
                k_hem_pass1_staged<false><<<1, 64, HEM_STAGED_SMEM, s>>>(n, bw, nia, cand, agg,
                                                                         work_n, out);
            count_launch(2);
            dfree(cand);
        } else {
            k_hem_pass1_ring<<<1, 32, HEM_RING_WORDS * 4, s>>>(n, bw, nia, nja, nval, agg,
                                                              work_n, out);
            count_launch();
        }
        k_flag_eq<<<g, 256, 0, s>>>(n, agg, -1, flag);
        count_launch();
        rc = scan_exclusive(flag, pos, n, tmp, s);
        int m = 0;
        if (!rc) {
            k_compact<<<g, 256, 0, s>>>(n, flag, pos, list);
            count_launch();
            cudaMemcpyAsync(&m, pos + n, sizeof(int), cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            if (m > 0) {
                k_hem_pass2_list<<<1, 32, 0, s>>>(m, list, nia, nja, agg, work_n, out);
                count_launch();
            }
            k_hem_final<<<g, 256, 0, s>>>(n, agg);
            count_launch();
        }
        dfree(flag); dfree(pos); dfree(list); dfree(tmp);
    } else {   // wide graph: the whole state in global memory
        k_hem_seq<<<1, 32, 0, s>>>(n, nia, nja, nval, agg, work_n, out);
        count_launch();
    }
    int h[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(h, out, 2 * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dfree(out);
    if (rc) return rc;
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
    *nagg = h[0];
    return h[1] < 0 ? ERROR_AMG_COARSEING : SUCCESS;
}

// ---------------------------------------------------------------------------
// deterministic parallel matching (fast mode)
//   PM_LEAD rounds of mutual choice: every free vertex points at its heaviest
//   free neighbour and mutual pairs match -- the edges that dominate both
//   their ends, which the reference's greedy walk takes too; then red/blue
//   handshake rounds until no pair forms.  Pairs are numbered through a scan.
//   Leftovers join the adjacent aggregate with the fewest members counted
//   before the leftover pass (first such neighbour on ties).  Mutual choice
//   alone stalls on chains of ever heavier edges (smooth coefficient fields);
//   the handshake alone pairs a vertex only with a neighbour of the other
//   colour, which on the 128^3 log-normal problem (sigma 1) left coarser
//   levels and 43 instead of the reference's 38 iterations; a few mutual
//   rounds first gave 39.
// ---------------------------------------------------------------------------
__global__ void k_pm_init(int n, const int *__restrict__ ia, int *state) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += gridDim.x * blockDim.x)
        state[k] = (ia[k + 1] - ia[k] > 1) ? -1 : -2;   // -1 free, -2 isolated
}

__device__ __forceinline__ unsigned hash_u32(unsigned x) {
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}

__device__ __forceinline__ unsigned edge_hash(int i, int j) {
    unsigned lo = (unsigned)min(i, j), hi = (unsigned)max(i, j);
    unsigned x = lo * 0x9e3779b1u ^ (hi + 0x7f4a7c15u + (lo << 6) + (lo >> 2));
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}

// Red/blue handshake (one round): a hashed coin splits the free vertices;
// every free red vertex proposes to its heaviest free blue neighbour (edge
// key: |a_ij| in FP32, then a hash of the unordered pair), every blue vertex
// accepts its heaviest proposer.  Accepted pairs are disjoint, and a constant
// fraction of the free vertices pairs up per round whatever the weights look
// like (heaviest-neighbour pointers alone form long chains on smooth
// coefficient fields).
__device__ __forceinline__ bool pm_red(int k, int round) {
    return (hash_u32((unsigned)k * 2654435761u + (unsigned)round * 0x632be5abu) >> 7) & 1u;
}

__device__ __forceinline__ bool pm_better(float w, unsigned h, int j, float bw,
                                          unsigned bh, int best) {
    return best < 0 || w > bw || (w == bw && (h > bh || (h == bh && j > best)));
}

constexpr int PM_LEAD = 4;

// red k proposes to its heaviest free blue neighbour; in a mutual round
// (round < PM_LEAD) every free k points at its heaviest free neighbour
__global__ void k_pm_propose(int n, int round, const int *__restrict__ ia,
                             const int *__restrict__ ja, const double *__restrict__ a,
                             const int *__restrict__ state, int *ptr) {
    const bool mutual = round < PM_LEAD;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += gridDim.x * blockDim.x) {
        int best = -1;
        if (state[k] == -1 && (mutual || pm_red(k, round))) {
            float bw = -1.0f;
            unsigned bh = 0u;
            for (int p = ia[k]; p < ia[k + 1]; ++p) {
                const int j = ja[p];
                if (j == k || state[j] != -1 || (!mutual && pm_red(j, round))) continue;
                const float w = (float)fabs(a[p]);
                const unsigned h = edge_hash(k, j);
                if (pm_better(w, h, j, bw, bh, best)) { best = j; bw = w; bh = h; }
            }
        }
        ptr[k] = best;
    }
}

// blue j: acc[j] = heaviest red neighbour proposing to j (or -1); flag marks
// accepted pairs, numbered by their blue end
__global__ void k_pm_accept(int n, int round, const int *__restrict__ ia,
                            const int *__restrict__ ja, const double *__restrict__ a,
                            const int *__restrict__ state, const int *__restrict__ ptr,
                            int *acc, int *flag, int *any) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += gridDim.x * blockDim.x) {
        int best = -1;
        if (state[j] == -1 && !pm_red(j, round)) {
            float bw = -1.0f;
            unsigned bh = 0u;
            for (int p = ia[j]; p < ia[j + 1]; ++p) {
                const int i = ja[p];
                if (i == j || ptr[i] != j) continue;
                const float w = (float)fabs(a[p]);
                const unsigned h = edge_hash(i, j);
                if (pm_better(w, h, i, bw, bh, best)) { best = i; bw = w; bh = h; }
            }
        }
        acc[j] = best;
        flag[j] = best >= 0;
        if (best >= 0) *any = 1;
    }
}

// mutual round: j pairs with i = ptr[j] when ptr[i] = j, numbered by the
// higher end
__global__ void k_pm_mutual(int n, const int *__restrict__ state, const int *__restrict__ ptr,
                            int *acc, int *flag, int *any) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        int i = -1;
        if (state[j] == -1) {
            const int p = ptr[j];
            if (p >= 0 && p < j && ptr[p] == j) i = p;
        }
        acc[j] = i;
        flag[j] = i >= 0;
        if (i >= 0) *any = 1;
    }
}

__global__ void k_pm_assign(int n, const int *__restrict__ acc,
                            const int *__restrict__ flag,
                            const int *__restrict__ pos, const int *__restrict__ base,
                            int *state) {
    const int b = *base;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += gridDim.x * blockDim.x)
        if (flag[j]) {
            const int c = b + pos[j];
            state[j] = c;
            state[acc[j]] = c;
        }
}
// the aggregate count after a round: base += the round's pairs
__global__ void k_pm_advance(int *base, const int *__restrict__ cnt) { *base += *cnt; }

// Renumbering by leader: aggregate ids follow their smallest member vertex,
// so coarse rows keep the fine ordering's locality (ids were handed out round
// by round).
__global__ void k_pm_lead(int n, const int *__restrict__ agg, int *lead) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += gridDim.x * blockDim.x)
        if (agg[v] >= 0) atomicMin(lead + agg[v], v);
}
__global__ void k_pm_leadflag(int n, const int *__restrict__ agg, const int *__restrict__ lead,
                              int *flag) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += gridDim.x * blockDim.x)
        flag[v] = agg[v] >= 0 && lead[agg[v]] == v;
}
__global__ void k_pm_renumber(int n, const int *__restrict__ lead, const int *__restrict__ pos,
                              int *agg) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += gridDim.x * blockDim.x)
        if (agg[v] >= 0) agg[v] = pos[lead[agg[v]]];
}

__global__ void k_pm_sizes(int n, const int *__restrict__ state, int *size) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += gridDim.x * blockDim.x)
        if (state[k] >= 0) atomicAdd(size + state[k], 1);
}

// Leftover free vertices join the adjacent aggregate with the fewest members
// (sizes counted before this pass; the first such neighbour on ties).  A
// free vertex without an aggregated neighbour becomes its own aggregate:
// flag[k] = 1, numbered after the pairs through a scan.
__global__ void k_pm_leftover(int n, const int *__restrict__ ia,
                              const int *__restrict__ ja,
                              const int *__restrict__ state,
                              const int *__restrict__ size, int *out, int *flag) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += gridDim.x * blockDim.x) {
        int st = state[k], f = 0;
        if (st == -1) {
            int bc = -1, bs = 0;
            for (int p = ia[k]; p < ia[k + 1]; ++p) {
                const int c = state[ja[p]];
                if (c >= 0 && (bc < 0 || size[c] < bs)) { bc = c; bs = size[c]; }
            }
            st = bc;
            f = bc < 0;
        }
        out[k] = st < 0 ? UNPT : st;
        flag[k] = f;
    }
}

__global__ void k_pm_singletons(int n, const int *__restrict__ flag,
                                const int *__restrict__ pos, int base, int *out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += gridDim.x * blockDim.x)
        if (flag[k]) out[k] = base + pos[k];
}

int hem_parallel(int n, const int *nia, const int *nja, const double *nval,
                 int *agg, int *nagg, int *work, cudaStream_t s) {
    // work layout (ints): state n | ptr n | flag n | pos n+1 | size n | scan tmp
    int *state = work, *ptr = work + n, *flag = work + 2 * n, *pos = work + 3 * n;
    int *size = work + 4 * n + 1, *tmp = work + 5 * n + 1;
    int *dflag = nullptr;
    HZB_TRY(dalloc(&dflag, 2));
    const int g = grid_for(n);
    k_pm_init<<<g, 256, 0, s>>>(n, nia, state);
    count_launch();
    cudaMemsetAsync(dflag + 1, 0, sizeof(int), s);   // the aggregate count
    int nc = 0;
    int *acc = size;   // free during the rounds
    for (int round = 0, idle = 0; round < 96 + PM_LEAD && idle < 4; ++round) {
        cudaMemsetAsync(dflag, 0, sizeof(int), s);
        k_pm_propose<<<g, 256, 0, s>>>(n, round, nia, nja, nval, state, ptr);
        if (round < PM_LEAD)
            k_pm_mutual<<<g, 256, 0, s>>>(n, state, ptr, acc, flag, dflag);
        else
            k_pm_accept<<<g, 256, 0, s>>>(n, round, nia, nja, nval, state, ptr, acc, flag,
                                          dflag);
        count_launch(2);
        int rc = scan_exclusive(flag, pos, n, tmp, s);
        if (rc) { dfree(dflag); return rc; }
        k_pm_assign<<<g, 256, 0, s>>>(n, acc, flag, pos, dflag + 1, state);
        k_pm_advance<<<1, 1, 0, s>>>(dflag + 1, pos + n);
        count_launch(2);
        int h[2];
        cudaMemcpyAsync(h, dflag, sizeof(h), cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { dfree(dflag); set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
        nc = h[1];
        // stop after a few handshake rounds in a row without a new pair
        idle = h[0] || round < PM_LEAD ? 0 : idle + 1;
    }
    cudaMemsetAsync(size, 0, sizeof(int) * (nc > 0 ? nc : 1), s);
    k_pm_sizes<<<g, 256, 0, s>>>(n, state, size);
    k_pm_leftover<<<g, 256, 0, s>>>(n, nia, nja, state, size, agg, flag);
    count_launch(2);
    int rc = scan_exclusive(flag, pos, n, tmp, s);
    int extra = 0;
    if (!rc) {
        k_pm_singletons<<<g, 256, 0, s>>>(n, flag, pos, nc, agg);
        count_launch();
        cudaMemcpyAsync(&extra, pos + n, sizeof(int), cudaMemcpyDeviceToHost, s);
    }
    if (!rc) {   // ids in the order of each aggregate's smallest vertex
        int *lead = size;
        cudaMemsetAsync(lead, 0x7f, sizeof(int) * (size_t)n, s);
        k_pm_lead<<<g, 256, 0, s>>>(n, agg, lead);
        k_pm_leadflag<<<g, 256, 0, s>>>(n, agg, lead, flag);
        count_launch(2);
        rc = scan_exclusive(flag, pos, n, tmp, s);
        if (!rc) {
            k_pm_renumber<<<g, 256, 0, s>>>(n, lead, pos, agg);
            count_launch();
        }
    }
    cudaError_t e = cudaStreamSynchronize(s);
    dfree(dflag);
    if (rc) return rc;
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
    *nagg = nc + extra;
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// Caller-supplied Galerkin inputs, checked before any kernel indexes by them
// (read-only): aggregate ids in [-1, nc), row pointers non-decreasing from 0
// to nnz, column indices in [0, n).  Bits of *bad: 1 aggregate id, 2 row
// pointers, 4 column index.
// ---------------------------------------------------------------------------
__global__ void k_check_rap_inputs(int n, int nnz, const int *__restrict__ ia,
                                   const int *__restrict__ ja, int nc,
                                   const int *__restrict__ agg, int *bad) {
    int b = 0;
    const int m = n > nnz ? n : nnz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += gridDim.x * blockDim.x) {
        if (i < n) {
            const int c = agg[i];
            if (c < -1 || c >= nc) b |= 1;
            if (ia[i + 1] < ia[i]) b |= 2;
        }
        if (i < nnz) {
            const int j = ja[i];
            if (j < 0 || j >= n) b |= 4;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (ia[0] != 0 || ia[n] != nnz)) b |= 2;
    if (b) atomicOr(bad, b);
}

int check_rap_inputs(int n, int nnz, const int *ia, const int *ja, int nc, const int *agg,
                     int *d_bad, cudaStream_t s) {
    HZB_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
    k_check_rap_inputs<<<grid_for(n > nnz ? n : nnz), 256, 0, s>>>(n, nnz, ia, ja, nc, agg,
                                                                    d_bad);
    count_launch();
    int bad = 0;
    HZB_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    if (bad & 1) {
        set_error_msg("Galerkin product: an aggregate id lies outside [-1, nc)");
        return ERROR_INPUT_PAR;
    }
    if (bad & 2) {
        set_error_msg("Galerkin product: row pointers do not rise from 0 to nnz");
        return ERROR_INPUT_PAR;
    }
    if (bad & 4) {
        set_error_msg("Galerkin product: a column index lies outside [0, n)");
        return ERROR_INPUT_PAR;
    }
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// R = P^T pattern with ascending fine indices per row
// ---------------------------------------------------------------------------
__global__ void k_agg_count(int n, const int *__restrict__ agg, int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        if (agg[i] >= 0) atomicAdd(cnt + agg[i], 1);
}
__global__ void k_agg_fill(int n, const int *__restrict__ agg,
                           const int *__restrict__ ria, int *fillc, int *rja) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const int c = agg[i];
        if (c >= 0) rja[ria[c] + atomicAdd(fillc + c, 1)] = i;
    }
}
__global__ void k_sort_rows(int nr, const int *__restrict__ ia, int *ja) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nr;
         r += gridDim.x * blockDim.x) {
        const int b0 = ia[r], b1 = ia[r + 1];
        for (int p = b0 + 1; p < b1; ++p) {      // insertion sort (short rows)
            int v = ja[p], q = p - 1;
            while (q >= b0 && ja[q] > v) { ja[q + 1] = ja[q]; --q; }
            ja[q + 1] = v;
        }
    }
}

int restriction_pattern(int n, int nc, const int *agg, int *ria, int *rja,
                        int *tmp, cudaStream_t s) {
    int *cnt = nullptr;
    HZB_TRY(dalloc(&cnt, nc));
    HZB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (nc > 0 ? nc : 1), s));
    k_agg_count<<<grid_for(n), 256, 0, s>>>(n, agg, cnt);
    count_launch();
    int rc = scan_exclusive(cnt, ria, nc, tmp, s);
    if (!rc) {
        cudaMemsetAsync(cnt, 0, sizeof(int) * (nc > 0 ? nc : 1), s);
        k_agg_fill<<<grid_for(n), 256, 0, s>>>(n, agg, ria, cnt, rja);
        k_sort_rows<<<grid_for(nc), 256, 0, s>>>(nc, ria, rja);
        count_launch(2);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; }
    }
    dfree(cnt);
    return rc;
}

// ---------------------------------------------------------------------------
// Galerkin product A_c = R A P for unit aggregation P (exact order)
// ---------------------------------------------------------------------------
__global__ void k_rap_bound(int nc, const int *__restrict__ ria,
                            const int *__restrict__ rja, const int *__restrict__ ia,
                            int *ub) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc;
         c += gridDim.x * blockDim.x) {
        int u = 1;
        for (int q = ria[c]; q < ria[c + 1]; ++q) {
            const int i = rja[q];
            u += ia[i + 1] - ia[i];
        }
        ub[c] = u;
    }
}

// One thread per coarse row builds its slot list in scratch: slot 0 is the
// diagonal (0.0, accumulated); other columns in first-encounter order; a new
// column takes the entry's value, a known column adds it.
__global__ void k_rap_build(int nc, const int *__restrict__ ria,
                            const int *__restrict__ rja, const int *__restrict__ ia,
                            const int *__restrict__ ja, const double *__restrict__ a,
                            const int *__restrict__ agg, const int *__restrict__ off,
                            int *scol, double *sval, int *rowcnt) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc;
         c += gridDim.x * blockDim.x) {
        int *cols = scol + off[c];
        double *vals = sval + off[c];
        int cnt = 1;
        cols[0] = c;
        vals[0] = 0.0;
        for (int q = ria[c]; q < ria[c + 1]; ++q) {
            const int i = rja[q];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                const int cc = agg[ja[k]];
                if (cc < 0) continue;
                int pos = -1;
                for (int t = 0; t < cnt; ++t)
                    if (cols[t] == cc) { pos = t; break; }
                if (pos >= 0) {
                    vals[pos] += a[k];
                } else {
                    cols[cnt] = cc;
                    vals[cnt] = a[k];
                    ++cnt;
                }
            }
        }
        rowcnt[c] = cnt;
    }
}

// The same slot lists with a warp per coarse row, for rows whose bound ub
// (1 + the fine rows' lengths) is at most 64: slot t lives in lane t % 32,
// register t / 32.  The warp loads 32 entries of a fine row at a time (their
// coarse columns in parallel), then takes the products one by one in CSR
// order: a ballot finds the slot holding the column, whose lane adds the
// value, or the next free slot takes it.  Every slot receives its values in
// the same order as above, so the sums are the same bit for bit.  Rows with
// a larger bound are left to k_rap_build (rowcnt untouched here).
__global__ void __launch_bounds__(256)
k_rap_build_warp(int nc, const int *__restrict__ ria, const int *__restrict__ rja,
                 const int *__restrict__ ia, const int *__restrict__ ja,
                 const double *__restrict__ a, const int *__restrict__ agg,
                 const int *__restrict__ off, const int *__restrict__ ub, int *scol,
                 double *sval, int *rowcnt, int *nbig) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nc; c += warps) {
        if (ub[c] > 64) {
            if (lane == 0) atomicAdd(nbig, 1);
            continue;
        }
        int col0 = lane == 0 ? c : -1, col1 = -1;
        double val0 = 0.0, val1 = 0.0;
        int cnt = 1;
        for (int q = ria[c]; q < ria[c + 1]; ++q) {
            const int i = rja[q];
            const int k0 = ia[i], k1 = ia[i + 1];
            for (int kb = k0; kb < k1; kb += 32) {
                const int k = kb + lane;
                int cc_l = -1;
                double v_l = 0.0;
                if (k < k1) {
                    cc_l = agg[ja[k]];
                    v_l = a[k];
                }
                const int m = min(32, k1 - kb);
                for (int j = 0; j < m; ++j) {
                    const int cc = __shfl_sync(FULL, cc_l, j);
                    const double v = __shfl_sync(FULL, v_l, j);
                    if (cc < 0) continue;
                    const unsigned h0 = __ballot_sync(FULL, col0 == cc);
                    const unsigned h1 = __ballot_sync(FULL, col1 == cc);
                    if (h0) {
                        if (lane == __ffs(h0) - 1) val0 += v;
                    } else if (h1) {
                        if (lane == __ffs(h1) - 1) val1 += v;
                    } else {
                        if (lane == (cnt & 31)) {
                            if (cnt < 32) { col0 = cc; val0 = v; }
                            else { col1 = cc; val1 = v; }
                        }
                        ++cnt;
                    }
                }
            }
        }
        int *cols = scol + off[c];
        double *vals = sval + off[c];
        if (lane < cnt) { cols[lane] = col0; vals[lane] = val0; }
        if (lane + 32 < cnt) { cols[lane + 32] = col1; vals[lane + 32] = val1; }
        if (lane == 0) rowcnt[c] = cnt;
    }
}

// k_rap_build for the rows k_rap_build_warp left (bound above 64)
__global__ void k_rap_build_big(int nc, const int *__restrict__ ria,
                                const int *__restrict__ rja, const int *__restrict__ ia,
                                const int *__restrict__ ja, const double *__restrict__ a,
                                const int *__restrict__ agg, const int *__restrict__ off,
                                const int *__restrict__ ub, int *scol, double *sval,
                                int *rowcnt) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc;
         c += gridDim.x * blockDim.x) {
        if (ub[c] <= 64) continue;
        int *cols = scol + off[c];
        double *vals = sval + off[c];
        int cnt = 1;
        cols[0] = c;
        vals[0] = 0.0;
        for (int q = ria[c]; q < ria[c + 1]; ++q) {
            const int i = rja[q];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                const int cc = agg[ja[k]];
                if (cc < 0) continue;
                int pos = -1;
                for (int t = 0; t < cnt; ++t)
                    if (cols[t] == cc) { pos = t; break; }
                if (pos >= 0) {
                    vals[pos] += a[k];
                } else {
                    cols[cnt] = cc;
                    vals[cnt] = a[k];
                    ++cnt;
                }
            }
        }
        rowcnt[c] = cnt;
    }
}

__global__ void k_rap_compact(int nc, const int *__restrict__ off,
                              const int *__restrict__ cia,
                              const int *__restrict__ scol,
                              const double *__restrict__ sval, int *cja,
                              double *cval) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc;
         c += gridDim.x * blockDim.x) {
        const int src = off[c], dst = cia[c], m = cia[c + 1] - cia[c];
        for (int t = 0; t < m; ++t) {
            cja[dst + t] = scol[src + t];
            cval[dst + t] = sval[src + t];
        }
    }
}

int rap_agg(const DCsr<double> &A, int nc, const int *agg, const int *ria,
            const int *rja, int **cia_out, int **cja_out, double **cval_out,
            int *cnnz, cudaStream_t s) {
    *cia_out = nullptr; *cja_out = nullptr; *cval_out = nullptr;
    int *ub = nullptr, *off = nullptr, *tmp = nullptr, *rowcnt = nullptr;
    int *scol = nullptr, *cia = nullptr, *cja = nullptr;
    double *sval = nullptr, *cval = nullptr;
    int rc = SUCCESS, total = 0;
    const int g = grid_for(nc);
    cudaError_t e;
    if ((rc = dalloc(&ub, nc))) goto fail;
    if ((rc = dalloc(&off, nc + 1))) goto fail;
    if ((rc = dalloc(&tmp, scan_tmp_size(nc + 1)))) goto fail;
    if ((rc = dalloc(&rowcnt, nc))) goto fail;
    if ((rc = dalloc(&cia, nc + 1))) goto fail;
    k_rap_bound<<<g, 256, 0, s>>>(nc, ria, rja, A.ia, ub);
    count_launch();
    if ((rc = scan_exclusive(ub, off, nc, tmp, s))) goto fail;
    e = cudaMemcpyAsync(&total, off + nc, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto fail; }
    if ((rc = dalloc(&scol, total))) goto fail;
    if ((rc = dalloc(&sval, total))) goto fail;
    {
        // a warp per coarse row; rows with a bound above 64 slots by a thread
        int *nbig = tmp;   // the scan scratch is free until the next scan
        e = cudaMemsetAsync(nbig, 0, sizeof(int), s);
        if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto fail; }
        k_rap_build_warp<<<grid_for(32LL * nc), 256, 0, s>>>(nc, ria, rja, A.ia, A.ja, A.val,
                                                            agg, off, ub, scol, sval, rowcnt,
                                                            nbig);
        int hbig = 0;
        e = cudaMemcpyAsync(&hbig, nbig, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto fail; }
        count_launch();
        if (hbig) {
            k_rap_build_big<<<g, 128, 0, s>>>(nc, ria, rja, A.ia, A.ja, A.val, agg, off, ub,
                                              scol, sval, rowcnt);
            count_launch();
        }
    }
    if ((rc = scan_exclusive(rowcnt, cia, nc, tmp, s))) goto fail;
    e = cudaMemcpyAsync(cnnz, cia + nc, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto fail; }
    if ((rc = dalloc(&cja, *cnnz))) goto fail;
    if ((rc = dalloc(&cval, *cnnz))) goto fail;
    k_rap_compact<<<g, 256, 0, s>>>(nc, off, cia, scol, sval, cja, cval);
    count_launch();
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto fail; }
    dfree(ub); dfree(off); dfree(tmp); dfree(rowcnt); dfree(scol); dfree(sval);
    *cia_out = cia; *cja_out = cja; *cval_out = cval;
    return SUCCESS;
fail:
    dfree(ub); dfree(off); dfree(tmp); dfree(rowcnt); dfree(scol); dfree(sval);
    dfree(cia); dfree(cja); dfree(cval);
    return rc;
}

// ---------------------------------------------------------------------------
// smoother diagonals
// ---------------------------------------------------------------------------
__global__ void k_diags(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                        const double *__restrict__ a, double *djac, double *dgs,
                        double *dsor, int *gs_ok, int *sor_ok, int *missing) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        double dj = 0.0, dg = 0.0, ds = 0.0;
        int okg = 0, oks = 0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            if (ja[k] != i) continue;
            dj = a[k];
            ds = a[k];
            oks = 1;
            if (fabs(a[k]) > SMALLREAL) { dg = 1.e+0 / a[k]; okg = 1; }
        }
        djac[i] = dj;
        dgs[i] = dg;
        dsor[i] = ds;
        gs_ok[i] = okg;
        sor_ok[i] = oks;
        if (!okg || !oks) atomicAdd(missing, 1);
    }
}

// Rows without a (usable) diagonal keep the previous row's d in the
// reference's sweep; resolve that carry sequentially (rare path).
__global__ void k_diag_carry(int n, const double *__restrict__ dgs,
                             const double *__restrict__ dsor,
                             const int *__restrict__ gs_ok,
                             const int *__restrict__ sor_ok, double *gf,
                             double *gb, double *sf, double *sb) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double c1 = 0.0, c2 = 0.0;
    for (int i = 0; i < n; ++i) {
        if (gs_ok[i]) c1 = dgs[i];
        if (sor_ok[i]) c2 = dsor[i];
        gf[i] = c1;
        sf[i] = c2;
    }
    c1 = 0.0; c2 = 0.0;
    for (int i = n - 1; i >= 0; --i) {
        if (gs_ok[i]) c1 = dgs[i];
        if (sor_ok[i]) c2 = dsor[i];
        gb[i] = c1;
        sb[i] = c2;
    }
}

int smoother_diagonals(const DCsr<double> &A, double *d_jac, double *d_gs_f,
                       double *d_gs_b, double *d_sor_f, double *d_sor_b,
                       cudaStream_t s) {
    const int n = A.n;
    int *ok = nullptr;
    HZB_TRY(dalloc(&ok, 2 * (size_t)n + 1));
    int *missing = ok + 2 * (size_t)n;
    HZB_CUDA(cudaMemsetAsync(missing, 0, sizeof(int), s));
    k_diags<<<grid_for(n), 256, 0, s>>>(n, A.ia, A.ja, A.val, d_jac, d_gs_f, d_sor_f,
                                        ok, ok + n, missing);
    count_launch();
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, missing, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { dfree(ok); set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
    if (h) {
        double *tg = nullptr, *ts = nullptr;
        int rc = dalloc(&tg, n);
        if (!rc) rc = dalloc(&ts, n);
        if (rc) { dfree(tg); dfree(ok); return rc; }
        cudaMemcpyAsync(tg, d_gs_f, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(ts, d_sor_f, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        k_diag_carry<<<1, 32, 0, s>>>(n, tg, ts, ok, ok + n, d_gs_f, d_gs_b, d_sor_f,
                                      d_sor_b);
        count_launch();
        e = cudaStreamSynchronize(s);
        dfree(tg); dfree(ts);
        if (e != cudaSuccess) { dfree(ok); set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
    } else {
        cudaMemcpyAsync(d_gs_b, d_gs_f, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d_sor_b, d_sor_f, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
    }
    dfree(ok);
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// A^T with ascending column indices per row (dcsr_transz, p = NULL)
// ---------------------------------------------------------------------------
__global__ void k_tr_count(int n, const int *__restrict__ ia,
                           const int *__restrict__ ja, int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        for (int k = ia[i]; k < ia[i + 1]; ++k) atomicAdd(cnt + ja[k], 1);
}
__global__ void k_tr_fill(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                          const double *__restrict__ a, const int *__restrict__ tia,
                          int *fillc, int *tja, double *tval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            const int q = tia[ja[k]] + atomicAdd(fillc + ja[k], 1);
            tja[q] = i;
            tval[q] = a[k];
        }
}
// rows of the transpose in ascending order (stable for equal indices is not
// needed: a row index appears once per source row entry)
__global__ void k_tr_sort(int n, const int *__restrict__ tia, int *tja, double *tval) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n;
         r += gridDim.x * blockDim.x) {
        const int b0 = tia[r], b1 = tia[r + 1];
        for (int p = b0 + 1; p < b1; ++p) {
            const int v = tja[p];
            const double x = tval[p];
            int q = p - 1;
            while (q >= b0 && tja[q] > v) { tja[q + 1] = tja[q]; tval[q + 1] = tval[q]; --q; }
            tja[q + 1] = v;
            tval[q + 1] = x;
        }
    }
}

int transpose_csr(const DCsr<double> &A, int **tia_out, int **tja_out,
                  double **tval_out, cudaStream_t s) {
    const int n = A.n;
    int *tia = nullptr, *tja = nullptr, *cnt = nullptr, *tmp = nullptr;
    double *tval = nullptr;
    int rc = SUCCESS;
    const int g = grid_for(n);
    if ((rc = dalloc(&tia, n + 1)) || (rc = dalloc(&tja, A.nnz)) ||
        (rc = dalloc(&tval, A.nnz)) || (rc = dalloc(&cnt, n)) ||
        (rc = dalloc(&tmp, scan_tmp_size(n + 1)))) goto fail;
    cudaMemsetAsync(cnt, 0, sizeof(int) * n, s);
    k_tr_count<<<g, 256, 0, s>>>(n, A.ia, A.ja, cnt);
    count_launch();
    if ((rc = scan_exclusive(cnt, tia, n, tmp, s))) goto fail;
    cudaMemsetAsync(cnt, 0, sizeof(int) * n, s);
    k_tr_fill<<<g, 256, 0, s>>>(n, A.ia, A.ja, A.val, tia, cnt, tja, tval);
    k_tr_sort<<<g, 256, 0, s>>>(n, tia, tja, tval);
    count_launch(2);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        set_error(cudaGetLastError(), __FILE__, __LINE__);
        rc = ERROR_SOLVER_MISC;
        goto fail;
    }
    dfree(cnt); dfree(tmp);
    *tia_out = tia; *tja_out = tja; *tval_out = tval;
    return SUCCESS;
fail:
    dfree(tia); dfree(tja); dfree(tval); dfree(cnt); dfree(tmp);
    return rc;
}

// ---------------------------------------------------------------------------
// level schedules (Kahn rounds on the DAG lower -> higher or reverse)
// ---------------------------------------------------------------------------
void Schedule::release() {
    dfree(rows);
    dfree(set_ptr);
    dfree(bar);
    h_ptr.clear();
    run_first.clear();
    run_last.clear();
    run_max.clear();
}

__global__ void k_transpose_count(int n, const int *__restrict__ ia,
                                  const int *__restrict__ ja, int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        for (int k = ia[i]; k < ia[i + 1]; ++k) atomicAdd(cnt + ja[k], 1);
}
__global__ void k_transpose_fill(int n, const int *__restrict__ ia,
                                 const int *__restrict__ ja,
                                 const int *__restrict__ tia, int *fillc, int *tja) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            const int j = ja[k];
            tja[tia[j] + atomicAdd(fillc + j, 1)] = i;
        }
}

// dependency count: neighbours that come earlier in the sweep
__global__ void k_indeg(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                        const int *__restrict__ tia, const int *__restrict__ tja,
                        int backward, int *indeg, int *rows, int *tail) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        int c = 0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            const int j = ja[k];
            c += backward ? (j > i) : (j < i);
        }
        for (int k = tia[i]; k < tia[i + 1]; ++k) {
            const int j = tja[k];
            c += backward ? (j > i) : (j < i);
        }
        indeg[i] = c;
        atomicMax(tail + 1, c);
        if (c == 0) rows[atomicAdd(tail, 1)] = i;
    }
}

__global__ void k_kahn_round(int head, int cnt, const int *__restrict__ ia,
                             const int *__restrict__ ja, const int *__restrict__ tia,
                             const int *__restrict__ tja, int backward, int *indeg,
                             int *rows, int *tail) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt;
         q += gridDim.x * blockDim.x) {
        const int i = rows[head + q];
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            const int j = ja[k];
            if (backward ? (j < i) : (j > i))
                if (atomicSub(indeg + j, 1) == 1) rows[atomicAdd(tail, 1)] = j;
        }
        for (int k = tia[i]; k < tia[i + 1]; ++k) {
            const int j = tja[k];
            if (backward ? (j < i) : (j > i))
                if (atomicSub(indeg + j, 1) == 1) rows[atomicAdd(tail, 1)] = j;
        }
    }
}

// Every round of Kahn's algorithm in one CTA: the frontier [head, cur) of the
// queue releases the rows that depend on it; the queue end moves by a
// shared-memory atomic and the rounds are separated by __syncthreads, so a
// level of many small sets costs no launch or host round trip per set.
// Each round removes at least one row, so at most n rounds run.  ptr
// receives the set boundaries (n + 1 ints at most), *nsets their count.
constexpr int KAHN_CTA_MAX_ROWS = 1 << 20;
__global__ void __launch_bounds__(1024)
k_kahn_all(int n, const int *__restrict__ ia, const int *__restrict__ ja,
           const int *__restrict__ tia, const int *__restrict__ tja, int backward,
           int *indeg, int *rows, const int *__restrict__ tail0, int *ptr, int *nsets) {
    __shared__ int s_tail, s_head, s_cur, s_ns;
    if (threadIdx.x == 0) {
        s_head = 0;
        s_cur = *tail0;
        s_tail = s_cur;
        s_ns = 0;
        ptr[0] = 0;
    }
    __syncthreads();
    for (int round = 0; round < n; ++round) {
        const int head = s_head, cur = s_cur;
        if (cur <= head) break;
        if (threadIdx.x == 0) ptr[++s_ns] = cur;
        for (int q = head + threadIdx.x; q < cur; q += blockDim.x) {
            const int i = rows[q];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                const int j = ja[k];
                if (backward ? (j < i) : (j > i))
                    if (atomicSub(indeg + j, 1) == 1) rows[atomicAdd(&s_tail, 1)] = j;
            }
            for (int k = tia[i]; k < tia[i + 1]; ++k) {
                const int j = tja[k];
                if (backward ? (j < i) : (j > i))
                    if (atomicSub(indeg + j, 1) == 1) rows[atomicAdd(&s_tail, 1)] = j;
            }
        }
        __threadfence_block();
        __syncthreads();
        if (threadIdx.x == 0) {
            s_head = cur;
            s_cur = s_tail;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        nsets[0] = s_ns;
        nsets[1] = s_head;   // rows placed
    }
}

// The same rounds for levels of at most KAHN_SMEM_ROWS rows whose in-degrees
// fit 16 bits: the in-degree counters sit in shared memory (two to a word;
// a counter is decremented exactly as often as it counts, so a halfword
// never borrows from its neighbour), and each round's new frontier is also
// kept in shared memory (double-buffered, up to KAHN_FRONT rows) for the next
// round to read, so a round costs two dependent global loads (row bounds,
// then columns) instead of a chain through global atomics.  The column
// indices of a row are loaded eight at a time before their counters are
// decremented.  Same sets as k_kahn_all (the order of rows inside a set may
// differ; the rows of a set are independent).
constexpr int KAHN_SMEM_ROWS = 96 * 1024;
constexpr int KAHN_FRONT = 4096;
constexpr size_t kahn_smem_bytes(int n) {
    return sizeof(unsigned) * ((size_t)(n + 1) / 2) + sizeof(int) * 2 * KAHN_FRONT;
}
__global__ void __launch_bounds__(1024)
k_kahn_smem(int n, const int *__restrict__ ia, const int *__restrict__ ja,
            const int *__restrict__ tia, const int *__restrict__ tja, int backward,
            const int *__restrict__ indeg, int *rows, const int *__restrict__ tail0, int *ptr,
            int *nsets) {
    extern __shared__ unsigned kahn_sm[];
    const int nw = (n + 1) / 2;
    unsigned *deg = kahn_sm;
    int *front = reinterpret_cast<int *>(kahn_sm + nw);
    __shared__ int s_tail, s_head, s_cur, s_ns;
    for (int w = threadIdx.x; w < nw; w += blockDim.x) {
        const unsigned lo = (unsigned)indeg[2 * w];
        const unsigned hi = 2 * w + 1 < n ? (unsigned)indeg[2 * w + 1] : 0u;
        deg[w] = lo | (hi << 16);
    }
    if (threadIdx.x == 0) {
        s_head = 0;
        s_cur = *tail0;
        s_tail = s_cur;
        s_ns = 0;
        ptr[0] = 0;
    }
    __syncthreads();
    for (int round = 0; round < n; ++round) {
        const int head = s_head, cur = s_cur;
        if (cur <= head) break;
        if (threadIdx.x == 0) ptr[++s_ns] = cur;
        const bool fin_ok = round > 0 && cur - head <= KAHN_FRONT;
        const int *fin = front + (round & 1) * KAHN_FRONT;
        int *fout = front + ((round + 1) & 1) * KAHN_FRONT;
        auto release = [&](int j) {
            const unsigned sh = 16u * (unsigned)(j & 1);
            const unsigned old = atomicSub(deg + (j >> 1), 1u << sh);
            if (((old >> sh) & 0xFFFFu) == 1u) {
                const int p = atomicAdd(&s_tail, 1);
                rows[p] = j;
                if (p - cur < KAHN_FRONT) fout[p - cur] = j;
            }
        };
        auto visit = [&](int i, const int *__restrict__ xa, const int *__restrict__ xj) {
            const int k1 = xa[i + 1];
            for (int k0 = xa[i]; k0 < k1; k0 += 8) {
                int c[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) c[u] = k0 + u < k1 ? xj[k0 + u] : -1;
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (c[u] >= 0 && (backward ? (c[u] < i) : (c[u] > i))) release(c[u]);
            }
        };
        for (int q = head + threadIdx.x; q < cur; q += blockDim.x) {
            const int i = fin_ok ? fin[q - head] : rows[q];
            visit(i, ia, ja);
            visit(i, tia, tja);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_head = cur;
            s_cur = s_tail;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        nsets[0] = s_ns;
        nsets[1] = s_head;   // rows placed
    }
}

static void make_runs(Schedule *sch) {
    const int ns = (int)sch->h_ptr.size() - 1;
    int k = 0;
    while (k < ns) {
        int k2 = k;
        int mx = 0;
        while (k2 < ns && k2 - k < GS_RUN_SETS &&
               sch->h_ptr[k2 + 1] - sch->h_ptr[k2] <= GS_SMALL_SET) {
            mx = std::max(mx, sch->h_ptr[k2 + 1] - sch->h_ptr[k2]);
            ++k2;
        }
        if (k2 > k) {   // run of small sets
            sch->run_first.push_back(k);
            sch->run_last.push_back(k2);
            sch->run_max.push_back(mx);
            k = k2;
        } else {        // one large set: a grid-wide launch (marked by -1)
            sch->run_first.push_back(k);
            sch->run_last.push_back(-1);
            sch->run_max.push_back(sch->h_ptr[k + 1] - sch->h_ptr[k]);
            ++k;
        }
    }
}

int gs_schedule(int n, const int *ia, const int *ja, int nnz, int backward,
                Schedule *sch, cudaStream_t s) {
    sch->release();
    int *tia = nullptr, *tja = nullptr, *fillc = nullptr, *indeg = nullptr;
    int *tail = nullptr, *tmp = nullptr;
    int rc = SUCCESS;
    std::vector<int> ptr;
    cudaError_t e;
    const int g = grid_for(n);
    if ((rc = dalloc(&tia, n + 1))) goto done;
    if ((rc = dalloc(&tja, nnz))) goto done;
    if ((rc = dalloc(&fillc, n))) goto done;
    if ((rc = dalloc(&indeg, n))) goto done;
    if ((rc = dalloc(&tail, 2))) goto done;   // frontier end, largest in-degree
    if ((rc = dalloc(&tmp, scan_tmp_size(n + 1)))) goto done;
    if ((rc = dalloc(&sch->rows, n))) goto done;
    cudaMemsetAsync(fillc, 0, sizeof(int) * n, s);
    cudaMemsetAsync(tail, 0, 2 * sizeof(int), s);
    k_transpose_count<<<g, 256, 0, s>>>(n, ia, ja, fillc);
    count_launch();
    if ((rc = scan_exclusive(fillc, tia, n, tmp, s))) goto done;
    cudaMemsetAsync(fillc, 0, sizeof(int) * n, s);
    k_transpose_fill<<<g, 256, 0, s>>>(n, ia, ja, tia, fillc, tja);
    k_indeg<<<g, 256, 0, s>>>(n, ia, ja, tia, tja, backward, indeg, sch->rows, tail);
    count_launch(2);
    if (n <= KAHN_CTA_MAX_ROWS) {
        // one CTA runs every round; set boundaries and counts come back once
        int *dptr = nullptr, *dns = nullptr;
        if ((rc = dalloc(&dptr, n + 1)) || (rc = dalloc(&dns, 2))) {
            dfree(dptr);
            goto done;
        }
        int maxdeg = 0;
        e = cudaMemcpyAsync(&maxdeg, tail + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            dfree(dptr);
            dfree(dns);
            set_error(e, __FILE__, __LINE__);
            rc = ERROR_SOLVER_MISC;
            goto done;
        }
        if (n <= KAHN_SMEM_ROWS && maxdeg <= 0xFFFF) {
            static bool attr = false;
            if (!attr) {
                cudaFuncSetAttribute(k_kahn_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kahn_smem_bytes(KAHN_SMEM_ROWS));
                attr = true;
            }
            k_kahn_smem<<<1, 1024, kahn_smem_bytes(n), s>>>(n, ia, ja, tia, tja, backward,
                                                            indeg, sch->rows, tail, dptr, dns);
        } else {
            k_kahn_all<<<1, 1024, 0, s>>>(n, ia, ja, tia, tja, backward, indeg, sch->rows,
                                          tail, dptr, dns);
        }
        count_launch();
        int hns[2] = {0, 0};
        e = cudaMemcpyAsync(hns, dns, sizeof(hns), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && hns[1] == n) {
            ptr.resize(hns[0] + 1);
            e = cudaMemcpyAsync(ptr.data(), dptr, sizeof(int) * (hns[0] + 1),
                                cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        }
        dfree(dptr);
        dfree(dns);
        if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
        if (hns[1] != n) {
            set_error_msg("gs_schedule: incomplete level schedule");
            rc = ERROR_DATA_STRUCTURE;
            goto done;
        }
    } else {
        int head = 0, cur = 0;
        e = cudaMemcpyAsync(&cur, tail, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
        ptr.push_back(0);
        while (cur > head) {
            ptr.push_back(cur);
            const int cnt = cur - head;
            k_kahn_round<<<grid_for(cnt), 256, 0, s>>>(head, cnt, ia, ja, tia, tja,
                                                       backward, indeg, sch->rows, tail);
            count_launch();
            head = cur;
            e = cudaMemcpyAsync(&cur, tail, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
        }
        if (head != n) {   // a cycle cannot occur in index order; guard anyway
            set_error_msg("gs_schedule: incomplete level schedule");
            rc = ERROR_DATA_STRUCTURE;
            goto done;
        }
    }
    sch->h_ptr = ptr;
    if ((rc = dalloc(&sch->bar, 2))) goto done;
    if (cudaMemsetAsync(sch->bar, 0, 2 * sizeof(unsigned), s) != cudaSuccess) {
        rc = ERROR_SOLVER_MISC;
        goto done;
    }
    if ((rc = dalloc(&sch->set_ptr, ptr.size()))) goto done;
    e = cudaMemcpyAsync(sch->set_ptr, ptr.data(), sizeof(int) * ptr.size(),
                        cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
    make_runs(sch);
done:
    dfree(tia); dfree(tja); dfree(fillc); dfree(indeg); dfree(tail); dfree(tmp);
    if (rc) sch->release();
    return rc;
}

// ---------------------------------------------------------------------------
// multicolouring (Jones-Plassmann, hashed priorities, smallest free colour)
// ---------------------------------------------------------------------------

__global__ void k_jp_round(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                           const int *__restrict__ col_in, int *col_out, int *left) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        int c = col_in[i];
        if (c >= 0) { col_out[i] = c; continue; }
        const unsigned pi = hash_u32((unsigned)i);
        bool top = true;
        unsigned long long used = 0ull;   // colours 0..63 taken by neighbours
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            const int j = ja[k];
            if (j == i) continue;
            const int cj = col_in[j];
            if (cj >= 0) {
                if (cj < 64) used |= 1ull << cj;
            } else {
                const unsigned pj = hash_u32((unsigned)j);
                if (pj > pi || (pj == pi && j > i)) { top = false; }
            }
        }
        if (top) {
            int cc = 0;
            while (cc < 64 && (used >> cc & 1ull)) ++cc;
            col_out[i] = cc;
        } else {
            col_out[i] = -1;
            atomicAdd(left, 1);
        }
    }
}

__global__ void k_color_count(int n, const int *__restrict__ col, int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        atomicAdd(cnt + col[i], 1);
}
__global__ void k_color_fill(int n, const int *__restrict__ col,
                             const int *__restrict__ ptr, int *fillc, int *rows) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        rows[ptr[col[i]] + atomicAdd(fillc + col[i], 1)] = i;
}

int multicolor(int n, const int *ia, const int *ja, Schedule *sch, cudaStream_t s) {
    sch->release();
    int *c0 = nullptr, *c1 = nullptr, *left = nullptr, *cnt = nullptr, *ptr = nullptr;
    int *tmp = nullptr;
    int rc = SUCCESS, ncol = 0;
    cudaError_t e;
    const int g = grid_for(n);
    std::vector<int> hp;
    if ((rc = dalloc(&c0, n))) goto done;
    if ((rc = dalloc(&c1, n))) goto done;
    if ((rc = dalloc(&left, 1))) goto done;
    if ((rc = dalloc(&cnt, 65))) goto done;
    if ((rc = dalloc(&ptr, 66))) goto done;
    if ((rc = dalloc(&tmp, scan_tmp_size(66)))) goto done;
    if ((rc = dalloc(&sch->rows, n))) goto done;
    cudaMemsetAsync(c0, 0xff, sizeof(int) * n, s);
    for (int round = 0; round < 4096; ++round) {
        int hl = 0;
        cudaMemsetAsync(left, 0, sizeof(int), s);
        k_jp_round<<<g, 256, 0, s>>>(n, ia, ja, c0, c1, left);
        count_launch();
        std::swap(c0, c1);
        e = cudaMemcpyAsync(&hl, left, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
        if (!hl) break;
    }
    cudaMemsetAsync(cnt, 0, sizeof(int) * 65, s);
    k_color_count<<<g, 256, 0, s>>>(n, c0, cnt);
    count_launch();
    if ((rc = scan_exclusive(cnt, ptr, 65, tmp, s))) goto done;
    hp.resize(66);
    e = cudaMemcpyAsync(hp.data(), ptr, sizeof(int) * 66, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
    if (hp[65] != n) { set_error_msg("multicolor: more than 64 colours"); rc = ERROR_DATA_STRUCTURE; goto done; }
    cudaMemsetAsync(cnt, 0, sizeof(int) * 65, s);
    k_color_fill<<<g, 256, 0, s>>>(n, c0, ptr, cnt, sch->rows);
    count_launch();
    ncol = 0;
    while (ncol < 65 && hp[ncol + 1] > hp[ncol]) ++ncol;
    sch->h_ptr.assign(hp.begin(), hp.begin() + ncol + 1);
    if ((rc = dalloc(&sch->set_ptr, ncol + 1))) goto done;
    e = cudaMemcpyAsync(sch->set_ptr, sch->h_ptr.data(), sizeof(int) * (ncol + 1),
                        cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); rc = ERROR_SOLVER_MISC; goto done; }
    make_runs(sch);
done:
    dfree(c0); dfree(c1); dfree(left); dfree(cnt); dfree(ptr); dfree(tmp);
    if (rc) sch->release();
    return rc;
}

// ---------------------------------------------------------------------------
// Galerkin product without device allocation.
//
// Some callers cannot call cudaMalloc: processes whose device memory is
// reserved up front by their own allocator (a framework's caching pool, an
// embedded solver with a fixed memory budget), and library code that must
// not trigger the implicit device synchronisation that cudaMalloc and
// cudaFree bring.  For them the product's scratch (restriction pattern,
// per-row bounds, slot lists, scan partials, an error flag) lives in one
// file-scope device array of fixed size, held by every device that loads
// this library until the process exits.  Its size bounds the problem:
// n <= HZB_NOALLOC_MAX_ROWS fine rows and nnz <= HZB_NOALLOC_MAX_NNZ stored
// entries.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t NA_ROWS = HZB_NOALLOC_MAX_ROWS;
constexpr size_t NA_NNZ = HZB_NOALLOC_MAX_NNZ;
constexpr size_t NA_TMP = (NA_ROWS + 1 + 2047) / 2048 + 8;
constexpr size_t NA_SLOTS = NA_NNZ + NA_ROWS;   // slot lists: nc + sum of row lengths
// int words: cnt, ria, rja, ub, off, rowcnt, scan tmp, error flag (padded), scol
constexpr size_t NA_INTS = 6 * (NA_ROWS + 1) + NA_TMP + 4 + NA_SLOTS;
constexpr size_t NA_INT_WORDS = (NA_INTS + 1) / 2;   // in 8-byte words
constexpr size_t NA_WORDS = NA_INT_WORDS + NA_SLOTS;   // + sval
}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[NA_WORDS];

// Device address of g_noalloc_scratch for each device, resolved once with
// that device current (in host code the symbol is only a host stand-in).
static void *g_noalloc_addr[64];
static std::mutex g_noalloc_mu;

static int noalloc_scratch(double **p) {
    int dev = 0;
    HZB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { set_error_msg("device ordinal out of range"); return ERROR_MISC; }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *a = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
        if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
        g_noalloc_addr[dev] = a;
    }
    *p = (double *)g_noalloc_addr[dev];
    return SUCCESS;
}

}  // namespace hzb

// The same kernels, in the same order, as hzb_rap_agg_device, so the result
// is identical bit for bit; only the scratch comes from the static array and
// the outputs from the caller.  The inputs are checked on the device before
// any kernel indexes by them, and the slot lists' total against the array
// before they are written.
extern "C" INT hzb_rap_agg_device_noalloc(INT n, INT nnz, const INT *ia, const INT *ja,
                                          const REAL *val, INT nc, const INT *agg,
                                          INT cap_nnz, INT *rap_ia, INT *rap_ja,
                                          REAL *rap_val, INT *rap_nnz) {
    using namespace hzb;
    if (n < 1 || nnz < 0 || nc < 1 || nc > n || (size_t)n > NA_ROWS || (size_t)nnz > NA_NNZ) {
        set_error_msg("hzb_rap_agg_device_noalloc: sizes beyond HZB_NOALLOC_MAX_ROWS / "
                      "HZB_NOALLOC_MAX_NNZ");
        return ERROR_MAT_SIZE;
    }
    if (!ia || !ja || !val || !agg || !rap_ia || !rap_nnz || cap_nnz < 0) {
        set_error_msg("hzb_rap_agg_device_noalloc: null array or negative capacity");
        return ERROR_INPUT_PAR;
    }
    double *base = nullptr;
    HZB_TRY(noalloc_scratch(&base));
    int *ip = (int *)base;
    int *cnt = ip;                       ip += NA_ROWS + 1;
    int *ria = ip;                       ip += NA_ROWS + 1;
    int *rja = ip;                       ip += NA_ROWS + 1;
    int *ub = ip;                        ip += NA_ROWS + 1;
    int *off = ip;                       ip += NA_ROWS + 1;
    int *rowcnt = ip;                    ip += NA_ROWS + 1;
    int *tmp = ip;                       ip += NA_TMP;
    int *bad = ip;                       ip += 4;
    int *scol = ip;
    double *sval = base + NA_INT_WORDS;
    cudaStream_t s = 0;
    const int gn = grid_for(n), gc = grid_for(nc);
    HZB_TRY(check_rap_inputs(n, nnz, ia, ja, nc, agg, bad, s));
    // R = P^T (counts start at zero: the array keeps the previous call's data)
    HZB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * nc, s));
    k_agg_count<<<gn, 256, 0, s>>>(n, agg, cnt);
    count_launch();
    HZB_TRY(scan_exclusive(cnt, ria, nc, tmp, s));
    HZB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * nc, s));
    k_agg_fill<<<gn, 256, 0, s>>>(n, agg, ria, cnt, rja);
    k_sort_rows<<<gc, 256, 0, s>>>(nc, ria, rja);
    // slot lists per coarse row, then the compacted product
    k_rap_bound<<<gc, 256, 0, s>>>(nc, ria, rja, ia, ub);
    count_launch(3);
    HZB_TRY(scan_exclusive(ub, off, nc, tmp, s));
    int slots = 0;
    HZB_CUDA(cudaMemcpyAsync(&slots, off + nc, sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    if (slots < 0 || (size_t)slots > NA_SLOTS) {
        set_error_msg("hzb_rap_agg_device_noalloc: the slot lists exceed the static scratch");
        return ERROR_MAT_SIZE;
    }
    k_rap_build<<<gc, 128, 0, s>>>(nc, ria, rja, ia, ja, val, agg, off, scol, sval, rowcnt);
    count_launch();
    HZB_TRY(scan_exclusive(rowcnt, rap_ia, nc, tmp, s));
    int total = 0;
    HZB_CUDA(cudaMemcpyAsync(&total, rap_ia + nc, sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    *rap_nnz = total;
    if (total > cap_nnz) {
        set_error_msg("hzb_rap_agg_device_noalloc: output capacity too small (*rap_nnz "
                      "holds the size needed)");
        return ERROR_INPUT_PAR;
    }
    if (total > 0 && (!rap_ja || !rap_val)) {
        set_error_msg("hzb_rap_agg_device_noalloc: null output array");
        return ERROR_INPUT_PAR;
    }
    k_rap_compact<<<gc, 256, 0, s>>>(nc, off, rap_ia, scol, sval, rap_ja, rap_val);
    count_launch();
    HZB_CUDA(cudaStreamSynchronize(s));
    return SUCCESS;
}
