// hzb_batch.cu -- many independent SPD systems solved in one pass.
//
// The systems are packed into one block-diagonal CSR arena: rows and columns
// of system s are [off[s], off[s+1]).  One UA-AMG hierarchy is built on the
// union.  Strength graph, matching and Galerkin product only ever combine
// coupled rows, so aggregates never cross systems, coarse rows of a system
// stay contiguous, and the block of every level that belongs to system s is
// a UA-AMG hierarchy of s alone.  One V-cycle over the union therefore
// applies every system's preconditioner in one set of launches (the level
// kernels are grid-wide row-bundle kernels with autotuned bundle sizes).
//
// The Krylov method is one flexible CG per system: every inner product,
// step length and convergence test is per system.  The per-system vector
// work runs on persistent kernels that pull (system, row range) items from a
// device work queue, so systems of 1k and 200k rows share the SMs evenly and
// the items of converged systems cost one flag read.  The items of a system
// are contiguous and reduced in order, so every per-system scalar is
// deterministic.  One iteration of all systems is captured in a CUDA graph;
// the host replays it and reads one counter (systems still active) per
// iteration.  A converged system keeps its iterate, and the kernel that
// retires it stamps the device clock, which gives per-system solve times.
//
// No counterpart in the reference, whose solvers take one system per call.
#include "hzb_solver.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace hzb {

constexpr int BAT_CHUNK = 4096;     // rows per work item
constexpr int BAT_TERM_ROWS = 128;  // a system's coarsening ends at this many rows
constexpr int BAT_THREADS = 256;
enum BatState { BAT_DONE = 0, BAT_ACTIVE = 1, BAT_CHECK = 2, BAT_FAILED = 3 };
// per-system scalars, sc[k * nsys + s]
enum BatScalar { B_ZR = 0, B_PT, B_ZT, B_RR, B_R0, B_REL, B_NS };

struct Batch {
    int nsys = 0, n = 0, nitems = 0, maxit = 0;
    double tol = 0.0;
    int *item_lo = nullptr, *item_hi = nullptr, *item_sys = nullptr;
    int *sys_item = nullptr;        // nsys + 1: items of s are [sys_item[s], sys_item[s+1])
    int *state = nullptr, *iters = nullptr;
    double *sc = nullptr, *part = nullptr;   // part: 2 per item
    unsigned long long *t_done = nullptr, *t_start = nullptr;
    unsigned *queue = nullptr;      // one counter per queued launch of an iteration
    int *nactive = nullptr;         // device count of active systems
    int *h_nactive = nullptr;       // pinned mirror
    GraphCache g_iter;
    // per level: the system of every row and the activity of 256-row blocks
    int nlev = 0, nblk_all = 0;
    std::vector<int *> sysmap;
    std::vector<unsigned char *> actv;
    int **d_sys = nullptr;          // device copies of the per-level pointers
    unsigned char **d_act = nullptr;
    int *d_nrows = nullptr, *d_blkoff = nullptr;   // rows, first block per level
    // Terminal levels: a system stops coarsening once it has at most
    // BAT_TERM_ROWS rows; on that level its block is solved with its dense
    // inverse (row-major, FP64 and an FP32 copy), and its rows leave the
    // coarser levels.  Per level: the blocks ending there.
    std::vector<unsigned char> done;          // host, per system: has its terminal block
    unsigned char *d_done = nullptr;          // device copy
    int *d_cnt = nullptr;                     // per-system row counts of a level
    std::vector<int> tl_n;                    // blocks per level
    std::vector<int *> tl_row0, tl_m;         // device: first row and size of each block
    std::vector<long long *> tl_off;          // device: offset of its inverse
    std::vector<double *> tl_inv;             // inverses of the level's blocks
    std::vector<float *> tl_inv32;
    void release() {
        g_iter.release();
        for (auto p : tl_row0) dfree(p);
        for (auto p : tl_m) dfree(p);
        for (auto p : tl_off) dfree(p);
        for (auto p : tl_inv) dfree(p);
        for (auto p : tl_inv32) dfree(p);
        tl_row0.clear(); tl_m.clear(); tl_off.clear(); tl_inv.clear(); tl_inv32.clear();
        tl_n.clear();
        done.clear();
        dfree(d_done); dfree(d_cnt);
        dfree(item_lo); dfree(item_hi); dfree(item_sys); dfree(sys_item);
        dfree(state); dfree(iters); dfree(sc); dfree(part);
        dfree(t_done); dfree(t_start); dfree(queue); dfree(nactive);
        for (auto p : sysmap) dfree(p);
        for (auto p : actv) dfree(p);
        sysmap.clear();
        actv.clear();
        dfree(d_sys); dfree(d_act); dfree(d_nrows); dfree(d_blkoff);
        if (h_nactive) cudaFreeHost(h_nactive);
        h_nactive = nullptr;
    }
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// every stored entry of a row of s must lie in s's column range
__global__ void k_bat_check_blocks(int nitems, const int *__restrict__ lo,
                                   const int *__restrict__ hi, const int *__restrict__ isys,
                                   const int *__restrict__ off, const int *__restrict__ ia,
                                   const int *__restrict__ ja, int *bad) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int s = isys[it], c0 = off[s], c1 = off[s + 1];
        for (int i = lo[it] + threadIdx.x; i < hi[it]; i += blockDim.x)
            for (int k = ia[i]; k < ia[i + 1]; ++k)
                if (ja[k] < c0 || ja[k] >= c1) atomicExch(bad, 1);
    }
}

// Work-queue loop: each CTA takes the next item until the queue is empty.
template <typename F>
__device__ __forceinline__ void bat_items(unsigned *queue, int nitems, F body) {
    __shared__ int item;
    for (;;) {
        if (threadIdx.x == 0) item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int it = item;
        __syncthreads();
        if (it >= nitems) break;
        body(it);
    }
}

enum BatOp { OP_PT = 0, OP_UPDATE, OP_ZTR, OP_PDIR, OP_TRUERES, OP_INIT };

// One kernel for the item-wise vector work of an iteration.
//   OP_PT      part = (p, t)                                     [active]
//   OP_UPDATE  x += a p, r -= a t, a = zr/pt; part = (r, r)      [active]
//   OP_TRUERES part = ||b - A x||^2 (thread per row, CSR order)  [check]
//   OP_ZTR     part = (z, t), (z, r)                             [active]
//   OP_PDIR    p = z + beta p, beta = -zt/pt                     [active]
//   OP_INIT    r = b - A x; part = (r, r)                         [all]
template <int OP>
__global__ void __launch_bounds__(BAT_THREADS)
k_bat_vec(int nitems, int nsys, unsigned *queue, const int *__restrict__ lo,
          const int *__restrict__ hi, const int *__restrict__ isys,
          const int *__restrict__ state, const double *__restrict__ sc,
          const int *__restrict__ ia, const int *__restrict__ ja,
          const double *__restrict__ a, const double *__restrict__ b, double *x,
          double *r, double *p, const double *__restrict__ z, const double *__restrict__ t,
          double *part) {
    __shared__ double sh[32];
    bat_items(queue, nitems, [&](int it) {
        const int s = isys[it];
        const int st = state[s];
        const bool run = OP == OP_INIT ? true
                         : OP == OP_TRUERES ? st == BAT_CHECK : st == BAT_ACTIVE;
        double u = 0.0, v = 0.0;
        if (run) {
            const int i0 = lo[it], i1 = hi[it];
            if (OP == OP_PT) {
                for (int i = i0 + threadIdx.x; i < i1; i += BAT_THREADS) u += p[i] * t[i];
            } else if (OP == OP_UPDATE) {
                const double al = sc[B_ZR * nsys + s] / sc[B_PT * nsys + s];
                for (int i = i0 + threadIdx.x; i < i1; i += BAT_THREADS) {
                    x[i] += al * p[i];
                    const double ri = r[i] - al * t[i];
                    r[i] = ri;
                    u += ri * ri;
                }
            } else if (OP == OP_ZTR) {
                for (int i = i0 + threadIdx.x; i < i1; i += BAT_THREADS) {
                    const double zi = z[i];
                    u += zi * t[i];
                    v += zi * r[i];
                }
            } else if (OP == OP_PDIR) {
                const double be = -sc[B_ZT * nsys + s] / sc[B_PT * nsys + s];
                for (int i = i0 + threadIdx.x; i < i1; i += BAT_THREADS)
                    p[i] = z[i] + be * p[i];
            } else {   // OP_TRUERES, OP_INIT
                for (int i = i0 + threadIdx.x; i < i1; i += BAT_THREADS) {
                    double acc = 0.0;
                    for (int k = ia[i]; k < ia[i + 1]; ++k) acc += a[k] * x[ja[k]];
                    const double ri = b[i] - acc;
                    if (OP == OP_INIT) r[i] = ri;
                    u += ri * ri;
                }
            }
        }
        if (OP != OP_PDIR) {
            u = block_sum(u, sh);
            if (OP == OP_ZTR) v = block_sum(v, sh);
            if (threadIdx.x == 0) {
                part[2 * it] = u;
                part[2 * it + 1] = v;
            }
        }
    });
}

enum BatFinal { FIN_PT = 0, FIN_UPDATE, FIN_TRUERES, FIN_ZTR, FIN_INIT, FIN_ZR0 };

// Per-system ordered sums of the item partials and the decisions on them.
template <int FIN>
__global__ void k_bat_final(int nsys, const int *__restrict__ sys_item,
                            const double *__restrict__ part, double *sc, int *state,
                            int *iters, unsigned long long *t_done, int maxit, double tol,
                            int *nactive) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys;
         s += gridDim.x * blockDim.x) {
        const int st = state[s];
        double u = 0.0, v = 0.0;
        for (int it = sys_item[s]; it < sys_item[s + 1]; ++it) {
            u += part[2 * it];
            v += part[2 * it + 1];
        }
        if (FIN == FIN_PT) {
            if (st == BAT_ACTIVE) sc[B_PT * nsys + s] = u;
        } else if (FIN == FIN_UPDATE) {
            if (st != BAT_ACTIVE) continue;
            const int k = ++iters[s];
            sc[B_RR * nsys + s] = u;
            const double rel = sqrt(u) / sc[B_R0 * nsys + s];
            sc[B_REL * nsys + s] = rel;
            if (rel < tol) state[s] = BAT_CHECK;
            else if (k >= maxit) { state[s] = BAT_FAILED; t_done[s] = global_ns(); }
        } else if (FIN == FIN_TRUERES) {
            if (st == BAT_CHECK) {
                const double rel = sqrt(u) / sc[B_R0 * nsys + s];
                if (rel < tol) {
                    sc[B_REL * nsys + s] = rel;
                    state[s] = BAT_DONE;
                    t_done[s] = global_ns();
                } else {
                    state[s] = iters[s] >= maxit ? BAT_FAILED : BAT_ACTIVE;
                    if (state[s] == BAT_FAILED) t_done[s] = global_ns();
                }
            }
            if (state[s] == BAT_ACTIVE) atomicAdd(nactive, 1);
        } else if (FIN == FIN_ZTR) {
            if (st == BAT_ACTIVE) {
                sc[B_ZT * nsys + s] = u;
                sc[B_ZR * nsys + s] = v;
            }
        } else if (FIN == FIN_INIT) {   // r0 = b - A x0
            const double r0 = sqrt(u);
            sc[B_R0 * nsys + s] = fmax(r0, SMALLREAL);
            const double rel = r0 / fmax(r0, SMALLREAL);
            sc[B_REL * nsys + s] = rel;
            iters[s] = 0;
            const bool done = rel < tol || r0 < 1e-3 * tol;
            state[s] = done ? BAT_DONE : BAT_ACTIVE;
            t_done[s] = 0ull;
        } else {   // FIN_ZR0: (z, r) of the first direction
            if (st == BAT_ACTIVE) sc[B_ZR * nsys + s] = v;
        }
    }
}

__global__ void k_bat_stamp(unsigned long long *t, int nsys, const int *state,
                            unsigned long long *t_done) {
    const unsigned long long now = global_ns();
    if (blockIdx.x == 0 && threadIdx.x == 0) *t = now;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys;
         s += gridDim.x * blockDim.x)
        if (state[s] == BAT_DONE) t_done[s] = now;
}

// row -> system on level 0 (from the work items) and on the levels below
// (every member of an aggregate belongs to the aggregate's system)
__global__ void k_bat_sys0(int nitems, const int *__restrict__ lo, const int *__restrict__ hi,
                           const int *__restrict__ isys, int *sys) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x)
        for (int i = lo[it] + threadIdx.x; i < hi[it]; i += blockDim.x) sys[i] = isys[it];
}
__global__ void k_bat_sys_down(int n, const int *__restrict__ agg,
                               const int *__restrict__ sys, int *sys_c) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (agg[i] >= 0) sys_c[agg[i]] = sys[i];
}

// Activity of every 256-row block of every level: a block is active if a row
// of it belongs to an active system.  A warp per block checks every row.
__global__ void k_bat_activity(int nlev, int nblk_all, const int *__restrict__ blkoff,
                               const int *__restrict__ nrows, int *const *__restrict__ sys,
                               unsigned char *const *__restrict__ act,
                               const int *__restrict__ state) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < nblk_all; g += nw) {
        int l = 0;
        while (l + 1 < nlev && blkoff[l + 1] <= g) ++l;
        const int blk = g - blkoff[l], n = nrows[l];
        const int r0 = blk * ACT_ROWS, r1 = min(r0 + ACT_ROWS, n);
        bool a = false;
        for (int r = r0 + lane; r < r1 && !a; r += 32) a = state[sys[l][r]] == BAT_ACTIVE;
        const unsigned any = __ballot_sync(0xffffffffu, a);
        if (lane == 0) act[l][blk] = any != 0u;
    }
}

static int bat_grid(int nitems) { return std::max(1, std::min(nitems, sm_count() * 8)); }

// rows of every system on a level
__global__ void k_bat_count(int n, const int *__restrict__ sys, int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(cnt + sys[i], 1);
}

// Dense inverse of each terminal block (one CTA per block, the block in
// shared memory): the block's CSR rows [row0, row0 + m) scattered into an
// m x m matrix (its columns lie in the same range: systems do not couple),
// then Gauss-Jordan elimination in place without pivoting (the block is
// SPD): for each k the pivot row is scaled by 1 / a_kk with a_kk replaced by
// 1, and every other row subtracts its column-k multiple of it with its
// column-k entry replaced by 0; after m steps the array holds the inverse.
// A pivot that is not positive and finite sets *bad.
__global__ void __launch_bounds__(256)
k_bat_term_inverse(int nblk, const int *__restrict__ row0, const int *__restrict__ msz,
                   const long long *__restrict__ off, const int *__restrict__ ia,
                   const int *__restrict__ ja, const double *__restrict__ val,
                   double *inv, float *inv32, int *bad) {
    extern __shared__ double sa[];
    const int blk = blockIdx.x;
    if (blk >= nblk) return;
    const int m = msz[blk], r0 = row0[blk];
    double *A = sa;               // m x m, row-major
    double *colk = sa + m * m;    // column k before the step
    for (int q = threadIdx.x; q < m * m; q += blockDim.x) A[q] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x)
        for (int p = ia[r0 + i]; p < ia[r0 + i + 1]; ++p) {
            const int j = ja[p] - r0;
            if (j >= 0 && j < m) A[i * m + j] += val[p];
        }
    bool ok = true;
    for (int k = 0; k < m; ++k) {
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) colk[i] = A[i * m + k];
        __syncthreads();
        const double piv = colk[k];
        if (!(piv > 0.0) || !isfinite(piv)) { ok = false; break; }
        for (int j = threadIdx.x; j < m; j += blockDim.x)
            A[k * m + j] = (j == k ? 1.0 : A[k * m + j]) / piv;
        __syncthreads();
        for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
            const int i = q / m, j = q - i * m;
            if (i != k) A[q] = (j == k ? 0.0 : A[q]) - colk[i] * A[k * m + j];
        }
    }
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(bad, 1);
        return;
    }
    __syncthreads();
    double *out = inv + off[blk];
    float *out32 = inv32 + off[blk];
    for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
        out[q] = A[q];
        out32[q] = (float)A[q];
    }
}

// x = inverse * b on every terminal block of a level (one CTA per block, a
// warp per row, lanes over the row's columns, fixed-order lane sums)
template <typename T, typename V>
__global__ void __launch_bounds__(256)
k_bat_term_solve(int nblk, const int *__restrict__ row0, const int *__restrict__ msz,
                 const long long *__restrict__ off, const V *__restrict__ inv,
                 const T *__restrict__ b, T *__restrict__ x) {
    __shared__ T sb[BAT_TERM_ROWS];
    const int blk = blockIdx.x;
    const int m = msz[blk], r0 = row0[blk];
    for (int j = threadIdx.x; j < m; j += blockDim.x) sb[j] = b[r0 + j];
    __syncthreads();
    const V *M = inv + off[blk];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = warp; i < m; i += nw) {
        T acc = T(0);
        for (int j = lane; j < m; j += 32) acc += T(M[(size_t)i * m + j]) * sb[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) x[r0 + i] = acc;
    }
}

// terminal systems' rows leave the next level; the surviving aggregates are
// renumbered in order (the rows of a system stay contiguous)
__global__ void k_bat_mask(int n, const int *__restrict__ sys,
                           const unsigned char *__restrict__ done, int *agg, int *kept) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (agg[i] < 0) continue;
        if (done[sys[i]]) agg[i] = UNPT;
        else kept[agg[i]] = 1;
    }
}
__global__ void k_bat_renumber(int n, const int *__restrict__ pos, int *agg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (agg[i] >= 0) agg[i] = pos[agg[i]];
}

// Which systems end their coarsening on level lvl (at most BAT_TERM_ROWS
// rows there, or every system left when force is set), their dense
// inverses, and the rows of the systems that go on (*live).
int batch_level_begin(hzb_solver *S, int lvl, bool force, int *live) {
    Batch &B = *S->batch;
    cudaStream_t s = S->s;
    const Level &L = S->lv[lvl];
    if (lvl == 0) {
        B.sysmap.clear();
        B.sysmap.push_back(nullptr);
        HZB_TRY(dalloc(&B.sysmap[0], std::max(1, L.n)));
        k_bat_sys0<<<bat_grid(B.nitems), 256, 0, s>>>(B.nitems, B.item_lo, B.item_hi,
                                                      B.item_sys, B.sysmap[0]);
        count_launch();
        B.done.assign(B.nsys, 0);
        if (!B.d_done) HZB_TRY(dalloc(&B.d_done, B.nsys));
        if (!B.d_cnt) HZB_TRY(dalloc(&B.d_cnt, B.nsys));
    }
    if ((int)B.tl_n.size() <= lvl) {
        B.tl_n.resize(lvl + 1, 0);
        B.tl_row0.resize(lvl + 1, nullptr);
        B.tl_m.resize(lvl + 1, nullptr);
        B.tl_off.resize(lvl + 1, nullptr);
        B.tl_inv.resize(lvl + 1, nullptr);
        B.tl_inv32.resize(lvl + 1, nullptr);
    }
    HZB_CUDA(cudaMemsetAsync(B.d_cnt, 0, sizeof(int) * B.nsys, s));
    if (L.n > 0) {
        k_bat_count<<<grid_for(L.n), 256, 0, s>>>(L.n, B.sysmap[lvl], B.d_cnt);
        count_launch();
    }
    std::vector<int> cnt(B.nsys);
    HZB_CUDA(cudaMemcpyAsync(cnt.data(), B.d_cnt, sizeof(int) * B.nsys, cudaMemcpyDeviceToHost,
                             s));
    HZB_CUDA(cudaStreamSynchronize(s));
    std::vector<int> row0, msz;
    std::vector<long long> off;
    long long words = 0;
    int r = 0, mmax = 0;
    *live = 0;
    for (int k = 0; k < B.nsys; ++k) {
        const int c = cnt[k];
        if (c > 0 && !B.done[k]) {
            if (c <= BAT_TERM_ROWS || force) {
                if (c > BAT_TERM_ROWS) {
                    set_error_msg("batch: a system still has more rows than its terminal "
                                  "block may hold on the last level (raise max_levels)");
                    return ERROR_AMG_COARSEING;
                }
                row0.push_back(r);
                msz.push_back(c);
                off.push_back(words);
                words += (long long)c * c;
                mmax = std::max(mmax, c);
                B.done[k] = 1;
            } else {
                *live += c;
            }
        }
        r += c;
    }
    if (r != L.n) {
        set_error_msg("batch: the rows of a level do not add up over the systems");
        return ERROR_SOLVER_MISC;
    }
    const int nb = (int)row0.size();
    B.tl_n[lvl] = nb;
    HZB_CUDA(cudaMemcpyAsync(B.d_done, B.done.data(), B.nsys, cudaMemcpyHostToDevice, s));
    if (nb == 0) return SUCCESS;
    int *bad = B.d_cnt;   // the counts are on the host now
    HZB_TRY(dalloc(&B.tl_row0[lvl], nb));
    HZB_TRY(dalloc(&B.tl_m[lvl], nb));
    HZB_TRY(dalloc(&B.tl_off[lvl], nb));
    HZB_TRY(dalloc(&B.tl_inv[lvl], (size_t)words));
    HZB_TRY(dalloc(&B.tl_inv32[lvl], (size_t)words));
    HZB_CUDA(cudaMemcpyAsync(B.tl_row0[lvl], row0.data(), sizeof(int) * nb,
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(B.tl_m[lvl], msz.data(), sizeof(int) * nb, cudaMemcpyHostToDevice,
                             s));
    HZB_CUDA(cudaMemcpyAsync(B.tl_off[lvl], off.data(), sizeof(long long) * nb,
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    const size_t smem = sizeof(double) * ((size_t)mmax * mmax + mmax);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_bat_term_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * (BAT_TERM_ROWS * BAT_TERM_ROWS +
                                                     BAT_TERM_ROWS)));
        attr = true;
    }
    k_bat_term_inverse<<<nb, 256, smem, s>>>(nb, B.tl_row0[lvl], B.tl_m[lvl], B.tl_off[lvl],
                                             L.ia, L.ja, L.val, B.tl_inv[lvl],
                                             B.tl_inv32[lvl], bad);
    count_launch();
    HZB_LAUNCH_CHECK();
    int hbad = 0;
    HZB_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    if (hbad) {
        set_error_msg("batch: a system's terminal block has a non-positive pivot");
        return ERROR_DATA_ZERODIAG;
    }
    return SUCCESS;
}

// After level lvl's aggregation: rows of systems that ended here leave the
// coarser levels, the other aggregates are renumbered in order; the row ->
// system map of the next level.  *nagg becomes the surviving count.
int batch_level_end(hzb_solver *S, int lvl, int *agg, int *nagg) {
    Batch &B = *S->batch;
    cudaStream_t s = S->s;
    const int n = S->lv[lvl].n;
    int *kept = nullptr, *pos = nullptr, *tmp = nullptr;
    int rc = SUCCESS;
    if ((rc = dalloc(&kept, std::max(1, *nagg))) || (rc = dalloc(&pos, *nagg + 1)) ||
        (rc = dalloc(&tmp, scan_tmp_size(*nagg + 1)))) {
        dfree(kept); dfree(pos); dfree(tmp);
        return rc;
    }
    int total = 0;
    cudaMemsetAsync(kept, 0, sizeof(int) * std::max(1, *nagg), s);
    k_bat_mask<<<grid_for(n), 256, 0, s>>>(n, B.sysmap[lvl], B.d_done, agg, kept);
    count_launch();
    rc = scan_exclusive(kept, pos, *nagg, tmp, s);
    if (!rc) {
        k_bat_renumber<<<grid_for(n), 256, 0, s>>>(n, pos, agg);
        count_launch();
        if (cudaMemcpyAsync(&total, pos + *nagg, sizeof(int), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            rc = ERROR_SOLVER_MISC;
    }
    dfree(kept); dfree(pos); dfree(tmp);
    if (rc) return rc;
    *nagg = total;
    if (total > 0) {
        int *sc = nullptr;
        HZB_TRY(dalloc(&sc, total));
        B.sysmap.push_back(sc);
        k_bat_sys_down<<<grid_for(n), 256, 0, s>>>(n, agg, B.sysmap[lvl], sc);
        count_launch();
    }
    return SUCCESS;
}

// x = A_T^{-1} b on the terminal blocks of level lvl (no-op without any)
int batch_terminal_solve(hzb_solver *S, int lvl, bool fp32) {
    Batch &B = *S->batch;
    if (lvl >= (int)B.tl_n.size() || B.tl_n[lvl] == 0) return SUCCESS;
    const Level &L = S->lv[lvl];
    if (fp32)
        k_bat_term_solve<float, float><<<B.tl_n[lvl], 256, 0, S->s>>>(
            B.tl_n[lvl], B.tl_row0[lvl], B.tl_m[lvl], B.tl_off[lvl], B.tl_inv32[lvl], L.b32,
            L.x32);
    else
        k_bat_term_solve<double, double><<<B.tl_n[lvl], 256, 0, S->s>>>(
            B.tl_n[lvl], B.tl_row0[lvl], B.tl_m[lvl], B.tl_off[lvl], B.tl_inv[lvl], L.b, L.x);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

bool batch_has_terminal(const hzb_solver *S, int lvl) {
    const Batch *B = S->batch;
    return B && lvl < (int)B->tl_n.size() && B->tl_n[lvl] > 0;
}

static int bat_activity(hzb_solver *S, Batch &B) {
    if (B.nblk_all == 0) return SUCCESS;
    k_bat_activity<<<grid_for(32LL * B.nblk_all), 256, 0, S->s>>>(
        B.nlev, B.nblk_all, B.d_blkoff, B.d_nrows, B.d_sys, B.d_act, B.state);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

template <int OP>
static int bat_vec(hzb_solver *S, Batch &B, unsigned *q, const double *b, double *x,
                   double *r, double *p, const double *z, const double *t) {
    const Level &L = S->lv[0];
    HZB_CUDA(cudaMemsetAsync(q, 0, sizeof(unsigned), S->s));
    k_bat_vec<OP><<<bat_grid(B.nitems), BAT_THREADS, 0, S->s>>>(
        B.nitems, B.nsys, q, B.item_lo, B.item_hi, B.item_sys, B.state, B.sc, L.ia, L.ja,
        L.val, b, x, r, p, z, t, B.part);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

template <int FIN>
static int bat_final(hzb_solver *S, Batch &B) {
    k_bat_final<FIN><<<std::max(1, (B.nsys + 127) / 128), 128, 0, S->s>>>(
        B.nsys, B.sys_item, B.part, B.sc, B.state, B.iters, B.t_done, B.maxit, B.tol,
        B.nactive);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

static int bat_precond(hzb_solver *S, const double *r, double *z);

// one flexible-CG iteration of every active system
static int bat_iteration(hzb_solver *S, Batch &B, const double *b, double *x) {
    KrylovWork &w = S->kw;
    const DCsr<double> A = S->lv[0].A64();
    unsigned *q = B.queue;
    HZB_TRY(spmv<double>(A, SPMV_Y, w.p, nullptr, w.t, 1.0, nullptr, S->s));
    HZB_TRY(bat_vec<OP_PT>(S, B, q + 0, b, x, w.r, w.p, w.z, w.t));
    HZB_TRY(bat_final<FIN_PT>(S, B));
    HZB_TRY(bat_vec<OP_UPDATE>(S, B, q + 1, b, x, w.r, w.p, w.z, w.t));
    HZB_TRY(bat_final<FIN_UPDATE>(S, B));
    HZB_TRY(bat_vec<OP_TRUERES>(S, B, q + 2, b, x, w.r, w.p, w.z, w.t));
    HZB_CUDA(cudaMemsetAsync(B.nactive, 0, sizeof(int), S->s));
    HZB_TRY(bat_final<FIN_TRUERES>(S, B));
    HZB_CUDA(cudaMemcpyAsync(B.h_nactive, B.nactive, sizeof(int), cudaMemcpyDeviceToHost,
                             S->s));
    HZB_TRY(bat_activity(S, B));       // the cycle and the next SpMV skip retired systems
    HZB_TRY(bat_precond(S, w.r, w.z));
    HZB_TRY(bat_vec<OP_ZTR>(S, B, q + 3, b, x, w.r, w.p, w.z, w.t));
    HZB_TRY(bat_final<FIN_ZTR>(S, B));
    HZB_TRY(bat_vec<OP_PDIR>(S, B, q + 4, b, x, w.r, w.p, w.z, w.t));
    return SUCCESS;
}

// the preconditioner of the union: FP32 cycle (mixed) or FP64 cycle
static int bat_precond(hzb_solver *S, const double *r, double *z) {
    Level &L0 = S->lv[0];
    AMG_param cyc = S->amg;
    if (S->bp.precision == HZB_PREC_MIXED) {
        HZB_TRY(d2f(L0.n, r, L0.b32, S->s, L0.act));
        for (int i = 0; i < std::max<int>(1, cyc.maxit); ++i) HZB_TRY(cycle32(S, cyc, i == 0));
        return f2d(L0.n, L0.x32, z, S->s, L0.act);
    }
    HZB_TRY(vcopy<double>(L0.n, r, L0.b, S->s));
    HZB_TRY(vzero<double>(L0.n, L0.x, S->s));
    for (int i = 0; i < std::max<int>(1, cyc.maxit); ++i) HZB_TRY(cycle64(S, cyc, 0));
    return vcopy<double>(L0.n, L0.x, z, S->s);
}

void batch_release(hzb_solver *S) {
    if (!S->batch) return;
    S->batch->release();
    delete S->batch;
    S->batch = nullptr;
}

int batch_setup(hzb_solver *S, int nsys, const int *off, int n, int nnz, const int *d_ia,
                const int *d_ja, const double *d_val) {
    if (nsys < 1 || !off || off[0] != 0 || off[nsys] != n || n < 1) return ERROR_INPUT_PAR;
    for (int s = 0; s < nsys; ++s)
        if (off[s + 1] < off[s]) return ERROR_INPUT_PAR;
    batch_release(S);
    Batch *B = new Batch();
    S->batch = B;
    B->nsys = nsys;
    B->n = n;
    std::vector<int> lo, hi, isys, sitem(nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) {
        sitem[s] = (int)lo.size();
        for (int i = off[s]; i < off[s + 1]; i += BAT_CHUNK) {
            lo.push_back(i);
            hi.push_back(std::min(off[s + 1], i + BAT_CHUNK));
            isys.push_back(s);
        }
    }
    sitem[nsys] = (int)lo.size();
    B->nitems = (int)lo.size();
    const int ni = std::max(1, B->nitems);
    int *doff = nullptr, *bad = nullptr;
    int rc = SUCCESS;
    if ((rc = dalloc(&B->item_lo, ni)) || (rc = dalloc(&B->item_hi, ni)) ||
        (rc = dalloc(&B->item_sys, ni)) || (rc = dalloc(&B->sys_item, nsys + 1)) ||
        (rc = dalloc(&B->state, nsys)) || (rc = dalloc(&B->iters, nsys)) ||
        (rc = dalloc(&B->sc, (size_t)B_NS * nsys)) || (rc = dalloc(&B->part, 2 * (size_t)ni)) ||
        (rc = dalloc(&B->t_done, nsys)) || (rc = dalloc(&B->t_start, 1)) ||
        (rc = dalloc(&B->queue, 8)) || (rc = dalloc(&B->nactive, 1)) ||
        (rc = dalloc(&doff, nsys + 1)) || (rc = dalloc(&bad, 1))) {
        dfree(doff); dfree(bad);
        batch_release(S);
        return rc;
    }
    if (cudaMallocHost((void **)&B->h_nactive, sizeof(int)) != cudaSuccess) {
        dfree(doff); dfree(bad);
        batch_release(S);
        return ERROR_ALLOC_MEM;
    }
    cudaStream_t s = S->s;
    HZB_CUDA(cudaMemcpyAsync(B->item_lo, lo.data(), lo.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(B->item_hi, hi.data(), hi.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(B->item_sys, isys.data(), isys.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(B->sys_item, sitem.data(), sitem.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(doff, off, (nsys + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    k_bat_check_blocks<<<bat_grid(B->nitems), 256, 0, s>>>(B->nitems, B->item_lo, B->item_hi,
                                                           B->item_sys, doff, d_ia, d_ja, bad);
    count_launch();
    int hbad = 0;
    HZB_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    dfree(doff);
    dfree(bad);
    if (hbad) {
        batch_release(S);
        return ERROR_INPUT_PAR;   // an entry couples two systems
    }
    rc = setup(S, n, nnz, d_ia, d_ja, d_val, true);
    if (rc) {
        batch_release(S);
        return rc;
    }
    if (S->bp.precision == HZB_PREC_MIXED) HZB_TRY(ensure_fp32(S));
    // activity blocks per level (the row -> system maps were built by the
    // setup's level loop along with the terminal blocks)
    B->nlev = S->nl;
    if ((int)B->sysmap.size() != S->nl) {
        set_error_msg("batch: row -> system maps missing for a level");
        batch_release(S);
        return ERROR_SOLVER_MISC;
    }
    std::vector<int> nrows(S->nl), blkoff(S->nl + 1, 0);
    B->actv.assign(S->nl, nullptr);
    for (int l = 0; l < S->nl; ++l) {
        const int nl_rows = S->lv[l].n;
        nrows[l] = nl_rows;
        blkoff[l + 1] = blkoff[l] + (nl_rows + ACT_ROWS - 1) / ACT_ROWS;
        HZB_TRY(dalloc(&B->actv[l], std::max(1, blkoff[l + 1] - blkoff[l])));
    }
    B->nblk_all = blkoff[S->nl];
    HZB_TRY(dalloc(&B->d_sys, S->nl));
    HZB_TRY(dalloc(&B->d_act, S->nl));
    HZB_TRY(dalloc(&B->d_nrows, S->nl));
    HZB_TRY(dalloc(&B->d_blkoff, S->nl + 1));
    HZB_CUDA(cudaMemcpyAsync(B->d_sys, B->sysmap.data(), S->nl * sizeof(int *),
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(B->d_act, B->actv.data(), S->nl * sizeof(unsigned char *),
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(B->d_nrows, nrows.data(), S->nl * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(B->d_blkoff, blkoff.data(), (S->nl + 1) * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaStreamSynchronize(s));   // the host vectors go out of scope
    return SUCCESS;
}

int batch_solve(hzb_solver *S, const double *b, double *x, double tol, int maxit,
                int *h_iters, double *h_relres, double *h_seconds) {
    Batch *B = S->batch;
    if (!B || S->lv.empty() || S->lv[0].n != B->n) return ERROR_SOLVER_MISC;
    B->tol = tol;
    B->maxit = maxit;
    KrylovWork &w = S->kw;
    cudaStream_t s = S->s;
    if (w.n != B->n) HZB_TRY(w.alloc(B->n));
    unsigned *q = B->queue;
    // the level kernels skip converged systems while this solve runs
    struct ActScope {
        hzb_solver *S;
        ~ActScope() { for (auto &L : S->lv) L.act = nullptr; }
    } act_scope{S};
    for (int l = 0; l < S->nl; ++l) S->lv[l].act = B->actv[l];
    // r = b - A x0, per-system norms; z = B r, p = z, (z, r)
    HZB_TRY(bat_vec<OP_INIT>(S, *B, q + 5, b, x, w.r, w.p, w.z, w.t));
    HZB_TRY(bat_final<FIN_INIT>(S, *B));
    HZB_TRY(bat_activity(S, *B));
    k_bat_stamp<<<std::max(1, (B->nsys + 127) / 128), 128, 0, s>>>(B->t_start, B->nsys,
                                                                   B->state, B->t_done);
    count_launch();
    HZB_TRY(bat_precond(S, w.r, w.z));
    HZB_TRY(vcopy<double>(B->n, w.z, w.p, s));
    HZB_TRY(bat_vec<OP_ZTR>(S, *B, q + 6, b, x, w.r, w.p, w.z, w.t));
    HZB_TRY(bat_final<FIN_ZR0>(S, *B));
    // the FP64 cycle is capturable without coarse scaling (its coarsest
    // solves are the systems' dense terminal blocks)
    const bool graph = S->bp.use_graph &&
                       (S->bp.precision == HZB_PREC_MIXED || S->amg.coarse_scaling != ON);
    int iter = 0;
    for (;;) {
        const long long tag = ((long long)S->omega_active << 1) | (S->bp.precision & 1);
        if (graph) {
            if (!B->g_iter.exec || B->g_iter.k0 != b || B->g_iter.k1 != x ||
                B->g_iter.tag != tag) {
                B->g_iter.release();
                const long long before = launch_count();
                HZB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                int rc = bat_iteration(S, *B, b, x);
                cudaGraph_t g = nullptr;
                cudaError_t e = cudaStreamEndCapture(s, &g);
                if (rc || e != cudaSuccess) {
                    if (g) cudaGraphDestroy(g);
                    if (e != cudaSuccess) set_error(e, __FILE__, __LINE__);
                    return rc ? rc : ERROR_SOLVER_MISC;
                }
                e = cudaGraphInstantiate(&B->g_iter.exec, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) {
                    B->g_iter.exec = nullptr;
                    set_error(e, __FILE__, __LINE__);
                    return ERROR_SOLVER_MISC;
                }
                B->g_iter.k0 = b;
                B->g_iter.k1 = x;
                B->g_iter.tag = tag;
                B->g_iter.kernels = launch_count() - before;
            } else {
                count_launch((int)B->g_iter.kernels);
            }
            HZB_CUDA(cudaGraphLaunch(B->g_iter.exec, s));
        } else {
            HZB_TRY(bat_iteration(S, *B, b, x));
        }
        HZB_CUDA(cudaStreamSynchronize(s));
        ++iter;
        if (*B->h_nactive == 0 || iter >= maxit) break;
    }
    // per-system results
    std::vector<int> st(B->nsys), its(B->nsys);
    std::vector<double> sc((size_t)B_NS * B->nsys);
    std::vector<unsigned long long> td(B->nsys);
    unsigned long long t0 = 0;
    HZB_CUDA(cudaMemcpyAsync(st.data(), B->state, B->nsys * sizeof(int),
                             cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaMemcpyAsync(its.data(), B->iters, B->nsys * sizeof(int),
                             cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaMemcpyAsync(sc.data(), B->sc, sc.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaMemcpyAsync(td.data(), B->t_done, B->nsys * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaMemcpyAsync(&t0, B->t_start, sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    int worst = 0;
    bool failed = false;
    for (int k = 0; k < B->nsys; ++k) {
        const bool ok = st[k] == BAT_DONE;
        failed |= !ok;
        if (h_iters) h_iters[k] = ok ? its[k] : ERROR_SOLVER_MAXIT;
        if (h_relres) h_relres[k] = sc[(size_t)B_REL * B->nsys + k];
        if (h_seconds) h_seconds[k] = td[k] >= t0 && td[k] ? (double)(td[k] - t0) * 1e-9 : 0.0;
        worst = std::max(worst, its[k]);
    }
    return failed ? ERROR_SOLVER_MAXIT : worst;
}

}  // namespace hzb
