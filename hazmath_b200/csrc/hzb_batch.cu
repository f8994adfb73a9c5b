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
    void release() {
        g_iter.release();
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
    // per-level row -> system maps and activity blocks
    B->nlev = S->nl;
    std::vector<int> nrows(S->nl), blkoff(S->nl + 1, 0);
    B->sysmap.assign(S->nl, nullptr);
    B->actv.assign(S->nl, nullptr);
    for (int l = 0; l < S->nl; ++l) {
        const int nl_rows = S->lv[l].n;
        nrows[l] = nl_rows;
        blkoff[l + 1] = blkoff[l] + (nl_rows + ACT_ROWS - 1) / ACT_ROWS;
        HZB_TRY(dalloc(&B->sysmap[l], std::max(1, nl_rows)));
        HZB_TRY(dalloc(&B->actv[l], std::max(1, blkoff[l + 1] - blkoff[l])));
    }
    B->nblk_all = blkoff[S->nl];
    k_bat_sys0<<<bat_grid(B->nitems), 256, 0, s>>>(B->nitems, B->item_lo, B->item_hi,
                                                   B->item_sys, B->sysmap[0]);
    count_launch();
    for (int l = 0; l + 1 < S->nl; ++l) {
        k_bat_sys_down<<<grid_for(S->lv[l].n), 256, 0, s>>>(S->lv[l].n, S->lv[l].agg,
                                                            B->sysmap[l], B->sysmap[l + 1]);
        count_launch();
    }
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
    // the FP64 cycle is capturable only with the dense coarse solve
    const bool graph = S->bp.use_graph &&
                       (S->bp.precision == HZB_PREC_MIXED ||
                        (S->amg.coarse_solver == SOLVER_UMFPACK && S->Ainv &&
                         S->amg.coarse_scaling != ON));
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
