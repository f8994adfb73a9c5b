// hzb_solver.cu -- UA-AMG hierarchy setup, V/W cycles and Krylov loops.
//
// Control flow mirrors the reference line by line (cited per function); all
// vector work is device kernels on one stream, the host only sequences them
// and reads back the scalars the reference's branches test.
#include "hzb_solver.cuh"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <chrono>

namespace hzb {

// ---------------------------------------------------------------------------
// small kernels local to the Krylov loops
// ---------------------------------------------------------------------------
__global__ void k_dot2_partial(int n, const double *__restrict__ z,
                               const double *__restrict__ t,
                               const double *__restrict__ r, double *part) {
    __shared__ double sh[32];
    double a = 0.0, b = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const double zi = z[i];
        a += zi * t[i];
        b += zi * r[i];
    }
    a = block_sum(a, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = a;
    b = block_sum(b, sh);
    if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = b;
}

// flexible-CG direction: p = z + beta p, beta = -(z, A p_old) / (p_old, A p_old)
__global__ void k_fcg_p(int n, const double *__restrict__ zt,
                        const double *__restrict__ pap,
                        const double *__restrict__ z, double *p) {
    const double beta = -zt[0] / pap[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

__global__ void k_copy_scalar(const double *src, double *dst) { *dst = *src; }

// The mixed solve's flexible-CG update: u += alpha p, r -= alpha t with
// alpha = num / den (the products as k_pcg_update forms them), the partial
// sums of (r, r), and the FP32 copy of r the cycle starts from.
__global__ void k_fcg_update(int n, const double *__restrict__ num,
                             const double *__restrict__ den, double *u, double *r,
                             const double *__restrict__ p, const double *__restrict__ t,
                             float *r32, double *part) {
    __shared__ double sh[32];
    const double alpha = num[0] / den[0];
    double rr = 0.0;
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
        r32[i] = (float)ri;
        rr += ri * ri;
    }
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = rr;
}

// (z, t) and (z, r) with z the cycle's FP32 output widened to FP64 (the
// values f2d would write), and p = z + beta p from the same z
__global__ void k_dot2_partial_f(int n, const float *__restrict__ z,
                                 const double *__restrict__ t,
                                 const double *__restrict__ r, double *part) {
    __shared__ double sh[32];
    double a = 0.0, b = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const double zi = (double)z[i];
        a += zi * t[i];
        b += zi * r[i];
    }
    a = block_sum(a, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = a;
    b = block_sum(b, sh);
    if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = b;
}
__global__ void k_fcg_p_f(int n, const double *__restrict__ zt,
                          const double *__restrict__ pap, const float *__restrict__ z,
                          double *p) {
    const double beta = -zt[0] / pap[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        p[i] = (double)z[i] + beta * p[i];
}

// ---------------------------------------------------------------------------
// containers
// ---------------------------------------------------------------------------
void Level::release() {
    if (own_A) { dfree(ia); dfree(ja); dfree(val); }
    ia = ja = nullptr; val = nullptr;
    dfree(val32);
    dfree(val64nz);
    sell32.release();
    if (own32) { dfree(ia32); dfree(ja32); }
    ia32 = ja32 = nullptr;
    own32 = false;
    dfree(agg); dfree(ria); dfree(rja);
    dfree(pia); dfree(pja); dfree(pval); dfree(rval);
    sa = false;
    dfree(b); dfree(x); dfree(w); dfree(t); dfree(r1);
    dfree(b32); dfree(x32); dfree(w32); dfree(t32);
    dfree(d_jac); dfree(d_gs_f); dfree(d_gs_b); dfree(d_sor_f); dfree(d_sor_b);
    dfree(d_gs32);
    dfree(l1_32);
    dfree(tia); dfree(tja); dfree(tval);
    fwd.release(); bwd.release(); col.release();
}

// scalar slots of KrylovWork::sc
// SC_ERR: raised (as an int) by a device wait that ran out; read with the
// scalars by every fetch
enum { SC_T1 = 0, SC_T2 = 1, SC_RR = 2, SC_UM = 3, SC_UU = 4, SC_PP = 5,
       SC_T3 = 6, SC_ZT = 7, SC_X = 8, SC_ERR = 15, SC_N = 16 };

int KrylovWork::alloc(int nn, cudaStream_t st) {
    // the device arrays follow the system size; the pinned host mirror of the
    // scalars has a fixed size and stays: page-locking host memory (and
    // freeing it, which waits for the whole device) took from a few to a few
    // hundred ms per setup
    release_device();
    n = nn;
    const int G = reduce_blocks(n);
    const int np = 4 * G + spmv_blocks_rows(n, 64) + 8;   // smallest bundle
    HZB_TRY(dalloc(&p, n));
    HZB_TRY(dalloc(&z, n));
    HZB_TRY(dalloc(&r, n));
    HZB_TRY(dalloc(&t, n));
    HZB_TRY(dalloc(&part, np));
    HZB_TRY(dalloc(&sc, SC_N));
    // on the stream the allocations were made on (the entry point's)
    HZB_CUDA(cudaMemsetAsync(sc, 0, SC_N * sizeof(double), st ? st : cur_stream()));
    if (!h_sc) HZB_CUDA(cudaMallocHost((void **)&h_sc, SC_N * sizeof(double)));
    return SUCCESS;
}
void KrylovWork::release_device() {
    dfree(p); dfree(z); dfree(r); dfree(t); dfree(part); dfree(sc);
    n = 0;
}
void KrylovWork::release() {
    release_device();
    if (h_sc) cudaFreeHost(h_sc);
    h_sc = nullptr;
}

static int fetch(hzb_solver *S, KrylovWork &w) {
    HZB_CUDA(cudaMemcpyAsync(w.h_sc, w.sc, SC_N * sizeof(double),
                             cudaMemcpyDeviceToHost, S->s));
    HZB_CUDA(cudaStreamSynchronize(S->s));
    int e = 0;
    memcpy(&e, w.h_sc + SC_ERR, sizeof(int));
    if (e) {
        cudaMemsetAsync(w.sc + SC_ERR, 0, sizeof(double), S->s);
        set_error_msg("a grid barrier of a Gauss-Seidel sweep ran out of time");
        return ERROR_SOLVER_MISC;
    }
    return SUCCESS;
}

// the word the cycle's device waits raise (for paths that do not fetch the
// outer loop's scalars every step)
int check_waits(hzb_solver *S) {
    if (!S->kw.sc) return SUCCESS;
    int e = 0;
    HZB_CUDA(cudaMemcpyAsync(&e, S->kw.sc + SC_ERR, sizeof(int), cudaMemcpyDeviceToHost, S->s));
    HZB_CUDA(cudaStreamSynchronize(S->s));
    if (e) {
        cudaMemsetAsync(S->kw.sc + SC_ERR, 0, sizeof(double), S->s);
        set_error_msg("a grid barrier of a Gauss-Seidel sweep ran out of time");
        return ERROR_SOLVER_MISC;
    }
    return SUCCESS;
}

int *wait_err(hzb_solver *S) {
    return S->kw.sc ? reinterpret_cast<int *>(S->kw.sc + SC_ERR) : nullptr;
}

// ||x||^2 into sc[slot] (deterministic)
static int norm2sq(hzb_solver *S, KrylovWork &w, int n, const double *x, int slot) {
    return dot(n, x, x, w.part, w.sc + slot, S->s);
}

// ---------------------------------------------------------------------------
// smoothing (mgcycle.c:76-240 dispatch) on one level
// ---------------------------------------------------------------------------
static int run_sets(hzb_solver *S, const DCsr<double> &A, const Schedule &sc,
                    int kind, const double *d, double w, const double *b,
                    double *x, bool reverse) {
    const int ns = (int)sc.h_ptr.size() - 1;
    // consecutive large sets go to one cooperative launch when the grid
    // barrier has its words (exact schedules) and a place to report to;
    // HZB_GS_GRID=0 launches them one by one instead (same results)
    static const bool grid_ok = [] {
        const char *e = getenv("HZB_GS_GRID");
        return !(e && e[0] == '0');
    }();
    int *err = grid_ok ? wait_err(S) : nullptr;
    if (!reverse) {
        const size_t nr = sc.run_first.size();
        for (size_t q = 0; q < nr; ++q) {
            const int f = sc.run_first[q], l = sc.run_last[q];
            if (l < 0) {
                size_t q2 = q;
                int max_set = 0;
                while (q2 < nr && sc.run_last[q2] < 0) {
                    const int k = sc.run_first[q2];
                    max_set = std::max(max_set, sc.h_ptr[k + 1] - sc.h_ptr[k]);
                    ++q2;
                }
                if (sc.bar && err && q2 - q > 1) {
                    const int f2 = sc.run_first[q2 - 1] + 1;
                    HZB_TRY(gs_sets_grid<double>(A, kind, sc.rows, sc.set_ptr, f, f2, max_set,
                                                 d, w, b, x, sc.bar, err, S->s));
                    q = q2 - 1;
                } else {
                    HZB_TRY(gs_rows<double>(A, kind, sc.rows + sc.h_ptr[f],
                                            sc.h_ptr[f + 1] - sc.h_ptr[f], d, w, b, x, S->s));
                }
            } else {
                HZB_TRY(gs_run<double>(A, kind, sc.rows, sc.set_ptr, f, l, sc.run_max[q], d, w,
                                       b, x, S->s));
            }
        }
    } else {
        for (int k = ns - 1; k >= 0; --k)
            HZB_TRY(gs_rows<double>(A, kind, sc.rows + sc.h_ptr[k],
                                    sc.h_ptr[k + 1] - sc.h_ptr[k], d, w, b, x, S->s));
    }
    return SUCCESS;
}

// forward Gauss-Seidel-type sweep (rows ascending) / backward (descending)
static int gs_sweep(hzb_solver *S, Level &L, int kind, bool forward, double w) {
    const DCsr<double> A = L.A64();
    const bool mc = S->bp.gs_schedule == HZB_GS_MULTICOLOR;
    const bool is_gs = (kind & 15) == 0;
    const double *d = is_gs ? (forward ? L.d_gs_f : L.d_gs_b)
                            : (forward ? L.d_sor_f : L.d_sor_b);
    if (mc) return run_sets(S, A, L.col, kind, d, w, L.b, L.x, !forward);
    return run_sets(S, A, forward ? L.fwd : L.bwd, kind, d, w, L.b, L.x, false);
}

// one forward Gauss-Seidel sweep of level l as the cycle runs it (the level's
// schedule, exact or multicolour), for hzb_time_kernel
int time_gs_sweep(hzb_solver *S, int l) {
    Level &L = S->lv[l];
    if (!L.d_gs_f) return ERROR_INPUT_PAR;   // the smoother of the setup is not GS
    return gs_sweep(S, L, 0, true, 1.0);
}

int smooth64(hzb_solver *S, int l, bool pre, const AMG_param &cyc) {
    Level &L = S->lv[l];
    const int sweeps = pre ? cyc.presmooth_iter : cyc.postsmooth_iter;
    const double w = cyc.relaxation;
    const DCsr<double> A = L.A64();
    switch (cyc.smoother) {
    // Jacobi-type sweeps read x and write a new iterate: they alternate
    // between x and t, and an odd count ends with one copy back into x.
    case SMOOTHER_JACOBI:
        for (int k = 0; k < sweeps; ++k)
            HZB_TRY(jacobi_sweep(A, L.d_jac, L.b, k & 1 ? L.t : L.x, k & 1 ? L.x : L.t, S->s));
        if (sweeps & 1) HZB_TRY(vcopy(L.n, L.t, L.x, S->s));
        return SUCCESS;
    case SMOOTHER_L1DIAG: {
        const float *om = (l == 0 && S->omega_active) ? S->omega : nullptr;
        for (int k = 0; k < sweeps; ++k)
            HZB_TRY(l1_sweep<double>(A, L.b, k & 1 ? L.t : L.x, k & 1 ? L.x : L.t, om, S->s));
        if (sweeps & 1) HZB_TRY(vcopy(L.n, L.t, L.x, S->s));
        return SUCCESS;
    }
    case SMOOTHER_GS:
        for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 0, pre, w));
        return SUCCESS;
    case SMOOTHER_SGS:
        for (int k = 0; k < sweeps; ++k) {
            HZB_TRY(gs_sweep(S, L, 2, true, w));
            HZB_TRY(gs_sweep(S, L, 2 | GS_SKIP_LAST, false, w));
        }
        return SUCCESS;
    case SMOOTHER_SOR:
        for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, pre, w));
        return SUCCESS;
    case SMOOTHER_SSOR:
        for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, true, w));
        for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, false, w));
        return SUCCESS;
    case SMOOTHER_GSOR:
        if (pre) {
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 0, true, w));
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, false, w));
        } else {
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, true, w));
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 0, false, w));
        }
        return SUCCESS;
    case SMOOTHER_SGSOR:
        if (pre) {
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 0, true, w));
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 0, false, w));
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, true, w));
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, false, w));
        } else {
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, true, w));
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 1, false, w));
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 0, true, w));
            for (int k = 0; k < sweeps; ++k) HZB_TRY(gs_sweep(S, L, 0, false, w));
        }
        return SUCCESS;
    }
    set_error_msg("unsupported smoother type");
    return ERROR_AMG_SMOOTH_TYPE;
}

static bool smoother_needs_gs(int sm) {
    return sm == SMOOTHER_GS || sm == SMOOTHER_SGS || sm == SMOOTHER_SOR ||
           sm == SMOOTHER_SSOR || sm == SMOOTHER_GSOR || sm == SMOOTHER_SGSOR;
}

// ---------------------------------------------------------------------------
// V / W cycle, mgcycle (mgcycle.c:245-415)
// ---------------------------------------------------------------------------
int restrict_level(hzb_solver *S, int l, const double *w, double *bc) {
    const Level &L = S->lv[l];
    if (L.sa) return spmv<double>(L.R64(), SPMV_Y, w, nullptr, bc, 1.0, nullptr, S->s);
    return restrict_agg<double>(L.nc, L.ria, L.rja, w, bc, S->s);
}

int prolong_level(hzb_solver *S, int l, const double *xc, double *x, double alpha) {
    const Level &L = S->lv[l];
    if (L.sa) return spmv<double>(L.P64(), SPMV_AXPY, xc, nullptr, x, alpha, nullptr, S->s);
    return prolong_agg<double>(L.n, L.agg, xc, x, alpha, S->s);
}
int coarse_solve64(hzb_solver *S, const AMG_param &cyc, double ctol) {
    Level &C = S->lv[S->nl - 1];
    if (cyc.coarse_solver == SOLVER_UMFPACK && S->Ainv)
        return dense_gemv<double>(C.n, S->Ainv, C.b, C.x, S->s);
    // coarse_itsolver (mgcycle.c:34-52): plain CG to ctol with maxit 20 n,
    // and GMRES(30) from CG's last iterate when CG reports a failure
    if (S->kwc.n != C.n) HZB_TRY(S->kwc.alloc(C.n));
    double rel = 0.0;
    int it = pcg(S, C.A64(), C.b, C.x, PC_NONE, nullptr, ctol, 20 * C.n, STOP_REL_RES, 0,
                 S->kwc, &rel, nullptr);
    if (it < 0 && it != ERROR_SOLVER_MISC)
        it = gmres(S, C.A64(), C.b, C.x, PC_NONE, nullptr, ctol, 20 * C.n, 30, STOP_REL_RES,
                   0, false, &rel, S->nl - 1);
    return it == ERROR_SOLVER_MISC ? it : SUCCESS;
}

int coarse_alpha(hzb_solver *S, int c, const double *rc, double *alpha) {
    Level &C = S->lv[c];
    KrylovWork &w = S->kw;
    HZB_TRY(dot(C.n, C.x, rc, w.part, w.sc + SC_X, S->s));
    HZB_TRY(spmv<double>(C.A64(), SPMV_Y, C.x, nullptr, C.t, 1.0, nullptr, S->s));
    HZB_TRY(dot(C.n, C.x, C.t, w.part, w.sc + SC_X + 1, S->s));
    HZB_TRY(fetch(S, w));
    *alpha = std::min(w.h_sc[SC_X] / w.h_sc[SC_X + 1], 2.0);
    return SUCCESS;
}

// l0 > 0 runs the same cycle on the sub-hierarchy below level l0 (the
// coarse-grid operator B_c used by the learned-weight training).
int cycle64(hzb_solver *S, const AMG_param &cyc, int l0) {
    const int nl = S->nl;
    int num_lvl[MAX_AMG_LVL] = {0};
    int l = l0;
    double alpha = 1.0;
forward:
    while (l < nl - 1) {
        Level &L = S->lv[l];
        num_lvl[l]++;
        HZB_TRY(smooth64(S, l, true, cyc));
        HZB_TRY(spmv<double>(L.A64(), SPMV_RES, L.x, L.b, L.w, 1.0, nullptr, S->s));
        HZB_TRY(restrict_level(S, l, L.w, S->lv[l + 1].b));
        ++l;
        HZB_TRY(vzero<double>(S->lv[l].n, S->lv[l].x, S->s));
    }
    if (S->batch) HZB_TRY(batch_terminal_solve(S, nl - 1, false));
    else HZB_TRY(coarse_solve64(S, cyc, cyc.tol * 1e-2));
    while (l > l0) {
        --l;
        Level &L = S->lv[l];
        if (cyc.coarse_scaling == ON) HZB_TRY(coarse_alpha(S, l + 1, S->lv[l + 1].b, &alpha));
        HZB_TRY(prolong_level(S, l, S->lv[l + 1].x, L.x, alpha));
        HZB_TRY(smooth64(S, l, false, cyc));
        // batched systems whose coarsening ended here: their block exactly
        if (S->batch) HZB_TRY(batch_terminal_solve(S, l, false));
        if (num_lvl[l] < cyc.cycle_type) break;
        else num_lvl[l] = 0;
    }
    if (l > l0) goto forward;
    return SUCCESS;
}

// precond_amg (precond.c:164-184)
static int precond64_body(hzb_solver *S, const double *r, double *z,
                          const AMG_param &cyc) {
    Level &L0 = S->lv[0];
    double *sb = L0.b, *sx = L0.x;
    L0.b = const_cast<double *>(r);
    L0.x = z;
    int rc = vzero<double>(L0.n, z, S->s);
    for (int i = 0; rc == SUCCESS && i < cyc.maxit; ++i) rc = cycle64(S, cyc);
    L0.b = sb;
    L0.x = sx;
    return rc;
}

// ---------------------------------------------------------------------------
// FP32 cycle (mixed precision): same structure, single-precision vectors and
// matrix values, FP32 accumulation; the coarse solve reads the FP64 inverse.
// ---------------------------------------------------------------------------
// xzero: x32 holds zeros on entry (first visit of the level in this cycle);
// the first sweep then needs no matrix and nothing has to zero x32 first.
static int smooth32(hzb_solver *S, int l, bool pre, const AMG_param &cyc, bool xzero) {
    Level &L = S->lv[l];
    const int sweeps = pre ? cyc.presmooth_iter : cyc.postsmooth_iter;
    const DCsr<float> A = L.A32();
    switch (cyc.smoother) {
    case SMOOTHER_L1DIAG:
    case SMOOTHER_JACOBI: {
        const float *om = (l == 0 && S->omega_active) ? S->omega : nullptr;
        if (sweeps == 0) return xzero ? vzero<float>(L.n, L.x32, S->s) : SUCCESS;
        if (!xzero && (sweeps & 1)) {
            // odd count from a nonzero x: ping-pong, copy back at the end
            for (int k = 0; k < sweeps; ++k) {
                const bool fwd = (k & 1) == 0;
                HZB_TRY(l1_sweep<float>(A, L.b32, fwd ? L.x32 : L.t32, fwd ? L.t32 : L.x32,
                                        om, S->s));
            }
            return vcopy<float>(L.n, L.t32, L.x32, S->s);
        }
        // sweep j writes x32 when (sweeps-1-j) is even, t32 otherwise, so the
        // last one lands in x32 without a copy
        float *prev = L.x32;
        for (int j = 0; j < sweeps; ++j) {
            float *dst = ((sweeps - 1 - j) & 1) ? L.t32 : L.x32;
            if (j == 0 && xzero)
                HZB_TRY(l1_first_sweep<float>(L.n, L.b32, L.l1_32, dst, om, S->s, L.act));
            else
                HZB_TRY(l1_sweep<float>(A, L.b32, prev, dst, om, S->s));
            prev = dst;
        }
        return SUCCESS;
    }
    case SMOOTHER_GS: {
        const Schedule &sc = L.col;
        const int ns = (int)sc.h_ptr.size() - 1;
        if (xzero) HZB_TRY(vzero<float>(L.n, L.x32, S->s));
        for (int k = 0; k < sweeps; ++k)
            for (int q = 0; q < ns; ++q) {
                const int c = pre ? q : ns - 1 - q;
                HZB_TRY(gs_rows<float>(A, 0, sc.rows + sc.h_ptr[c],
                                       sc.h_ptr[c + 1] - sc.h_ptr[c], L.d_gs32, 1.0f,
                                       L.b32, L.x32, S->s));
            }
        return SUCCESS;
    }
    }
    set_error_msg("mixed precision supports the l1-Jacobi and multicolour GS smoothers");
    return ERROR_AMG_SMOOTH_TYPE;
}

// level0_zero: the caller left x32 of level 0 at zero
int cycle32(hzb_solver *S, const AMG_param &cyc, bool level0_zero) {
    const int nl = S->nl;
    int num_lvl[MAX_AMG_LVL] = {0};
    bool zero[MAX_AMG_LVL] = {false};
    zero[0] = level0_zero;
    int l = 0;
forward:
    while (l < nl - 1) {
        Level &L = S->lv[l];
        num_lvl[l]++;
        HZB_TRY(smooth32(S, l, true, cyc, zero[l]));
        zero[l] = false;
        HZB_TRY(spmv<float>(L.A32(), SPMV_RES, L.x32, L.b32, L.w32, 1.0f, nullptr, S->s));
        HZB_TRY(restrict_agg<float>(L.nc, L.ria, L.rja, L.w32, S->lv[l + 1].b32, S->s,
                                    S->lv[l + 1].act));
        ++l;
        if (l < nl - 1) zero[l] = true;   // x_l = 0, folded into its first sweep
    }
    if (S->batch) {
        HZB_TRY(batch_terminal_solve(S, nl - 1, true));
    } else {
        Level &C = S->lv[nl - 1];
        HZB_TRY(dense_gemv<float>(C.n, S->Ainv, C.b32, C.x32, S->s));
    }
    while (l > 0) {
        --l;
        Level &L = S->lv[l];
        HZB_TRY(prolong_agg<float>(L.n, L.agg, S->lv[l + 1].x32, L.x32, 1.0f, S->s, L.act));
        HZB_TRY(smooth32(S, l, false, cyc, false));
        // batched systems whose coarsening ended here: their block exactly
        if (S->batch) HZB_TRY(batch_terminal_solve(S, l, true));
        if (num_lvl[l] < cyc.cycle_type) break;
        else num_lvl[l] = 0;
    }
    if (l > 0) goto forward;
    return SUCCESS;
}

int ensure_fp32(hzb_solver *S) {
    // HZB_SETUP_TRACE=1: the stream synchronised after each part, and a level
    // whose parts took more than 20 ms reported to stderr
    static const bool trace = [] {
        const char *e = getenv("HZB_SETUP_TRACE");
        return e && e[0] == '1';
    }();
    using clk = std::chrono::steady_clock;
    auto lap = [&](clk::time_point &t) {
        if (!trace) return 0.0;
        cudaStreamSynchronize(S->s);
        const auto now = clk::now();
        const double ms = std::chrono::duration<double, std::milli>(now - t).count();
        t = now;
        return ms;
    };
    for (int l = 0; l < S->nl; ++l) {
        Level &L = S->lv[l];
        clk::time_point t = clk::now();
        double ms_count = 0, ms_copy = 0, ms_vec = 0, ms_norms = 0, ms_sell = 0, ms_sched = 0;
        lap(t);
        if (!L.val32) {
            // drop the stored exact zeros: they add nothing to a row sum
            int *cnt = nullptr, *ia32 = nullptr, *tmp = nullptr;
            HZB_TRY(dalloc(&cnt, L.n));
            HZB_TRY(dalloc(&ia32, L.n + 1));
            HZB_TRY(dalloc(&tmp, scan_tmp_size(L.n + 1)));
            HZB_TRY(csr_nonzero_count(L.n, L.ia, L.val, cnt, S->s));
            HZB_TRY(scan_exclusive(cnt, ia32, L.n, tmp, S->s));
            int nz = 0;
            HZB_CUDA(cudaMemcpyAsync(&nz, ia32 + L.n, sizeof(int), cudaMemcpyDeviceToHost, S->s));
            HZB_CUDA(cudaStreamSynchronize(S->s));
            ms_count = lap(t);
            dfree(cnt);
            dfree(tmp);
            if (nz == L.nnz) {   // nothing to drop: share the pattern
                dfree(ia32);
                HZB_TRY(dalloc(&L.val32, L.nnz));
                HZB_TRY(csr_val_d2f(L.nnz, L.val, L.val32, S->s));
                L.ia32 = L.ia;
                L.ja32 = L.ja;
                L.own32 = false;
            } else {
                L.ia32 = ia32;
                HZB_TRY(dalloc(&L.ja32, nz));
                HZB_TRY(dalloc(&L.val32, nz));
                HZB_TRY(csr_nonzero_fill(L.n, L.ia, L.ja, L.val, L.ia32, L.ja32, L.val32, S->s));
                L.own32 = true;
                if (l == 0 && !S->batch) {   // the outer loop's operator
                    HZB_TRY(dalloc(&L.val64nz, nz));
                    HZB_TRY(csr_nonzero_fill64(L.n, L.ia, L.val, L.ia32, L.val64nz, S->s));
                }
            }
            L.nnz32 = nz;
            HZB_TRY(bundle_capacity_rows(L.n, L.bundle_rows, L.ia32, S->s, &L.bundle_cap32));
        }
        ms_copy = lap(t);
        if (!L.b32) {
            HZB_TRY(dalloc(&L.b32, L.n));
            HZB_TRY(dalloc(&L.x32, L.n));
            HZB_TRY(dalloc(&L.w32, L.n));
            HZB_TRY(dalloc(&L.t32, L.n));
        }
        ms_vec = lap(t);
        if (!L.l1_32) {
            HZB_TRY(dalloc(&L.l1_32, L.n));
            HZB_TRY(l1_norms<float>(L.A32(), L.l1_32, S->s));
            ms_norms = lap(t);
            // staged bundles, lanes per row or the sliced-ELL copy, by
            // timing; HZB_FP32_LANES (0, 2, 4, 8, 16 or "sell") names one for
            // every level instead.  Batched solves run the kernels with an
            // activity array, which the sliced-ELL kernels do not take.
            const char *force = getenv("HZB_FP32_LANES");
            const bool force_sell = force && strcmp(force, "sell") == 0;
            const int fl = force && !force_sell ? atoi(force) : -1;
            const bool sell_ok = !S->batch && L.n >= 4096;
            if (force_sell && sell_ok) {
                HZB_TRY(sell_build(L.n, L.ia32, L.ja32, L.val32, &L.sell32, S->s));
                L.vec32 = SELL_LANES;
            } else if (fl == 0 || fl == 2 || fl == 4 || fl == 8 || fl == 16) {
                L.vec32 = fl;
            } else if (L.n >= 4096) {
                int known = 0;
                const bool have = fp32_schedule_known(L.n, L.nnz32, &known);
                if (sell_ok && (!have || known == SELL_LANES))
                    HZB_TRY(sell_build(L.n, L.ia32, L.ja32, L.val32, &L.sell32, S->s));
                ms_sell = lap(t);
                HZB_TRY(vzero<float>(L.n, L.b32, S->s));
                HZB_TRY(vzero<float>(L.n, L.x32, S->s));
                DCsr<float> A = L.A32();
                HZB_TRY(autotune_fp32(A, L.b32, L.x32, L.w32, S->s));
                L.vec32 = A.vec_lanes;
                if (L.vec32 != SELL_LANES) L.sell32.release();
            }
        }
        ms_sched = lap(t);
        if (trace && ms_count + ms_copy + ms_vec + ms_norms + ms_sell + ms_sched > 1.0)
            fprintf(stderr, "hzb setup trace: fp32 level %d (%d rows): count %.2f copy %.2f "
                    "vectors %.2f norms %.2f sell %.2f schedule %.2f ms\n", l, L.n, ms_count,
                    ms_copy, ms_vec, ms_norms, ms_sell, ms_sched);
        if (S->amg.smoother == SMOOTHER_GS && l < S->nl - 1 && !L.d_gs32) {
            if (!L.col.rows) HZB_TRY(multicolor(L.n, L.ia, L.ja, &L.col, S->s));
            HZB_TRY(dalloc(&L.d_gs32, L.n));
            HZB_TRY(d2f(L.n, L.d_gs_f, L.d_gs32, S->s));
        }
    }
    HZB_CUDA(cudaStreamSynchronize(S->s));
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// setup, amg_setup_unsmoothP_unsmoothR (amg_setup_ua.c:1228-1452)
// ---------------------------------------------------------------------------
int level_smoother_data(hzb_solver *S, Level &L) {
    const int sm = S->amg.smoother;
    const bool gsf = smoother_needs_gs(sm);
    if (sm == SMOOTHER_JACOBI || gsf || S->bp.precision == HZB_PREC_MIXED) {
        HZB_TRY(dalloc(&L.d_jac, L.n));
        HZB_TRY(dalloc(&L.d_gs_f, L.n));
        HZB_TRY(dalloc(&L.d_gs_b, L.n));
        HZB_TRY(dalloc(&L.d_sor_f, L.n));
        HZB_TRY(dalloc(&L.d_sor_b, L.n));
        HZB_TRY(smoother_diagonals(L.A64(), L.d_jac, L.d_gs_f, L.d_gs_b, L.d_sor_f,
                                   L.d_sor_b, S->s));
    }
    if (gsf) {
        if (S->bp.gs_schedule == HZB_GS_MULTICOLOR) {
            HZB_TRY(multicolor(L.n, L.ia, L.ja, &L.col, S->s));
        } else {
            HZB_TRY(gs_schedule(L.n, L.ia, L.ja, L.nnz, 0, &L.fwd, S->s));
            HZB_TRY(gs_schedule(L.n, L.ia, L.ja, L.nnz, 1, &L.bwd, S->s));
        }
    }
    return SUCCESS;
}

// HZB_SETUP_TRACE=1: each setup prints to stderr the host time of its phases
// (the stream synchronised at every mark) and how much the device's memory
// pool grew, for finding where a slow setup spent its time.
namespace {
struct SetupTrace {
    bool on = false;
    cudaStream_t s = nullptr;
    std::chrono::steady_clock::time_point t0, last;
    unsigned long long pool0 = 0;
    std::string line;
    static unsigned long long reserved() {
        int dev = 0;
        cudaMemPool_t pool;
        unsigned long long v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v);
        return v;
    }
    explicit SetupTrace(cudaStream_t st) : s(st) {
        const char *e = getenv("HZB_SETUP_TRACE");
        on = e && e[0] == '1';
        if (!on) return;
        cudaStreamSynchronize(s);
        t0 = last = std::chrono::steady_clock::now();
        pool0 = reserved();
    }
    void mark(const char *what) {
        if (!on) return;
        cudaStreamSynchronize(s);
        const auto t = std::chrono::steady_clock::now();
        char buf[96];
        snprintf(buf, sizeof(buf), " %s %.2f", what,
                 std::chrono::duration<double, std::milli>(t - last).count());
        line += buf;
        last = t;
    }
    ~SetupTrace() {
        if (!on) return;
        const double tot =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                .count();
        const long long grew = (long long)reserved() - (long long)pool0;
        fprintf(stderr, "hzb setup trace (ms):%s total %.2f pool_growth_MB %.1f\n", line.c_str(),
                tot, grew / 1048576.0);
    }
};
}  // namespace

int setup(hzb_solver *S, int n, int nnz, const int *d_ia, const int *d_ja,
          const double *d_val, bool copy_in) {
    SetupTrace trace(S->s);
    S->g64.release();
    S->g32.release();
    S->g32c.release();
    S->gcyc.release();
    gmres_release(S);
    gcg_release(S);
    for (auto &L : S->lv) L.release();
    S->lv.clear();
    dfree(S->Ainv);
    S->nl = 0;
    cudaStream_t s = S->s;
    trace.mark("release");
    HZB_CUDA(cudaEventRecord(S->e0, s));
    S->lv.emplace_back();
    {
        Level &L0 = S->lv[0];
        L0.n = n;
        L0.nnz = nnz;
        if (copy_in) {
            L0.own_A = true;
            HZB_TRY(dalloc(&L0.ia, n + 1));
            HZB_TRY(dalloc(&L0.ja, nnz));
            HZB_TRY(dalloc(&L0.val, nnz));
            HZB_CUDA(cudaMemcpyAsync(L0.ia, d_ia, sizeof(int) * (n + 1), cudaMemcpyDefault, s));
            HZB_CUDA(cudaMemcpyAsync(L0.ja, d_ja, sizeof(int) * nnz, cudaMemcpyDefault, s));
            HZB_CUDA(cudaMemcpyAsync(L0.val, d_val, sizeof(double) * nnz, cudaMemcpyDefault, s));
        } else {
            L0.own_A = false;
            L0.ia = const_cast<int *>(d_ia);
            L0.ja = const_cast<int *>(d_ja);
            L0.val = const_cast<double *>(d_val);
        }
        HZB_TRY(bundle_capacity(n, L0.ia, s, &L0.bundle_cap));
    }
    const short min_cdof = (short)std::max(S->amg.coarse_dof, 1);
    const int max_levels = std::min<int>(S->amg.max_levels, MAX_AMG_LVL);
    // smoothed aggregation (amg_setup_sa) for SA_AMG, else unsmoothed
    const bool sa = S->amg.AMG_type == SA_AMG;
    if (sa && S->bp.precision == HZB_PREC_MIXED) {
        set_error_msg("the mixed-precision cycle runs unsmoothed aggregation");
        return ERROR_INPUT_PAR;
    }
    int lvl = 0;
    int *tmp = nullptr;
    HZB_TRY(dalloc(&tmp, scan_tmp_size(n + 2)));
    int rc = SUCCESS;
    // batch mode: every system coarsens until its own terminal block (the
    // union's size does not decide), see batch_level_begin
    const bool batch = S->batch != nullptr;
    int batch_begun = -1;   // the last level batch_level_begin has seen
    while (lvl < max_levels - 1 && (batch || S->lv[lvl].n > min_cdof)) {
        if (batch) {
            int live = 0;
            batch_begun = lvl;
            if ((rc = batch_level_begin(S, lvl, false, &live))) break;
            if (live == 0) break;   // every system ends on this level
        }
        Level &L = S->lv[lvl];
        const int m = L.n;
        int *nia = nullptr, *nja = nullptr, *agg = nullptr, *work = nullptr;
        double *nval = nullptr;
        int nnnz = 0, nagg = 0;
        // aggregation_type: VMB in the reference's order; HEM exact, or the
        // deterministic parallel matching (hzb_param.matching, and for HEC,
        // whose reference order comes from an unseeded rand())
        const bool vmb = S->amg.aggregation_type == VMB;
        const bool par = !vmb && S->bp.matching == HZB_MATCH_PARALLEL;
        const bool hec = !vmb && !par && S->amg.aggregation_type == HEC;
        if ((rc = dalloc(&nia, m + 1)) || (rc = dalloc(&nja, L.nnz)) ||
            (rc = dalloc(&nval, L.nnz)) || (rc = dalloc(&agg, m)) ||
            (rc = dalloc(&work, par ? (size_t)6 * m + scan_tmp_size(m + 1) + 8
                                : hec ? hec_work_ints(m)
                                      : (size_t)(vmb ? 2 : 1) * m))) {
            dfree(nia); dfree(nja); dfree(nval); dfree(agg); dfree(work);
            break;
        }
        // HEC draws from rand() as a fresh process does: seeded 1 per setup
        if (hec && lvl == 0) {
            if (!S->hec_state) rc = dalloc(&S->hec_state, 35);
            if (!rc) rc = hec_seed(S->hec_state, 1u, s);
        }
        if (!rc) rc = strength_graph(L.A64(), S->amg.strong_coupled, nia, nja, nval, &nnnz,
                                     tmp, s);
        if (!rc) {
            if (vmb) rc = vmb_aggregate(m, nia, nja, S->amg.max_aggregation, agg, &nagg, work, s);
            else if (par) rc = hem_parallel(m, nia, nja, nval, agg, &nagg, work, s);
            else if (hec) rc = hec_aggregate(m, nia, nja, nval, agg, &nagg, S->hec_state, work, s);
            else rc = hem_exact(m, nia, nja, nval, agg, &nagg, work, s);
        }
        dfree(work);
        // smoothed aggregation still needs the strength graph (or A's copy)
        if (!rc && sa && S->amg.smooth_filter != ON) {
            dfree(nia); dfree(nja); dfree(nval);
            if (!(rc = dalloc(&nval, L.nnz)))
                rc = cudaMemcpyAsync(nval, L.val, sizeof(double) * L.nnz,
                                     cudaMemcpyDeviceToDevice, s) == cudaSuccess
                         ? SUCCESS : ERROR_SOLVER_MISC;
        }
        if (!sa || rc) { dfree(nia); dfree(nja); dfree(nval); }
        if (rc) { dfree(agg); dfree(nval); break; }
        // adaptive threshold (amg_setup_ua.c:1325-1328), caller's param too
        if (nagg * 4 > m) S->amg.strong_coupled /= 2;
        else if (nagg * 1.25 < m) S->amg.strong_coupled *= 2;
        if (S->caller_amg) S->caller_amg->strong_coupled = S->amg.strong_coupled;
        if (batch && (rc = batch_level_end(S, lvl, agg, &nagg))) {
            dfree(agg);
            break;
        }
        if (batch ? nagg == 0 : nagg < MIN_CDOF) {
            dfree(agg);
            if (sa) { dfree(nia); dfree(nja); dfree(nval); }
            break;
        }
        L.nc = nagg;
        L.agg = agg;
        int *cia = nullptr, *cja = nullptr, cnnz = 0;
        double *cval = nullptr;
        if (sa) {
            // smooth_aggregation_p, dcsr_trans, dcsr_rap (amg_setup_ua.c:1600-1624)
            const bool filter = S->amg.smooth_filter == ON;
            rc = sa_prolongation(L.A64(), filter ? nia : L.ia, filter ? nja : L.ja, nval, nagg,
                                 agg, S->amg.tentative_smooth, filter, &L.pia, &L.pja, &L.pval,
                                 &L.pnnz, s);
            dfree(nia); dfree(nja); dfree(nval);
            L.sa = true;
            if (rc) break;
            if ((rc = transpose_rect(m, nagg, L.pnnz, L.pia, L.pja, L.pval, &L.ria, &L.rja,
                                     &L.rval, s)))
                break;
            if ((rc = bundle_capacity(m, L.pia, s, &L.pcap)) ||
                (rc = bundle_capacity(nagg, L.ria, s, &L.rcap)))
                break;
            if ((rc = rap_general(nagg, L.ria, L.rja, L.rval, L.A64(), L.pia, L.pja, L.pval,
                                  &cia, &cja, &cval, &cnnz, s)))
                break;
        } else {
            if ((rc = dalloc(&L.ria, nagg + 1)) || (rc = dalloc(&L.rja, m))) break;
            if ((rc = restriction_pattern(m, nagg, agg, L.ria, L.rja, tmp, s))) break;
            if ((rc = rap_agg(L.A64(), nagg, agg, L.ria, L.rja, &cia, &cja, &cval, &cnnz, s)))
                break;
        }
        S->lv.emplace_back();
        Level &C = S->lv.back();
        C.n = nagg; C.nnz = cnnz; C.ia = cia; C.ja = cja; C.val = cval; C.own_A = true;
        if ((rc = bundle_capacity(C.n, C.ia, s, &C.bundle_cap))) break;
        ++lvl;
    }
    dfree(tmp);
    if (rc) return rc;
    S->nl = lvl + 1;
    if (batch && batch_begun != lvl) {
        // systems still coarsening when the level cap ends the loop end there
        int live = 0;
        HZB_TRY(batch_level_begin(S, lvl, true, &live));
    }
    trace.mark("levels");
    // coarsest level: dense inverse (coarse_solver 32, and always for the
    // FP32 cycle); batched systems use their terminal blocks instead
    if (!batch &&
        (S->amg.coarse_solver == SOLVER_UMFPACK || S->bp.precision == HZB_PREC_MIXED)) {
        // amg_setup_ua.c:1392-1401: the coarsest matrix is transposed (columns
        // ascending) and that transpose is factored
        Level &C = S->lv[S->nl - 1];
        HZB_TRY(transpose_csr(C.A64(), &C.tia, &C.tja, &C.tval, s));
        HZB_TRY(dense_inverse(C.AT64(), &S->Ainv, s));
    }
    trace.mark("coarse");
    for (int l = 0; l < S->nl; ++l) {
        Level &L = S->lv[l];
        HZB_TRY(dalloc(&L.b, L.n));
        HZB_TRY(dalloc(&L.x, L.n));
        HZB_TRY(dalloc(&L.w, L.n));
        HZB_TRY(dalloc(&L.t, L.n));
        if (l < S->nl - 1) HZB_TRY(level_smoother_data(S, L));
        if (L.n >= 32768) {   // large levels: time the bundle sizes once
            HZB_TRY(vzero<double>(L.n, L.x, s));
            DCsr<double> A = L.A64();
            HZB_TRY(autotune_bundle(A, L.x, L.w, s));
            L.bundle_rows = A.bundle_rows;
            L.bundle_cap = A.bundle_cap;
        }
    }
    trace.mark("smoothers");
    HZB_TRY(S->kw.alloc(n, s));
    if (S->amg.coarse_solver != SOLVER_UMFPACK)
        HZB_TRY(S->kwc.alloc(S->lv[S->nl - 1].n, s));
    if (S->bp.precision == HZB_PREC_MIXED) HZB_TRY(ensure_fp32(S));
    trace.mark("fp32");
    HZB_CUDA(cudaEventRecord(S->e1, s));
    HZB_CUDA(cudaEventSynchronize(S->e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, S->e0, S->e1);
    S->st.setup_seconds = ms * 1e-3;
    S->st.num_levels = S->nl;
    for (int l = 0; l < S->nl && l < MAX_AMG_LVL; ++l) {
        S->st.rows[l] = S->lv[l].n;
        S->st.nnz[l] = S->lv[l].nnz;
    }
    S->st.strong_coupled = S->amg.strong_coupled;
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// condition estimate of dcsr_pcg_w_cond_est (krylov.c:400-740): extreme
// eigenvalues of the Lanczos tridiagonal built from alpha/beta, here by
// Sturm-sequence bisection instead of LAPACK dsterf.
// ---------------------------------------------------------------------------
static int sturm_count(const std::vector<double> &d, const std::vector<double> &e,
                       double x) {
    int cnt = 0;
    double q = d[0] - x;
    if (q < 0) ++cnt;
    for (size_t i = 1; i < d.size(); ++i) {
        double qq = (q == 0.0) ? 1e-300 : q;
        q = d[i] - x - e[i - 1] * e[i - 1] / qq;
        if (q < 0) ++cnt;
    }
    return cnt;
}
static double tri_eig(const std::vector<double> &d, const std::vector<double> &e,
                      int k) {
    double lo = d[0], hi = d[0];
    for (size_t i = 0; i < d.size(); ++i) {
        double r = (i > 0 ? fabs(e[i - 1]) : 0) + (i + 1 < d.size() ? fabs(e[i]) : 0);
        lo = std::min(lo, d[i] - r);
        hi = std::max(hi, d[i] + r);
    }
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (sturm_count(d, e, mid) > k) hi = mid; else lo = mid;
    }
    return 0.5 * (lo + hi);
}
static double cond_estimate(const std::vector<double> &al,
                            const std::vector<double> &be, int m) {
    if (m < 1) return 0.0;
    std::vector<double> d(m), e(m > 1 ? m - 1 : 0);
    d[0] = 1.0 / al[0];
    for (int i = 0; i < m - 1; ++i) {
        d[i + 1] = 1.0 / al[i + 1] + be[i] / al[i];
        e[i] = sqrt(be[i]) / al[i];
    }
    if (m == 1) return 1.0;
    const double lmin = tri_eig(d, e, 0), lmax = tri_eig(d, e, m - 1);
    return lmax / lmin;
}

// ---------------------------------------------------------------------------
// PCG, dcsr_pcg (krylov.c:122-398)
// ---------------------------------------------------------------------------
static void print_info(int prt, int stop_type, int iter, double rel, double abs,
                       double factor) {
    if (prt < PRINT_SOME) return;
    if (iter > 0) {
        printf("%6lld | %13.6e   | %13.6e  | %10.4f\n", (long long)iter, rel, abs, factor);
    } else {
        printf("-----------------------------------------------------------\n");
        if (stop_type == STOP_REL_RES)
            printf("It Num |   ||r||/||b||   |     ||r||      |  Conv. Factor\n");
        else if (stop_type == STOP_REL_PRECRES)
            printf("It Num | ||r||_B/||b||_B |    ||r||_B     |  Conv. Factor\n");
        else
            printf("It Num |   ||r||/||x||   |     ||r||      |  Conv. Factor\n");
        printf("-----------------------------------------------------------\n");
        printf("%6lld | %13.6e   | %13.6e  |     -.-- \n", (long long)iter, rel, abs);
    }
    fflush(stdout);
}

int pc_kind_of_cycle(int cycle_type) {
    switch (cycle_type) {
    case AMLI_CYCLE: return PC_AMLI;
    case NL_AMLI_CYCLE: return PC_NLAMLI;
    case ADD_CYCLE: return PC_ADD;
    default: return PC_AMG;
    }
}

static int precond_alt(hzb_solver *S, int kind, const double *r, double *z);

static int apply_pc(hzb_solver *S, int kind, HostPrecond *hp, int n,
                    const double *r, double *z) {
    if (kind == PC_AMG) return precond64(S, r, z, S->pc_cyc);
    if (kind == PC_AMLI || kind == PC_ADD) return precond_alt(S, kind, r, z);
    if (kind == PC_BSR) return bsr_precond(S, r, z);
    if (kind >= PC_NLAMLI) {
        // the solve's preconditioner runs maxit cycles; the coarse-level
        // Krylov solves of the cycle itself run one (mgcycle.c:623)
        const int l = kind - PC_NLAMLI;
        return precond_cycles(S, PC_NLAMLI, l, l == 0 ? S->pc_cyc.maxit : 1, r, z, S->pc_cyc);
    }
    if (kind == PC_HOST) {
        HZB_CUDA(cudaMemcpyAsync(hp->h_r, r, sizeof(double) * n, cudaMemcpyDeviceToHost, S->s));
        HZB_CUDA(cudaStreamSynchronize(S->s));
        hp->fct(hp->h_r, hp->h_z, hp->data);
        HZB_CUDA(cudaMemcpyAsync(z, hp->h_z, sizeof(double) * n, cudaMemcpyHostToDevice, S->s));
        return SUCCESS;
    }
    return vcopy<double>(n, r, z, S->s);
}

int apply_precond(hzb_solver *S, int kind, HostPrecond *hp, int n, const double *r,
                  double *z) {
    return apply_pc(S, kind, hp, n, r, z);
}

// residual measure for the stopping type (krylov.c:157-170, 211-227)
static int measure(hzb_solver *S, KrylovWork &w, int kind, HostPrecond *hp,
                   int stop_type, double *absres) {
    const int n = w.n;
    if (stop_type == STOP_REL_PRECRES) {
        HZB_TRY(apply_pc(S, kind, hp, n, w.r, w.z));
        HZB_TRY(dot(n, w.z, w.r, w.part, w.sc + SC_X, S->s));
        HZB_TRY(fetch(S, w));
        *absres = sqrt(fabs(w.h_sc[SC_X]));
    } else {
        HZB_TRY(norm2sq(S, w, n, w.r, SC_X));
        HZB_TRY(fetch(S, w));
        *absres = sqrt(w.h_sc[SC_X]);
    }
    return SUCCESS;
}

int pcg(hzb_solver *S, const DCsr<double> &A, const double *b, double *u,
        int kind, HostPrecond *hp, double tol, int MaxIt, int stop_type,
        int prtlvl, KrylovWork &w, double *relres_out, double *condest) {
    const int MaxStag = MAX_STAG, MaxRestartStep = MAX_RESTART;
    const int m = A.n;
    const double maxdiff = tol * STAG_RATIO;
    const double sol_inf_tol = SMALLREAL;
    cudaStream_t s = S->s;
    int iter = 0, stag = 1, more_step = 1, restart_step = 1;
    double absres0 = BIGREAL, absres = BIGREAL, relres = BIGREAL;
    double normu = BIGREAL, normr0 = BIGREAL;
    double reldiff, factor, infnormu, alpha, temp1 = 0.0, temp2;
    std::vector<double> al, be;
    int iter_condest = 0;
    const int G = reduce_blocks(m);
    double *part4 = w.part, *partd = w.part + 4 * G;
    if (w.n != m) HZB_TRY(w.alloc(m));

    // r = b - A u ; z = B r
    HZB_TRY(spmv<double>(A, SPMV_RES, u, b, w.r, 1.0, nullptr, s));
    HZB_TRY(apply_pc(S, kind, hp, m, w.r, w.z));
    switch (stop_type) {
    case STOP_REL_RES:
        HZB_TRY(measure(S, w, kind, hp, STOP_REL_RES, &absres0));
        normr0 = std::max(SMALLREAL, absres0);
        relres = absres0 / normr0;
        break;
    case STOP_REL_PRECRES:
        HZB_TRY(dot(m, w.r, w.z, w.part, w.sc + SC_X, s));
        HZB_TRY(fetch(S, w));
        absres0 = sqrt(w.h_sc[SC_X]);
        normr0 = std::max(SMALLREAL, absres0);
        relres = absres0 / normr0;
        break;
    case STOP_MOD_REL_RES:
        HZB_TRY(measure(S, w, kind, hp, STOP_REL_RES, &absres0));
        HZB_TRY(norm2sq(S, w, m, u, SC_X));
        HZB_TRY(fetch(S, w));
        normu = std::max(SMALLREAL, sqrt(w.h_sc[SC_X]));
        relres = absres0 / normu;
        break;
    default:
        printf("### ERROR: Unrecognised stopping type for %s!\n", __FUNCTION__);
        goto finished;
    }
    if (relres < tol || absres0 < 1e-3 * tol) goto finished;
    print_info(prtlvl, stop_type, iter, relres, absres0, 0.0);

    HZB_TRY(vcopy<double>(m, w.z, w.p, s));
    HZB_TRY(dot(m, w.z, w.r, w.part, w.sc + SC_T1, s));

    while (iter++ < MaxIt) {
        // t = A p ; temp2 = (t, p) ; alpha = temp1 / temp2 (device)
        HZB_TRY(spmv<double>(A, SPMV_Y_DOT, w.p, nullptr, w.t, 1.0, partd, s));
        HZB_TRY(reduce_final(partd, spmv_blocks_rows(m, A.bundle_rows), w.sc + SC_T2, s));
        // u += alpha p ; r -= alpha t ; norms for checks I and II
        HZB_TRY(pcg_update(m, w.sc + SC_T1, w.sc + SC_T2, u, w.r, w.p, w.t, part4, s));
        HZB_TRY(reduce_final(part4, G, w.sc + SC_RR, s));
        HZB_TRY(reduce_final_max(part4 + G, G, w.sc + SC_UM, s));
        HZB_TRY(reduce_final(part4 + 2 * G, G, w.sc + SC_UU, s));
        HZB_TRY(reduce_final(part4 + 3 * G, G, w.sc + SC_PP, s));
        HZB_TRY(fetch(S, w));
        if (condest && iter > 1) be.push_back(w.h_sc[SC_T1] / temp1);   // beta_{k-1}
        temp1 = w.h_sc[SC_T1];
        temp2 = w.h_sc[SC_T2];
        alpha = temp1 / temp2;
        if (condest) al.push_back(alpha);
        switch (stop_type) {
        case STOP_REL_RES:
            absres = sqrt(w.h_sc[SC_RR]);
            relres = absres / normr0;
            break;
        case STOP_REL_PRECRES:
            HZB_TRY(measure(S, w, kind, hp, STOP_REL_PRECRES, &absres));
            relres = absres / normr0;
            break;
        case STOP_MOD_REL_RES:
            absres = sqrt(w.h_sc[SC_RR]);
            relres = absres / normu;
            break;
        }
        factor = absres / absres0;
        print_info(prtlvl, stop_type, iter, relres, absres, factor);

        // Check I: solution close to zero
        infnormu = w.h_sc[SC_UM];
        if (infnormu <= sol_inf_tol) {
            if (prtlvl > PRINT_MIN)
                printf("### HAZMATH WARNING: Iteration stopped due to the solution is almost zero! %s : %lld\n",
                       __FUNCTION__, (long long)__LINE__);
            iter = ERROR_SOLVER_SOLSTAG;
            break;
        }
        // Check II: stagnation
        normu = sqrt(w.h_sc[SC_UU]);
        reldiff = fabs(alpha) * sqrt(w.h_sc[SC_PP]) / normu;
        if ((stag <= MaxStag) & (reldiff < maxdiff)) {
            if (prtlvl >= PRINT_MORE) {
                printf("||u-u'|| = %e and the comp. rel. res. = %e.\n", reldiff, relres);
                printf("### HAZMATH WARNING: Iteration restarted due to stagnation! %s : %lld\n",
                       __FUNCTION__, (long long)__LINE__);
            }
            if (stag == 1 && restart_step == 1) iter_condest = iter;
            HZB_TRY(spmv<double>(A, SPMV_RES, u, b, w.r, 1.0, nullptr, s));
            HZB_TRY(measure(S, w, kind, hp, stop_type == STOP_REL_PRECRES ? STOP_REL_PRECRES : STOP_REL_RES, &absres));
            relres = absres / (stop_type == STOP_MOD_REL_RES ? normu : normr0);
            if (prtlvl >= PRINT_MORE)
                printf("### HAZMATH WARNING: The actual relative residual = %e!\n", relres);
            if (relres < tol) break;
            if (stag >= MaxStag) {
                if (prtlvl > PRINT_MIN)
                    printf("### HAZMATH WARNING: Iteration stopped due to staggnation! %s : %lld\n",
                           __FUNCTION__, (long long)__LINE__);
                iter = ERROR_SOLVER_STAG;
                break;
            }
            HZB_TRY(vzero<double>(m, w.p, s));
            ++stag;
            ++restart_step;
        }
        // Check III: false convergence
        if (relres < tol) {
            const double computed = relres;
            if (stag == 1 && restart_step == 1) iter_condest = iter;
            HZB_TRY(spmv<double>(A, SPMV_RES, u, b, w.r, 1.0, nullptr, s));
            HZB_TRY(measure(S, w, kind, hp, stop_type == STOP_REL_PRECRES ? STOP_REL_PRECRES : STOP_REL_RES, &absres));
            relres = absres / (stop_type == STOP_MOD_REL_RES ? normu : normr0);
            if (relres < tol) break;
            if (prtlvl >= PRINT_MORE) {
                printf("### HAZMATH WARNING: The computed relative residual = %e!\n", computed);
                printf("### HAZMATH WARNING: The actual relative residual = %e!\n", relres);
            }
            if (more_step >= MaxRestartStep) {
                if (prtlvl > PRINT_MIN)
                    printf("### HAZMATH WARNING: The tolerence might be too small! %s : %lld\n",
                           __FUNCTION__, (long long)__LINE__);
                iter = ERROR_SOLVER_TOLSMALL;
                break;
            }
            HZB_TRY(vzero<double>(m, w.p, s));
            ++more_step;
            ++restart_step;
        }
        absres0 = absres;
        if (stop_type != STOP_REL_PRECRES) HZB_TRY(apply_pc(S, kind, hp, m, w.r, w.z));
        // beta = (z, r)_new / temp1 ; p = z + beta p ; temp1 = (z, r)_new
        HZB_TRY(dot(m, w.z, w.r, w.part, w.sc + SC_T3, s));
        HZB_TRY(pcg_axpby(m, w.sc + SC_T3, w.sc + SC_T1, w.z, w.p, s));
        k_copy_scalar<<<1, 1, 0, s>>>(w.sc + SC_T3, w.sc + SC_T1);
        count_launch();
    }
finished:
    if (prtlvl > PRINT_NONE) {
        if (iter > MaxIt)
            printf("### HAZMATH WARNING: Max iter %lld reached with rel. resid. %e.\n",
                   (long long)MaxIt, relres);
        else if (iter >= 0)
            printf("Num_iter(krylov.c) = %lld with relative residual %e.\n",
                   (long long)iter, relres);
        fflush(stdout);
    }
    if (relres_out) *relres_out = relres;
    if (condest) {
        if (stag == 1 && restart_step == 1) iter_condest = std::max(0, std::min(iter, MaxIt));
        const int mm = std::min<int>(iter_condest, (int)al.size());
        *condest = cond_estimate(al, be, std::min<int>(mm, (int)be.size() + 1));
    }
    if (iter > MaxIt) return ERROR_SOLVER_MAXIT;
    return iter;
}

// ---------------------------------------------------------------------------
// flexible CG with the FP32 cycle (mixed precision; no reference counterpart
// beyond dcsr_pgcg's flexible idea, krylov.c:2309)
// ---------------------------------------------------------------------------
static int apply_pc32_body(hzb_solver *S, const double *r, double *z) {
    Level &L0 = S->lv[0];
    AMG_param cyc = S->amg;
    HZB_TRY(d2f(L0.n, r, L0.b32, S->s));
    for (int i = 0; i < std::max<int>(1, cyc.maxit); ++i) HZB_TRY(cycle32(S, cyc, i == 0));
    return f2d(L0.n, L0.x32, z, S->s);
}

// Replays `body` from a CUDA graph captured on the solver's stream; the
// capture is redone whenever the key (vector pointers, tag) changes.
template <typename F>
static int with_graph(hzb_solver *S, GraphCache &G, const void *k0, const void *k1,
                      long long tag, F body, long long tag2 = 0) {
    if (!S->bp.use_graph) return body();
    if (!G.exec || G.k0 != k0 || G.k1 != k1 || G.tag != tag || G.tag2 != tag2) {
        G.release();
        const long long before = launch_count();
        HZB_CUDA(cudaStreamBeginCapture(S->s, cudaStreamCaptureModeThreadLocal));
        int rc = body();
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(S->s, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) set_error(e, __FILE__, __LINE__);
            return rc ? rc : ERROR_SOLVER_MISC;
        }
        e = cudaGraphInstantiate(&G.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            G.exec = nullptr;
            set_error(e, __FILE__, __LINE__);
            return ERROR_SOLVER_MISC;
        }
        G.k0 = k0;
        G.k1 = k1;
        G.tag = tag;
        G.tag2 = tag2;
        G.kernels = launch_count() - before;   // counted once by the capture
    } else {
        count_launch((int)G.kernels);
    }
    HZB_CUDA(cudaGraphLaunch(G.exec, S->s));
    return SUCCESS;
}

static long long cycle_tag(const hzb_solver *S, const AMG_param &c) {
    return (long long)c.maxit | ((long long)c.cycle_type << 8) |
           ((long long)c.smoother << 12) | ((long long)c.presmooth_iter << 20) |
           ((long long)c.postsmooth_iter << 26) | ((long long)S->omega_active << 32) |
           ((long long)c.coarse_solver << 34) | ((long long)(c.relaxation * 1e6) << 42);
}

static int apply_pc32(hzb_solver *S, const double *r, double *z) {
    return with_graph(S, S->g32, r, z, cycle_tag(S, S->amg),
                      [&]() { return apply_pc32_body(S, r, z); });
}

// the FP32 cycles alone: level 0's b32 is already the residual, the result
// stays in level 0's x32
static int cycles32(hzb_solver *S) {
    Level &L0 = S->lv[0];
    return with_graph(S, S->g32c, L0.b32, L0.x32, cycle_tag(S, S->amg), [&]() {
        AMG_param cyc = S->amg;
        for (int i = 0; i < std::max<int>(1, cyc.maxit); ++i) HZB_TRY(cycle32(S, cyc, i == 0));
        return SUCCESS;
    });
}

// The FP64 preconditioner is replayed from a graph unless a branch of the
// cycle reads a device value on the host (coarse scaling, coarse CG).
int precond64(hzb_solver *S, const double *r, double *z, const AMG_param &cyc) {
    const bool capturable = cyc.coarse_solver == SOLVER_UMFPACK && S->Ainv &&
                            cyc.coarse_scaling != ON;
    if (!capturable) return precond64_body(S, r, z, cyc);
    return with_graph(S, S->g64, r, z, cycle_tag(S, cyc),
                      [&]() { return precond64_body(S, r, z, cyc); });
}

// precond_amli / precond_amg_add: replayed from a graph under the same
// conditions as precond_amg; the key holds the AMLI coefficients' bits.
static int precond_alt(hzb_solver *S, int kind, const double *r, double *z) {
    const AMG_param &cyc = S->pc_cyc;
    const bool capturable = cyc.coarse_solver == SOLVER_UMFPACK && S->Ainv &&
                            cyc.coarse_scaling != ON;
    HZB_TRY(cycles_prepare(S, kind, cyc));
    auto body = [&]() { return precond_cycles(S, kind, 0, cyc.maxit, r, z, cyc); };
    if (!capturable) return body();
    unsigned long long h = 1469598103934665603ull ^ (unsigned long long)kind;
    if (kind == PC_AMLI) {
        for (double c : S->amli_coef) {
            unsigned long long u;
            memcpy(&u, &c, sizeof(u));
            h = (h ^ u) * 1099511628211ull;
        }
    }
    return with_graph(S, S->gcyc, r, z, cycle_tag(S, cyc), body, (long long)(h >> 1));
}

int solver_precond(hzb_solver *S, const double *r, double *z) {
    if (S->bp.precision == HZB_PREC_MIXED) return apply_pc32(S, r, z);
    return apply_pc(S, pc_kind_of_cycle(S->pc_cyc.cycle_type), nullptr, S->lv[0].n, r, z);
}

int fcg_mixed(hzb_solver *S, const double *b, double *x, double tol, int maxit,
              int prtlvl, double *relres_out) {
    KrylovWork &w = S->kw;
    const DCsr<double> A = S->lv[0].A64outer();
    const int m = A.n;
    cudaStream_t s = S->s;
    const int G = reduce_blocks(m);
    double *part4 = w.part, *partd = w.part + 4 * G;
    double normr0, relres, absres, absres0;
    int iter = 0;
    HZB_TRY(spmv<double>(A, SPMV_RES, x, b, w.r, 1.0, nullptr, s));
    HZB_TRY(norm2sq(S, w, m, w.r, SC_X));
    HZB_TRY(fetch(S, w));
    absres0 = sqrt(w.h_sc[SC_X]);
    normr0 = std::max(SMALLREAL, absres0);
    relres = absres0 / normr0;
    if (relres < tol || absres0 < 1e-3 * tol) {
        if (relres_out) *relres_out = relres;
        return 0;
    }
    print_info(prtlvl, STOP_REL_RES, 0, relres, absres0, 0.0);
    HZB_TRY(apply_pc32(S, w.r, w.z));
    HZB_TRY(vcopy<double>(m, w.z, w.p, s));
    HZB_TRY(dot(m, w.z, w.r, w.part, w.sc + SC_T1, s));
    // the update writes the cycle's FP32 residual, and the cycle's FP32 output
    // feeds the inner products and the new direction directly: z is never
    // stored in FP64 (the values are the same as through d2f / f2d)
    Level &L0 = S->lv[0];
    while (iter++ < maxit) {
        HZB_TRY(spmv<double>(A, SPMV_Y_DOT, w.p, nullptr, w.t, 1.0, partd, s));
        HZB_TRY(reduce_final(partd, spmv_blocks_rows(m, A.bundle_rows), w.sc + SC_T2, s));
        k_fcg_update<<<G, 256, 0, s>>>(m, w.sc + SC_T1, w.sc + SC_T2, x, w.r, w.p, w.t,
                                        L0.b32, part4);
        count_launch();
        HZB_TRY(reduce_final(part4, G, w.sc + SC_RR, s));
        HZB_TRY(fetch(S, w));
        absres = sqrt(w.h_sc[SC_RR]);
        relres = absres / normr0;
        print_info(prtlvl, STOP_REL_RES, iter, relres, absres, absres / absres0);
        absres0 = absres;
        if (relres < tol) {
            // recompute the true FP64 residual before accepting
            HZB_TRY(spmv<double>(A, SPMV_RES, x, b, w.r, 1.0, nullptr, s));
            HZB_TRY(norm2sq(S, w, m, w.r, SC_X));
            HZB_TRY(fetch(S, w));
            relres = sqrt(w.h_sc[SC_X]) / normr0;
            if (relres < tol) break;
            HZB_TRY(d2f(m, w.r, L0.b32, s));   // the cycle starts from the true residual
        }
        HZB_TRY(cycles32(S));
        k_dot2_partial_f<<<G, 256, 0, s>>>(m, L0.x32, w.t, w.r, part4);
        count_launch();
        HZB_TRY(reduce_final(part4, G, w.sc + SC_ZT, s));
        HZB_TRY(reduce_final(part4 + G, G, w.sc + SC_T3, s));
        k_fcg_p_f<<<grid_for(m), 256, 0, s>>>(m, w.sc + SC_ZT, w.sc + SC_T2, L0.x32, w.p);
        k_copy_scalar<<<1, 1, 0, s>>>(w.sc + SC_T3, w.sc + SC_T1);
        count_launch(2);
        HZB_LAUNCH_CHECK();
    }
    if (prtlvl > PRINT_NONE) {
        printf("Num_iter(fcg) = %lld with relative residual %e.\n", (long long)iter, relres);
        fflush(stdout);
    }
    if (relres_out) *relres_out = relres;
    return iter > maxit ? ERROR_SOLVER_MAXIT : iter;
}

void destroy(hzb_solver *S) {
    batch_release(S);
    bsr_release(S);
    S->g64.release();
    S->g32.release();
    S->g32c.release();
    S->gcyc.release();
    gmres_release(S);
    gcg_release(S);
    for (auto &L : S->lv) L.release();
    S->lv.clear();
    dfree(S->Ainv);
    dfree(S->omega);
    dfree(S->hec_state);
    dfree(S->pr);
    dfree(S->pz);
    S->kw.release();
    S->kwc.release();
}

}  // namespace hzb
