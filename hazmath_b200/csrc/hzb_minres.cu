// hzb_minres.cu -- preconditioned MINRES, dcsr_pminres (krylov.c:2449-2840),
// Krylov type 2 of solver_dcsr_linear_itsolver (itsolver.c:170-177).
//
// The reference's three-term recurrence with B-normalised directions: per
// step u += alpha p1, r -= alpha A p1 with alpha = (r, z1), the next
// direction p2 = z1 - (z1, A z1) p1 - (z1, A z0) p0 normalised by
// sqrt|(B A p2, A p2)|, and the same three safety checks as its CG (solution
// near zero, stagnation restart, false convergence).  All vectors stay on the
// device; the copies of the recurrence (p0 <- p1 <- p2, t0 <- t1, z0 <- z1)
// are pointer rotations, and the scalar updates read their coefficients
// from device memory.  The host reads the scalars twice per step: the
// normalisation (for the breakdown test) and the norms of the checks.
// Per-element arithmetic is the reference's (y + a*x, 0 + s*x), compiled
// without FMA contraction; inner products are fixed-order tree reductions.
#include "hzb_solver.cuh"
#include <cmath>
#include <cstdio>
#include <utility>

namespace hzb {

namespace {
// device scalar slots
enum { MR_ALPHA = 0, MR_A1 = 1, MR_A0 = 2, MR_NP = 3, MR_RR = 4, MR_UM = 5, MR_UU = 6,
       MR_PP = 7, MR_RB = 8, MR_N = 16 };

struct MinresWork {
    int n = 0;
    double *p0 = nullptr, *p1 = nullptr, *p2 = nullptr, *z0 = nullptr, *z1 = nullptr;
    double *t0 = nullptr, *t1 = nullptr, *t = nullptr, *tp = nullptr, *tz = nullptr,
           *r = nullptr;
    double *part = nullptr, *sc = nullptr, *h = nullptr;
    int alloc(int nn) {
        n = nn;
        for (double **v : {&p0, &p1, &p2, &z0, &z1, &t0, &t1, &t, &tp, &tz, &r})
            HZB_TRY(dalloc(v, n));
        HZB_TRY(dalloc(&part, 4 * reduce_blocks(n) + 8));
        HZB_TRY(dalloc(&sc, MR_N));
        HZB_CUDA(cudaMallocHost((void **)&h, MR_N * sizeof(double)));
        return SUCCESS;
    }
    ~MinresWork() {
        for (double **v : {&p0, &p1, &p2, &z0, &z1, &t0, &t1, &t, &tp, &tz, &r}) dfree(*v);
        dfree(part);
        dfree(sc);
        if (h) cudaFreeHost(h);
    }
};

// u += alpha p1; r += (-alpha) t1 with alpha = sc[MR_ALPHA]
__global__ void k_mr_step(int n, const double *__restrict__ sc, const double *__restrict__ p1,
                          const double *__restrict__ t1, double *__restrict__ u,
                          double *__restrict__ r) {
    const double alpha = sc[MR_ALPHA], ma = -alpha;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u[i] += alpha * p1[i];
        r[i] += ma * t1[i];
    }
}

// p2 = z1; p2 += (-alpha1) p1; p2 += (-alpha0) p0
__global__ void k_mr_direction(int n, const double *__restrict__ sc,
                               const double *__restrict__ z1, const double *__restrict__ p1,
                               const double *__restrict__ p0, double *__restrict__ p2) {
    const double a1 = -sc[MR_A1], a0 = -sc[MR_A0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v = z1[i];
        v += a1 * p1[i];
        v += a0 * p0[i];
        p2[i] = v;
    }
}

// a = 0 + s a; b = 0 + s c; d = 0 + s e (the reference's copy, zero, axpy);
// any of b/d may be null
__global__ void k_mr_scale(int n, double s, double *__restrict__ a, double *__restrict__ b,
                           const double *__restrict__ c, double *__restrict__ d,
                           const double *__restrict__ e) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a[i] = 0.0 + s * a[i];
        if (b) b[i] = 0.0 + s * c[i];
        if (d) d[i] = 0.0 + s * e[i];
    }
}

// per-block partials: [0, G) (r, r), [G, 2G) max |u|, [2G, 3G) (u, u), [3G, 4G) (p, p)
__global__ void k_mr_norms(int n, const double *__restrict__ r, const double *__restrict__ u,
                           const double *__restrict__ p, double *part4) {
    __shared__ double sh[32];
    double rr = 0.0, um = 0.0, uu = 0.0, pp = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ri = r[i], ui = u[i], pi = p[i];
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

void row(int prt, int stop_type, int iter, double rel, double abs, double factor) {
    if (prt < PRINT_SOME) return;
    if (iter > 0) {
        printf("%6lld | %13.6e   | %13.6e  | %10.4f\n", (long long)iter, rel, abs, factor);
        return;
    }
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
}  // namespace

int minres(hzb_solver *S, const DCsr<double> &A, const double *b, double *u, int kind,
           HostPrecond *hp, double tol, int MaxIt, int stop_type, int prtlvl,
           double *relres_out) {
    const int MaxStag = MAX_STAG, MaxRestartStep = MAX_RESTART;
    const int m = A.n;
    const double maxdiff = tol * STAG_RATIO, sol_inf_tol = SMALLREAL;
    cudaStream_t s = S->s;
    const int G = reduce_blocks(m);
    int iter = 0, stag = 1, more_step = 1, restart_step = 1;
    double absres0 = BIGREAL, absres = BIGREAL, normr0 = BIGREAL, relres = BIGREAL;
    double normu2 = 0.0, alpha = 0.0;
    MinresWork w;
    HZB_TRY(w.alloc(m));
    auto grid = grid_for(m);
    auto fetch = [&](int lo, int cnt) -> int {
        HZB_CUDA(cudaMemcpyAsync(w.h + lo, w.sc + lo, cnt * sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
        HZB_CUDA(cudaStreamSynchronize(s));
        return SUCCESS;
    };
    auto scalar_dot = [&](const double *x, const double *y, int slot, double *out) -> int {
        HZB_TRY(dot(m, x, y, w.part, w.sc + slot, s));
        HZB_TRY(fetch(slot, 1));
        *out = w.h[slot];
        return SUCCESS;
    };
    auto pc = [&](const double *r, double *z) { return apply_precond(S, kind, hp, m, r, z); };
    // the residual measure of the stopping type from the current r (uses t)
    auto measure = [&](double nu2, double *absr, double *relr) -> int {
        double v = 0.0;
        if (stop_type == STOP_REL_PRECRES) {
            HZB_TRY(pc(w.r, w.t));
            HZB_TRY(scalar_dot(w.r, w.t, MR_RB, &v));
            *absr = sqrt(fabs(v));
            *relr = *absr / normr0;
        } else {
            HZB_TRY(scalar_dot(w.r, w.r, MR_RR, &v));
            *absr = sqrt(v);
            *relr = *absr / (stop_type == STOP_MOD_REL_RES ? nu2 : normr0);
        }
        return SUCCESS;
    };
    // p1 = B r on entry: tp = A p1, tz = B tp, normp = sqrt((tz, tp)), then
    // p1, t1, z1 = (p1, tp, tz) / normp and t0 = z0 = 0
    auto start = [&](bool absolute) -> int {
        HZB_TRY(spmv<double>(A, SPMV_Y, w.p1, nullptr, w.tp, 1.0, nullptr, s));
        HZB_TRY(pc(w.tp, w.tz));
        double v = 0.0;
        HZB_TRY(scalar_dot(w.tz, w.tp, MR_NP, &v));
        const double normp = sqrt(absolute ? fabs(v) : v);
        HZB_TRY(vzero<double>(m, w.t0, s));
        HZB_TRY(vzero<double>(m, w.z0, s));
        k_mr_scale<<<grid, 256, 0, s>>>(m, 1 / normp, w.p1, w.t1, w.tp, w.z1, w.tz);
        count_launch();
        HZB_LAUNCH_CHECK();
        return SUCCESS;
    };

    HZB_TRY(vzero<double>(m, w.p0, s));
    HZB_TRY(spmv<double>(A, SPMV_RES, u, b, w.r, 1.0, nullptr, s));
    HZB_TRY(pc(w.r, w.p1));
    switch (stop_type) {
    case STOP_REL_RES: {
        double v = 0.0;
        HZB_TRY(scalar_dot(w.r, w.r, MR_RR, &v));
        absres0 = sqrt(v);
        normr0 = std::max(SMALLREAL, absres0);
        relres = absres0 / normr0;
        break;
    }
    case STOP_REL_PRECRES: {
        double v = 0.0;
        HZB_TRY(scalar_dot(w.r, w.p1, MR_RB, &v));
        absres0 = sqrt(v);
        normr0 = std::max(SMALLREAL, absres0);
        relres = absres0 / normr0;
        break;
    }
    case STOP_MOD_REL_RES: {
        double v = 0.0, uu = 0.0;
        HZB_TRY(scalar_dot(w.r, w.r, MR_RR, &v));
        HZB_TRY(scalar_dot(u, u, MR_UU, &uu));
        absres0 = sqrt(v);
        normu2 = std::max(SMALLREAL, sqrt(uu));
        relres = absres0 / normu2;
        break;
    }
    default:
        printf("### ERROR: Unrecognized stopping type for %s!\n", "dcsr_pminres");
        goto finished;
    }
    if (relres < tol || absres0 < 1e-3 * tol) goto finished;
    row(prtlvl, stop_type, iter, relres, absres0, 0.0);
    HZB_TRY(start(true));

    while (iter++ < MaxIt) {
        // alpha = (r, z1); u += alpha p1; r -= alpha A p1
        HZB_TRY(dot(m, w.r, w.z1, w.part, w.sc + MR_ALPHA, s));
        k_mr_step<<<grid, 256, 0, s>>>(m, w.sc, w.p1, w.t1, u, w.r);
        count_launch();
        // p2 = z1 - (z1, A z1) p1 - (z1, A z0) p0
        HZB_TRY(spmv<double>(A, SPMV_Y, w.z1, nullptr, w.t, 1.0, nullptr, s));
        HZB_TRY(dot(m, w.z1, w.t, w.part, w.sc + MR_A1, s));
        HZB_TRY(spmv<double>(A, SPMV_Y, w.z0, nullptr, w.t, 1.0, nullptr, s));
        HZB_TRY(dot(m, w.z1, w.t, w.part, w.sc + MR_A0, s));
        k_mr_direction<<<grid, 256, 0, s>>>(m, w.sc, w.z1, w.p1, w.p0, w.p2);
        count_launch();
        HZB_LAUNCH_CHECK();
        // normalise by sqrt|(B A p2, A p2)|
        HZB_TRY(spmv<double>(A, SPMV_Y, w.p2, nullptr, w.tp, 1.0, nullptr, s));
        HZB_TRY(pc(w.tp, w.tz));
        HZB_TRY(dot(m, w.tz, w.tp, w.part, w.sc + MR_NP, s));
        HZB_TRY(fetch(0, MR_NP + 1));
        alpha = w.h[MR_ALPHA];
        const double normp = sqrt(fabs(w.h[MR_NP]));
        if (normp < 1e-14) {   // lucky breakdown: u solves the system
            iter--;
            break;
        }
        // p2 /= normp; the new t1, z1 = (tp, tz) / normp go into the buffers
        // of t0, z0, which the rotation below retires
        k_mr_scale<<<grid, 256, 0, s>>>(m, 1 / normp, w.p2, w.t0, w.tp, w.z0, w.tz);
        count_launch();
        HZB_LAUNCH_CHECK();
        {
            double *op0 = w.p0;
            w.p0 = w.p1;
            w.p1 = w.p2;
            w.p2 = op0;
            std::swap(w.t0, w.t1);
            std::swap(w.z0, w.z1);
        }
        // ||u||, max |u|, (r, r), ||p1|| in one pass
        k_mr_norms<<<G, 256, 0, s>>>(m, w.r, u, w.p1, w.part);
        count_launch();
        HZB_LAUNCH_CHECK();
        HZB_TRY(reduce_final(w.part, G, w.sc + MR_RR, s));
        HZB_TRY(reduce_final_max(w.part + G, G, w.sc + MR_UM, s));
        HZB_TRY(reduce_final(w.part + 2 * G, G, w.sc + MR_UU, s));
        HZB_TRY(reduce_final(w.part + 3 * G, G, w.sc + MR_PP, s));
        HZB_TRY(fetch(MR_RR, 4));
        normu2 = sqrt(w.h[MR_UU]);
        if (stop_type == STOP_REL_PRECRES) {
            double v = 0.0;
            HZB_TRY(pc(w.r, w.t));
            HZB_TRY(scalar_dot(w.r, w.t, MR_RB, &v));
            absres = sqrt(fabs(v));
            relres = absres / normr0;
        } else {
            absres = sqrt(w.h[MR_RR]);
            relres = absres / (stop_type == STOP_MOD_REL_RES ? normu2 : normr0);
        }
        const double factor = absres / absres0;
        row(prtlvl, stop_type, iter, relres, absres, factor);

        // Check I: solution close to zero
        if (w.h[MR_UM] <= sol_inf_tol) {
            if (prtlvl > PRINT_MIN)
                printf("### HAZMATH WARNING: Iteration stopped due to the solution is almost "
                       "zero! %s : %lld\n", __FUNCTION__, (long long)__LINE__);
            iter = ERROR_SOLVER_SOLSTAG;
            break;
        }
        // Check II: stagnation
        const double normuu = fabs(alpha) * (sqrt(w.h[MR_PP]) / normu2);
        if (normuu < maxdiff) {
            if (stag < MaxStag && prtlvl >= PRINT_MORE) {
                printf("||u-u'|| = %e and the comp. rel. res. = %e.\n", normuu, relres);
                printf("### HAZMATH WARNING: Iteration restarted due to stagnation! %s : %lld\n",
                       __FUNCTION__, (long long)__LINE__);
            }
            HZB_TRY(spmv<double>(A, SPMV_RES, u, b, w.r, 1.0, nullptr, s));
            HZB_TRY(measure(normu2, &absres, &relres));
            if (prtlvl >= PRINT_MORE)
                printf("### HAZMATH WARNING: The actual relative residual = %e!\n", relres);
            if (relres < tol) break;
            if (stag >= MaxStag) {
                if (prtlvl > PRINT_MIN)
                    printf("### HAZMATH WARNING: Iteration stopped due to staggnation! %s : "
                           "%lld\n", __FUNCTION__, (long long)__LINE__);
                iter = ERROR_SOLVER_STAG;
                break;
            }
            HZB_TRY(vzero<double>(m, w.p0, s));
            ++stag;
            ++restart_step;
            HZB_TRY(pc(w.r, w.p1));
            HZB_TRY(start(true));
        }
        // Check III: false convergence
        if (relres < tol) {
            if (prtlvl >= PRINT_MORE)
                printf("### HAZMATH WARNING: The computed relative residual = %e!\n", relres);
            HZB_TRY(spmv<double>(A, SPMV_RES, u, b, w.r, 1.0, nullptr, s));
            HZB_TRY(measure(normu2, &absres, &relres));
            if (prtlvl >= PRINT_MORE)
                printf("### HAZMATH WARNING: The actual relative residual = %e!\n", relres);
            if (relres < tol) break;
            if (more_step >= MaxRestartStep) {
                if (prtlvl > PRINT_MIN)
                    printf("### HAZMATH WARNING: The tolerence might be too small! %s : %lld\n",
                           __FUNCTION__, (long long)__LINE__);
                iter = ERROR_SOLVER_TOLSMALL;
                break;
            }
            HZB_TRY(vzero<double>(m, w.p0, s));
            ++more_step;
            ++restart_step;
            HZB_TRY(pc(w.r, w.p1));
            HZB_TRY(start(false));   // the reference takes no absolute value here
        }
        absres0 = absres;
    }
finished:
    if (prtlvl > PRINT_NONE) {
        if (iter > MaxIt)
            printf("### HAZMATH WARNING: Max iter %lld reached with rel. resid. %e.\n",
                   (long long)MaxIt, relres);
        else if (iter >= 0)
            printf("Num_iter(krylov.c) = %lld with relative residual %e.\n", (long long)iter,
                   relres);
        fflush(stdout);
    }
    if (relres_out) *relres_out = relres;
    HZB_CUDA(cudaStreamSynchronize(s));
    (void)restart_step;
    return iter > MaxIt ? ERROR_SOLVER_MAXIT : iter;
}

}  // namespace hzb
