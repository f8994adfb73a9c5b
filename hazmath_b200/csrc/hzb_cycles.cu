// hzb_cycles.cu -- the multilevel cycles behind cycle_type 3, 4 and 5 and the
// generalized conjugate gradient method.
//
// linear_solver_dcsr_krylov_amg (itsolver.c:899-917) hands its Krylov method
// precond_amli, precond_nl_amli or precond_amg_add instead of precond_amg
// when cycle_type is AMLI_CYCLE (3), NL_AMLI_CYCLE (4) or ADD_CYCLE (5):
//
//   amli (mgcycle.c:430-555): the coarse-grid correction is a polynomial in
//     the recursive coarse cycle, with the coefficients of the best uniform
//     approximation of 1/x on [0.5, 2] (amg_amli_coef, parameters.c:714-775;
//     interval set in amg_setup_ua.c:1276-1281), evaluated through
//     degree + 1 recursive calls on the coarse level;
//   nl_amli (mgcycle.c:561-690): the coarse-grid correction is degree + 1
//     steps of flexible GMRES (restart 30) or of GCG on the coarse operator,
//     preconditioned by the same cycle one level down; the second-coarsest
//     level goes straight to the coarsest solve;
//   mgcycle_add (mgcycle.c:700-820): each level pre-smooths its restricted
//     residual with a zero start, the corrections are prolongated back with
//     no post-smoothing.
//
// Everything runs on the device data of the hierarchy with the FP64 level
// kernels of the V-cycle.  Vector updates keep the reference's per-element
// arithmetic (y + a*x, x*a; compiled without FMA contraction); inner
// products are fixed-order tree reductions.
#include "hzb_solver.cuh"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

namespace hzb {

// y += a x (array_axpy; the reference's a = +-1 branches give the same
// IEEE results as y + a*x)
__global__ void k_cy_axpy(int n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] += a * x[i];
}

// x *= a (array_ax)
__global__ void k_cy_scale(int n, double a, double *__restrict__ x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] *= a;
}

static int axpy(int n, double a, const double *x, double *y, cudaStream_t s) {
    k_cy_axpy<<<grid_for(n), 256, 0, s>>>(n, a, x, y);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

static int scale(int n, double a, double *x, cudaStream_t s) {
    if (a == 1.0) return SUCCESS;
    k_cy_scale<<<grid_for(n), 256, 0, s>>>(n, a, x);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// AMLI polynomial
// ---------------------------------------------------------------------------
// Coefficients q_0 .. q_degree of the polynomial of best uniform
// approximation of 1/x on [lambda_min, lambda_max] (Kraus, Vassilevski,
// Zikatanov 2013), by its three-term recurrence in the degree.
int amli_coefficients(double lambda_max, double lambda_min, int degree, double *coef) {
    if (degree < 0) {
        set_error_msg("wrong AMLI degree");
        return ERROR_INPUT_PAR;
    }
    const double mu0 = 1.0 / lambda_max, mu1 = 1.0 / lambda_min;
    const double c = (sqrt(mu0) + sqrt(mu1)) * (sqrt(mu0) + sqrt(mu1));
    const double a = (4 * mu0 * mu1) / c;
    const double kappa = lambda_max / lambda_min;
    const double delta = (sqrt(kappa) - 1.0) / (sqrt(kappa) + 1.0);
    const double b = delta * delta;
    if (degree == 0) {
        coef[0] = 0.5 * (mu0 + mu1);
        return SUCCESS;
    }
    if (degree == 1) {
        coef[0] = 0.5 * c;
        coef[1] = -1.0 * mu0 * mu1;
        return SUCCESS;
    }
    std::vector<double> q1(degree), q2(degree - 1);   // degrees - 1 and - 2
    amli_coefficients(lambda_max, lambda_min, degree - 1, q1.data());
    amli_coefficients(lambda_max, lambda_min, degree - 2, q2.data());
    coef[0] = a - b * q2[0] + (1 + b) * q1[0];
    for (int i = 1; i < degree - 1; ++i) coef[i] = -b * q2[i] + (1 + b) * q1[i] - a * q1[i - 1];
    coef[degree - 1] = (1 + b) * q1[degree - 1] - a * q1[degree - 2];
    coef[degree] = -a * q1[degree - 1];
    return SUCCESS;
}

int cycles_prepare(hzb_solver *S, int kind, const AMG_param &cyc) {
    if (kind != PC_AMLI) return SUCCESS;
    const int deg = cyc.amli_degree;
    if (deg < 0) {
        set_error_msg("wrong AMLI degree");
        return ERROR_INPUT_PAR;
    }
    if (cyc.amli_coef) {
        S->amli_coef.assign(cyc.amli_coef, cyc.amli_coef + deg + 1);
    } else if ((int)S->amli_coef.size() != deg + 1) {
        S->amli_coef.assign(deg + 1, 0.0);
        HZB_TRY(amli_coefficients(2.0, 0.5, deg, S->amli_coef.data()));
    }
    for (int l = 1; l < S->nl; ++l)
        if (!S->lv[l].r1) HZB_TRY(dalloc(&S->lv[l].r1, S->lv[l].n));
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// the cycles
// ---------------------------------------------------------------------------
int amli64(hzb_solver *S, const AMG_param &cyc, const double *coef, int l) {
    cudaStream_t s = S->s;
    if (l >= S->nl - 1) return coarse_solve64(S, cyc, cyc.tol * 1e-4);
    Level &L = S->lv[l], &C = S->lv[l + 1];
    const int degree = cyc.amli_degree;
    HZB_TRY(smooth64(S, l, true, cyc));
    HZB_TRY(spmv<double>(L.A64(), SPMV_RES, L.x, L.b, L.w, 1.0, nullptr, s));
    HZB_TRY(restrict_level(S, l, L.w, C.b));
    HZB_TRY(vcopy<double>(C.n, C.b, C.r1, s));
    // b_c = A_c e_c + (q_{degree-i} / q_degree) r_c after each inner cycle
    for (int i = 1; i <= degree; ++i) {
        HZB_TRY(vzero<double>(C.n, C.x, s));
        HZB_TRY(amli64(S, cyc, coef, l + 1));
        HZB_TRY(spmv<double>(C.A64(), SPMV_Y, C.x, nullptr, C.b, 1.0, nullptr, s));
        HZB_TRY(axpy(C.n, coef[degree - i] / coef[degree], C.r1, C.b, s));
    }
    HZB_TRY(vzero<double>(C.n, C.x, s));
    HZB_TRY(amli64(S, cyc, coef, l + 1));
    HZB_TRY(scale(C.n, coef[degree], C.x, s));
    double alpha = 1.0;
    if (cyc.coarse_scaling == ON) HZB_TRY(coarse_alpha(S, l + 1, C.r1, &alpha));
    HZB_TRY(prolong_level(S, l, C.x, L.x, alpha));
    return smooth64(S, l, false, cyc);
}

int nl_amli64(hzb_solver *S, const AMG_param &cyc, int l) {
    cudaStream_t s = S->s;
    const double tol = cyc.tol * 1e-4;
    if (l >= S->nl - 1) return coarse_solve64(S, cyc, tol);
    Level &L = S->lv[l], &C = S->lv[l + 1];
    HZB_TRY(smooth64(S, l, true, cyc));
    HZB_TRY(spmv<double>(L.A64(), SPMV_RES, L.x, L.b, L.w, 1.0, nullptr, s));
    HZB_TRY(restrict_level(S, l, L.w, C.b));
    HZB_TRY(vzero<double>(C.n, C.x, s));
    if (l == S->nl - 2) {
        HZB_TRY(nl_amli64(S, cyc, l + 1));
    } else {
        // degree + 1 Krylov steps on A_c e_c = b_c preconditioned by this
        // cycle from level l + 1.  The preconditioner points level l + 1's
        // b and x at the Krylov vectors while it runs, so b_c and e_c serve
        // as the Krylov method's own right-hand side and iterate (the
        // reference copies them through work vectors instead).
        const int maxit = cyc.amli_degree + 1;
        double rel = 0.0;
        int it;
        if (cyc.nl_amli_krylov_type == SOLVER_GCG)
            it = gcg(S, C.A64(), C.b, C.x, PC_NLAMLI + l + 1, nullptr, tol, maxit, STOP_REL_RES,
                     PRINT_NONE, &rel, l + 1);
        else
            it = gmres(S, C.A64(), C.b, C.x, PC_NLAMLI + l + 1, nullptr, tol, maxit, 30,
                       STOP_REL_RES, PRINT_NONE, true, &rel, l + 1);
        if (it < 0 && it != ERROR_SOLVER_MAXIT) return it;
    }
    HZB_TRY(prolong_level(S, l, C.x, L.x, 1.0));
    return smooth64(S, l, false, cyc);
}

int add_cycle64(hzb_solver *S, const AMG_param &cyc) {
    cudaStream_t s = S->s;
    const int nl = S->nl;
    Level &L0 = S->lv[0];
    // the fine residual before any smoothing; coarser levels start from 0,
    // so their right-hand side is their residual
    HZB_TRY(spmv<double>(L0.A64(), SPMV_RES, L0.x, L0.b, L0.w, 1.0, nullptr, s));
    int l = 0;
    while (l < nl - 1) {
        Level &L = S->lv[l];
        HZB_TRY(smooth64(S, l, true, cyc));
        HZB_TRY(restrict_level(S, l, l == 0 ? L.w : L.b, S->lv[l + 1].b));
        ++l;
        HZB_TRY(vzero<double>(S->lv[l].n, S->lv[l].x, s));
    }
    HZB_TRY(coarse_solve64(S, cyc, cyc.tol * 1e-2));
    double alpha = 1.0;
    while (l > 0) {
        --l;
        Level &L = S->lv[l];
        if (cyc.coarse_scaling == ON) HZB_TRY(coarse_alpha(S, l + 1, S->lv[l + 1].b, &alpha));
        HZB_TRY(prolong_level(S, l, S->lv[l + 1].x, L.x, alpha));
    }
    return SUCCESS;
}

int precond_cycles(hzb_solver *S, int kind, int l, int maxit, const double *r, double *z,
                   const AMG_param &cyc) {
    if (l < 0 || l >= S->nl) return ERROR_INPUT_PAR;
    Level &L = S->lv[l];
    double *sb = L.b, *sx = L.x;
    L.b = const_cast<double *>(r);
    L.x = z;
    int rc = vzero<double>(L.n, z, S->s);
    for (int i = 0; rc == SUCCESS && i < maxit; ++i) {
        if (kind == PC_AMLI) rc = amli64(S, cyc, S->amli_coef.data(), l);
        else if (kind == PC_ADD) rc = add_cycle64(S, cyc);
        else rc = nl_amli64(S, cyc, l);
    }
    L.b = sb;
    L.x = sx;
    return rc;
}

// ---------------------------------------------------------------------------
// GCG, dcsr_pgcg (krylov.c:2309-2420): steepest descent first, then each
// preconditioned residual A-orthogonalised against every earlier direction
// (no restart).  A p_i and (p_i, A p_i) are kept with the directions, so
// each step costs one preconditioner call and one product with A; the
// scalars stay on the device and one norm per step is read back.
// ---------------------------------------------------------------------------
struct GcgWork {
    int n = 0;
    std::vector<double *> p, ap;        // directions and A times them
    double **d_p = nullptr;             // device copy of p's pointers
    int dcap = 0;
    double *r = nullptr, *br = nullptr;
    double *part = nullptr;             // 4 reduce_blocks(n) + 8
    double *sc = nullptr;               // [0] (r, p) [1] (r, r) [2 ..] (B r, A p_i), then (p_i, A p_i)
    int scap = 0;
    double *h = nullptr;                // pinned host scalar
    int alloc(int nn) {
        n = nn;
        HZB_TRY(dalloc(&r, n));
        HZB_TRY(dalloc(&br, n));
        HZB_TRY(dalloc(&part, 4 * reduce_blocks(n) + 8));
        HZB_CUDA(cudaMallocHost((void **)&h, 2 * sizeof(double)));
        return SUCCESS;
    }
    // room for k directions and their scalars
    int reserve(int k) {
        while ((int)p.size() < k) {
            double *v = nullptr, *w = nullptr;
            HZB_TRY(dalloc(&v, n));
            p.push_back(v);
            HZB_TRY(dalloc(&w, n));
            ap.push_back(w);
        }
        if (dcap < k) {
            dfree(d_p);
            dcap = std::max(k, 2 * dcap);
            HZB_TRY(dalloc(&d_p, dcap));
        }
        HZB_CUDA(cudaMemcpyAsync(d_p, p.data(), k * sizeof(double *), cudaMemcpyHostToDevice,
                                 cur_stream()));
        if (scap < 2 + 2 * k) {
            dfree(sc);
            scap = std::max(2 + 2 * k, 2 * scap);
            HZB_TRY(dalloc(&sc, scap));
        }
        return SUCCESS;
    }
    ~GcgWork() {
        for (auto v : p) dfree(v);
        for (auto v : ap) dfree(v);
        dfree(d_p); dfree(r); dfree(br); dfree(part); dfree(sc);
        if (h) cudaFreeHost(h);
    }
};

void gcg_release(hzb_solver *S) {
    for (auto &g : S->gcg_ws) delete g;
    S->gcg_ws.clear();
}

// out = br + sum_{i < m} beta_i p_i with beta_i = -(nb_i / den_i), added in
// i order per element as the reference's sequence of array_axpy calls
__global__ void k_gcg_direction(int n, int m, const double *__restrict__ br,
                                const double *const *__restrict__ p,
                                const double *__restrict__ nb, const double *__restrict__ den,
                                double *__restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double v = br[k];
        for (int i = 0; i < m; ++i) {
            const double beta = (-1.0) * (nb[i] / den[i]);
            v += beta * p[i][k];
        }
        out[k] = v;
    }
}

static void gcg_row(int prt, int iter, double rel, double abs, double factor) {
    if (prt < PRINT_SOME) return;
    printf("%6lld | %13.6e   | %13.6e  | %10.4f\n", (long long)iter, rel, abs, factor);
}

int gcg(hzb_solver *S, const DCsr<double> &A, const double *b, double *u, int kind,
        HostPrecond *hp, double tol, int MaxIt, int stop_type, int prtlvl, double *relres_out,
        int ws_slot) {
    (void)stop_type;   // the reference's GCG tests ||r|| / ||b|| whatever the type
    const int m = A.n;
    cudaStream_t s = S->s;
    std::unique_ptr<GcgWork> own;
    GcgWork *gp = nullptr;
    if (ws_slot >= 0 && ws_slot < (int)S->gcg_ws.size() && S->gcg_ws[ws_slot] &&
        S->gcg_ws[ws_slot]->n == m) {
        gp = S->gcg_ws[ws_slot];
    } else {
        own.reset(new GcgWork());
        HZB_TRY(own->alloc(m));
        if (ws_slot >= 0) {
            if ((int)S->gcg_ws.size() <= ws_slot) S->gcg_ws.resize(ws_slot + 1, nullptr);
            delete S->gcg_ws[ws_slot];
            S->gcg_ws[ws_slot] = own.release();
            gp = S->gcg_ws[ws_slot];
        } else {
            gp = own.get();
        }
    }
    GcgWork &g = *gp;
    const int ndir = std::max(MaxIt, 1);
    HZB_TRY(g.reserve(ndir));
    const int G = reduce_blocks(m);
    double *num = g.sc, *rr = g.sc + 1, *nb = g.sc + 2, *den = g.sc + 2 + ndir;
    auto read = [&](const double *d, double *hv) -> int {
        HZB_CUDA(cudaMemcpyAsync(g.h, d, sizeof(double), cudaMemcpyDeviceToHost, s));
        HZB_CUDA(cudaStreamSynchronize(s));
        *hv = g.h[0];
        return SUCCESS;
    };
    // u += alpha p_k, r -= alpha A p_k with alpha = (r, p_k) / (p_k, A p_k);
    // then ||r||
    auto step = [&](int k, double *absres) -> int {
        HZB_TRY(spmv<double>(A, SPMV_Y, g.p[k], nullptr, g.ap[k], 1.0, nullptr, s));
        HZB_TRY(dot(m, g.p[k], g.ap[k], g.part, den + k, s));
        HZB_TRY(dot(m, g.r, g.p[k], g.part, num, s));
        HZB_TRY(pcg_update(m, num, den + k, u, g.r, g.p[k], g.ap[k], g.part, s));
        HZB_TRY(reduce_final(g.part, G, rr, s));
        double t = 0.0;
        HZB_TRY(read(rr, &t));
        *absres = sqrt(t);
        return SUCCESS;
    };

    int iter = 0;
    double absres0 = BIGREAL, absres = 0.0, relres = BIGREAL, factor = 0.0, normb = 0.0;
    HZB_TRY(dot(m, b, b, g.part, rr, s));
    HZB_TRY(read(rr, &normb));
    normb = sqrt(normb);
    // first step: steepest descent along B r
    HZB_TRY(spmv<double>(A, SPMV_RES, u, b, g.r, 1.0, nullptr, s));
    HZB_TRY(apply_precond(S, kind, hp, m, g.r, g.p[0]));
    HZB_TRY(step(0, &absres));
    factor = absres / absres0;
    relres = absres / normb;
    gcg_row(prtlvl, iter + 1, relres, absres, factor);
    absres0 = absres;
    for (iter = 1; iter < MaxIt; ++iter) {
        HZB_TRY(apply_precond(S, kind, hp, m, g.r, g.br));
        for (int i = 0; i < iter; ++i) HZB_TRY(dot(m, g.br, g.ap[i], g.part, nb + i, s));
        k_gcg_direction<<<grid_for(m), 256, 0, s>>>(m, iter, g.br, g.d_p, nb, den, g.p[iter]);
        count_launch();
        HZB_LAUNCH_CHECK();
        HZB_TRY(step(iter, &absres));
        factor = absres / absres0;
        relres = absres / normb;
        gcg_row(prtlvl, iter + 1, relres, absres, factor);
        if (relres < tol) break;
        absres0 = absres;
    }
    if (prtlvl > PRINT_NONE) {
        if (iter > MaxIt)
            printf("### HAZMATH WARNING: Max iter %lld reached with rel. resid. %e.\n",
                   (long long)MaxIt, relres);
        else
            printf("Num_iter(krylov.c) = %lld with relative residual %e.\n", (long long)iter,
                   relres);
        fflush(stdout);
    }
    if (relres_out) *relres_out = relres;
    return iter > MaxIt ? ERROR_SOLVER_MAXIT : iter;
}

}  // namespace hzb
