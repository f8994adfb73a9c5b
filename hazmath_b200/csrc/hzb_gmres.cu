// hzb_gmres.cu -- variable-restart GMRES and flexible GMRES with the AMG
// preconditioner: dcsr_pvgmres (krylov.c:4612-4930) and dcsr_pvfgmres
// (krylov.c:5974-6250), the Krylov types 3 and 4 of
// solver_dcsr_linear_itsolver (itsolver.c:135); type 4 with restart 100 is the
// reference's default (param_linear_solver_init, parameters.c:241-245).
//
// The Krylov basis lives on the device.  Every vector operation keeps the
// reference's per-element arithmetic (y + a*x, x*a, sums over the basis in the
// reference's j order), compiled without FMA contraction; the modified
// Gram-Schmidt step fuses each update p_i -= h_j p_j with the next inner
// product (p_{j+1}, p_i), which reads the same updated values.  Inner products
// and norms are fixed-order tree reductions (the reference sums left to
// right, so they agree to rounding).  The Hessenberg column, the Givens
// rotations, the restart adaptation and the stopping tests run on the host
// in the reference's order, one device-to-host read per iteration.
#include "hzb_solver.cuh"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <memory>
#include <vector>

namespace hzb {

// pi[k] += (-h[j]) * pj[k]; then partial sums of q[k] * pi[k] (q = p_{j+1},
// or pi itself for the norm) per block
__global__ void k_gm_mgs(int n, const double *__restrict__ h, int j,
                         const double *__restrict__ pj, double *__restrict__ pi,
                         const double *__restrict__ q, double *part) {
    __shared__ double sh[32];
    const double a = -h[j];
    double acc = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double v = pi[k] + a * pj[k];
        pi[k] = v;
        acc += (q ? q[k] : v) * v;
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// x *= 1 / sqrt(t2[0]) when the norm is not zero (array_ax with t = 1/||x||)
__global__ void k_gm_normalize(int n, const double *__restrict__ t2, double *x) {
    const double t = sqrt(t2[0]);
    if (t == 0.0) return;
    const double r = 1.0 / t;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        x[k] *= r;
}

// y[k] *= a (array_ax; a == 1 leaves y as is, as the reference does)
__global__ void k_gm_scale(int n, double a, double *y) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        y[k] *= a;
}

// w = c[m-1] * v[m-1], then w += c[j] * v[j] for j = m-2 .. 0 (array_cp,
// array_ax, array_axpy in the reference's order), per element
__global__ void k_gm_combine(int n, int m, const double *const *__restrict__ v,
                             const double *__restrict__ c, double *w) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double acc = v[m - 1][k];
        if (c[m - 1] != 1.0) acc *= c[m - 1];
        for (int j = m - 2; j >= 0; --j) acc = acc + c[j] * v[j][k];
        w[k] = acc;
    }
}

// The residual direction after a cycle (krylov.c:4887-4903):
//   p_i += (rs_i - 1) p_i;  p_i += rs_j p_j for j = i-1 .. 1;
//   p_0 += (rs_0 - 1) p_0;  p_0 += p_i
__global__ void k_gm_residual(int n, int i, double *const *__restrict__ p,
                              const double *__restrict__ rs) {
    double *pi = p[i], *p0 = p[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double v = pi[k];
        v = v + (rs[i] - 1.0) * v;
        for (int j = i - 1; j > 0; --j) v = v + rs[j] * p[j][k];
        pi[k] = v;
        double u = p0[k];
        u = u + (rs[0] - 1.0) * u;
        p0[k] = u + v;
    }
}

// y += x
__global__ void k_gm_add(int n, const double *__restrict__ x, double *y) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        y[k] += x[k];
}

struct GmresWork {
    int n = 0, restart = 0, req = 0;   // allocated / requested restart
    bool flexible = false;
    std::vector<double *> p, z;       // restart + 1 each (z only when flexible)
    double *r = nullptr, *w = nullptr;
    double *col = nullptr;            // Hessenberg column of the current step
    double *coef = nullptr;           // coefficients of a combination
    double **d_p = nullptr, **d_z = nullptr;
    double *part = nullptr, *sc = nullptr, *h_sc = nullptr;
    int alloc(int nn, int rst, bool flex) {
        n = nn;
        restart = rst;
        flexible = flex;
        p.assign(rst + 1, nullptr);
        z.assign(flex ? rst + 1 : 0, nullptr);
        for (auto &v : p) HZB_TRY(dalloc(&v, n));
        for (auto &v : z) HZB_TRY(dalloc(&v, n));
        HZB_TRY(dalloc(&r, n));
        HZB_TRY(dalloc(&w, n));
        HZB_TRY(dalloc(&col, rst + 2));
        HZB_TRY(dalloc(&coef, rst + 2));
        HZB_TRY(dalloc(&d_p, rst + 1));
        if (flex) HZB_TRY(dalloc(&d_z, rst + 1));
        HZB_TRY(dalloc(&part, reduce_blocks(n) + 8));
        HZB_TRY(dalloc(&sc, 4));
        HZB_CUDA(cudaMallocHost((void **)&h_sc, (rst + 4) * sizeof(double)));
        HZB_CUDA(cudaMemcpyAsync(d_p, p.data(), (rst + 1) * sizeof(double *),
                                 cudaMemcpyHostToDevice, cur_stream()));
        if (flex)
            HZB_CUDA(cudaMemcpyAsync(d_z, z.data(), (rst + 1) * sizeof(double *),
                                     cudaMemcpyHostToDevice, cur_stream()));
        return SUCCESS;
    }
    ~GmresWork() {
        for (auto v : p) dfree(v);
        for (auto v : z) dfree(v);
        dfree(r); dfree(w); dfree(col); dfree(coef); dfree(d_p); dfree(d_z);
        dfree(part); dfree(sc);
        if (h_sc) cudaFreeHost(h_sc);
    }
};

void gmres_release(hzb_solver *S) {
    for (auto &g : S->gm_ws) delete g;
    S->gm_ws.clear();
}

namespace {
void print_row(int prt, int iter, double rel, double abs, double factor) {
    if (prt < PRINT_SOME) return;
    printf("%6lld | %13.6e   | %13.6e  | %10.4f\n", (long long)iter, rel, abs, factor);
    fflush(stdout);
}
void print_head(int prt, int stop_type, double rel, double abs) {
    if (prt < PRINT_SOME) return;
    printf("-----------------------------------------------------------\n");
    if (stop_type == STOP_REL_RES)
        printf("It Num |   ||r||/||b||   |     ||r||      |  Conv. Factor\n");
    else if (stop_type == STOP_REL_PRECRES)
        printf("It Num | ||r||_B/||b||_B |    ||r||_B     |  Conv. Factor\n");
    else
        printf("It Num |   ||r||/||x||   |     ||r||      |  Conv. Factor\n");
    printf("-----------------------------------------------------------\n");
    printf("%6lld | %13.6e   | %13.6e  |     -.-- \n", 0LL, rel, abs);
    fflush(stdout);
}
}  // namespace

// host value of a device scalar
static int read_scalar(hzb_solver *S, const double *d, double *h) {
    HZB_CUDA(cudaMemcpyAsync(h, d, sizeof(double), cudaMemcpyDeviceToHost, S->s));
    HZB_CUDA(cudaStreamSynchronize(S->s));
    return SUCCESS;
}

static int norm2_host(hzb_solver *S, GmresWork &g, const double *x, double *out) {
    HZB_TRY(dot(g.n, x, x, g.part, g.sc, S->s));
    double t2 = 0.0;
    HZB_TRY(read_scalar(S, g.sc, &t2));
    *out = sqrt(t2);
    return SUCCESS;
}

static int dot_host(hzb_solver *S, GmresWork &g, const double *x, const double *y,
                    double *out) {
    HZB_TRY(dot(g.n, x, y, g.part, g.sc, S->s));
    return read_scalar(S, g.sc, out);
}

// One Arnoldi step on the device: p_i = A M p_{i-1} (M p_{i-1} into zout),
// orthogonalised against p_0 .. p_{i-1} by modified Gram-Schmidt and
// normalised; col[0 .. i] receives h_{0..i-1,i-1} and ||p_i||^2.
static int arnoldi(hzb_solver *S, GmresWork &g, const DCsr<double> &A, int kind,
                   HostPrecond *hp, int i, double *zout, std::vector<double> &h) {
    const int n = g.n;
    cudaStream_t s = S->s;
    HZB_TRY(apply_precond(S, kind, hp, n, g.p[i - 1], zout));   // z = M p_{i-1}
    HZB_TRY(spmv<double>(A, SPMV_Y, zout, nullptr, g.p[i], 1.0, nullptr, s));
    const int G = reduce_blocks(n);
    HZB_TRY(dot(n, g.p[0], g.p[i], g.part, g.col + 0, s));
    for (int j = 0; j < i; ++j) {
        const double *q = j + 1 < i ? g.p[j + 1] : nullptr;
        k_gm_mgs<<<G, 256, 0, s>>>(n, g.col, j, g.p[j], g.p[i], q, g.part);
        count_launch();
        HZB_TRY(reduce_final(g.part, G, g.col + j + 1, s));
    }
    k_gm_normalize<<<grid_for(n), 256, 0, s>>>(n, g.col + i, g.p[i]);
    count_launch();
    HZB_LAUNCH_CHECK();
    HZB_CUDA(cudaMemcpyAsync(g.h_sc, g.col, (i + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                             s));
    HZB_CUDA(cudaStreamSynchronize(s));
    h.assign(g.h_sc, g.h_sc + i + 1);
    h[i] = sqrt(h[i]);
    return SUCCESS;
}

// w = sum over the basis with the coefficients c (the reference's order)
static int combine(hzb_solver *S, GmresWork &g, double *const *d_v, int m,
                   const std::vector<double> &c, double *w) {
    HZB_CUDA(cudaMemcpyAsync(g.coef, c.data(), m * sizeof(double), cudaMemcpyHostToDevice,
                             S->s));
    k_gm_combine<<<grid_for(g.n), 256, 0, S->s>>>(g.n, m, d_v, g.coef, w);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

int gmres(hzb_solver *S, const DCsr<double> &A, const double *b, double *x, int kind,
          HostPrecond *hp, double tol, int MaxIt, int restart, int stop_type, int prtlvl,
          bool flexible, double *relres_out, int ws_slot) {
    const int n = A.n;
    cudaStream_t s = S->s;
    const double cr_max = 0.99, cr_min = 0.174, epsmac = SMALLREAL;
    const int d = 3, restart_min = 3, restart_max = restart;
    if (restart < 1) return ERROR_INPUT_PAR;
    int Restart = restart;
    // A kept basis serves the coarse-level solves of the nonlinear AMLI
    // cycle (MaxIt = degree + 1).  Its basis holds min(restart, MaxIt)
    // vectors when MaxIt <= 4 <= restart: the restart adaptation below never
    // takes the cycle length under 4 then, so every cycle runs to MaxIt
    // either way and the iterates are the same.
    const int want = (ws_slot >= 0 && MaxIt <= 4 && restart >= 4) ? std::max(MaxIt, 1) : restart;
    std::unique_ptr<GmresWork> gw;
    GmresWork *gp = nullptr;
    if (ws_slot >= 0 && ws_slot < (int)S->gm_ws.size() && S->gm_ws[ws_slot] &&
        S->gm_ws[ws_slot]->n == n && S->gm_ws[ws_slot]->req == want &&
        S->gm_ws[ws_slot]->flexible == flexible) {
        gp = S->gm_ws[ws_slot];
        Restart = gp->restart;
    } else {
        // the reference shrinks the restart by 5 while its work space does
        // not fit
        Restart = want;
        gw.reset(new GmresWork());
        int rc = gw->alloc(n, Restart, flexible);
        while (rc == ERROR_ALLOC_MEM && Restart > 5) {
            Restart -= 5;
            gw.reset(new GmresWork());
            rc = gw->alloc(n, Restart, flexible);
        }
        if (rc) return rc;
        gw->req = want;
        if (prtlvl > PRINT_MIN && Restart < want)
            printf("### WARNING: %s restart number set to %lld!\n",
                   flexible ? "vFGMRES" : "vGMRES", (long long)Restart);
        if (ws_slot >= 0) {
            if ((int)S->gm_ws.size() <= ws_slot) S->gm_ws.resize(ws_slot + 1, nullptr);
            delete S->gm_ws[ws_slot];
            S->gm_ws[ws_slot] = gw.release();
            gp = S->gm_ws[ws_slot];
        } else {
            gp = gw.get();
        }
    }
    GmresWork &g = *gp;
    std::vector<double> c(Restart + 1), sn(Restart + 1), rs(Restart + 2), h;
    std::vector<std::vector<double>> hh(Restart + 1, std::vector<double>(Restart + 1, 0.0));
    std::vector<double> norms(MaxIt + 2, 0.0);
    int iter = 0, i = 0;
    double r_norm = 0.0, relres = BIGREAL, absres0 = BIGREAL, absres = BIGREAL;
    double den_norm = 0.0, b_norm = 0.0, epsilon = 0.0, cr = 1.0, r_norm_old = 0.0;
    // r = b - A x
    HZB_TRY(spmv<double>(A, SPMV_RES, x, b, g.p[0], 1.0, nullptr, s));
    HZB_TRY(norm2_host(S, g, g.p[0], &r_norm));
    if (!flexible) {
        switch (stop_type) {
        case STOP_REL_RES:
            absres0 = std::max(SMALLREAL, r_norm);
            relres = r_norm / absres0;
            break;
        case STOP_REL_PRECRES: {
            HZB_TRY(apply_precond(S, kind, hp, n, g.p[0], g.r));
            double t = 0.0;
            HZB_TRY(dot_host(S, g, g.p[0], g.r, &t));
            const double r_normb = sqrt(t);
            absres0 = std::max(SMALLREAL, r_normb);
            relres = r_normb / absres0;
            break;
        }
        case STOP_MOD_REL_RES: {
            double nu = 0.0;
            HZB_TRY(norm2_host(S, g, x, &nu));
            absres0 = r_norm;
            relres = absres0 / std::max(SMALLREAL, nu);
            break;
        }
        default:
            printf("### ERROR: Unrecognised stopping type for dcsr_pvgmres!\n");
            goto finished;
        }
        if (relres < tol || absres0 < 1e-3 * tol) goto finished;
        print_head(prtlvl, stop_type, relres, absres0);
        norms[0] = relres;
    } else {
        HZB_TRY(norm2_host(S, g, b, &b_norm));
        norms[0] = r_norm;
        den_norm = b_norm > 0.0 ? b_norm : r_norm;
        epsilon = tol * den_norm;
        if (r_norm < epsilon || r_norm < 1e-3 * tol) goto finished;
        print_head(prtlvl, stop_type, b_norm > 0.0 ? r_norm / b_norm : r_norm, r_norm);
    }

    while (iter < MaxIt) {
        rs[0] = r_norm_old = r_norm;
        if (flexible && r_norm == 0.0) {
            if (relres_out) *relres_out = 0.0;
            return iter;
        }
        // adjust the restart length (Baker, Jessup and Kolev)
        if (cr > cr_max || iter == 0) {
            Restart = restart_max;
        } else if (cr < cr_min) {
            // keep it
        } else if (Restart - d > restart_min) {
            Restart -= d;
        } else {
            Restart = restart_max;
        }
        Restart = std::min(Restart, g.restart);
        k_gm_scale<<<grid_for(n), 256, 0, s>>>(n, 1.0 / r_norm, g.p[0]);
        count_launch();
        i = 0;
        while (i < Restart && iter < MaxIt) {
            ++i;
            ++iter;
            HZB_TRY(arnoldi(S, g, A, kind, hp, i, flexible ? g.z[i - 1] : g.r, h));
            for (int j = 0; j <= i; ++j) hh[j][i - 1] = h[j];
            for (int j = 1; j < i; ++j) {
                const double t = hh[j - 1][i - 1];
                hh[j - 1][i - 1] = sn[j - 1] * hh[j][i - 1] + c[j - 1] * t;
                hh[j][i - 1] = -sn[j - 1] * t + c[j - 1] * hh[j][i - 1];
            }
            double t = hh[i][i - 1] * hh[i][i - 1];
            t += hh[i - 1][i - 1] * hh[i - 1][i - 1];
            double gamma = sqrt(t);
            if (gamma == 0.0) gamma = epsmac;
            c[i - 1] = hh[i - 1][i - 1] / gamma;
            sn[i - 1] = hh[i][i - 1] / gamma;
            rs[i] = -sn[i - 1] * rs[i - 1];
            rs[i - 1] = c[i - 1] * rs[i - 1];
            hh[i - 1][i - 1] = sn[i - 1] * hh[i][i - 1] + c[i - 1] * hh[i - 1][i - 1];
            r_norm = fabs(rs[i]);
            if (!flexible) {
                absres = r_norm;
                relres = absres / absres0;
                norms[iter] = relres;
                print_row(prtlvl, iter, relres, absres, norms[iter] / norms[iter - 1]);
                if (relres < tol) break;
            } else {
                norms[iter] = r_norm;
                print_row(prtlvl, iter, b_norm > 0.0 ? norms[iter] / b_norm : norms[iter],
                          norms[iter], norms[iter] / norms[iter - 1]);
                if (r_norm <= epsilon) break;
            }
        }
        // solve the upper triangular system
        rs[i - 1] = rs[i - 1] / hh[i - 1][i - 1];
        for (int k = i - 2; k >= 0; --k) {
            double t = 0.0;
            for (int j = k + 1; j < i; ++j) t -= hh[k][j] * rs[j];
            t += rs[k];
            rs[k] = t / hh[k][k];
        }
        // update the solution
        {
            std::vector<double> cf(rs.begin(), rs.begin() + i);
            if (!flexible) {
                HZB_TRY(combine(S, g, g.d_p, i, cf, g.w));
                HZB_TRY(apply_precond(S, kind, hp, n, g.w, g.r));
            } else {
                HZB_TRY(combine(S, g, g.d_z, i, cf, g.r));
            }
            k_gm_add<<<grid_for(n), 256, 0, s>>>(n, g.r, x);
            count_launch();
        }
        const bool conv = flexible ? r_norm <= epsilon : relres < tol;
        if (conv) {
            // prevent false convergence: the true residual
            const double computed = relres;
            HZB_TRY(spmv<double>(A, SPMV_RES, x, b, g.r, 1.0, nullptr, s));
            HZB_TRY(norm2_host(S, g, g.r, &r_norm));
            double measure = r_norm;
            if (stop_type == STOP_REL_PRECRES) {
                double *dst = flexible ? g.p[0] : g.w;
                HZB_TRY(apply_precond(S, kind, hp, n, g.r, dst));
                double t = 0.0;
                HZB_TRY(dot_host(S, g, dst, g.r, &t));
                measure = sqrt(t);
            }
            double den = flexible ? den_norm : absres0;
            if (stop_type == STOP_MOD_REL_RES) {
                double nu = 0.0;
                HZB_TRY(norm2_host(S, g, x, &nu));
                den = std::max(SMALLREAL, nu);
            }
            if (!flexible) absres = measure;
            relres = measure / den;
            if (!flexible) norms[iter] = relres;
            if (flexible ? relres <= tol : relres < tol) break;
            // restart from the true residual
            HZB_CUDA(cudaMemcpyAsync(g.p[0], g.r, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                     s));
            i = 0;
            if (prtlvl >= PRINT_MORE && !flexible) {
                printf("### WARNING: The computed residual %e is not accurate; "
                       "the true one is %e\n", computed, relres);
            } else if (prtlvl >= PRINT_SOME && flexible) {
                printf("### WARNING: False convergence!\n");
            }
        }
        // the residual direction for the next cycle
        for (int j = i; j > 0; --j) {
            rs[j - 1] = -sn[j - 1] * rs[j];
            rs[j] = c[j - 1] * rs[j];
        }
        if (i) {
            HZB_CUDA(cudaMemcpyAsync(g.coef, rs.data(), (i + 1) * sizeof(double),
                                     cudaMemcpyHostToDevice, s));
            k_gm_residual<<<grid_for(n), 256, 0, s>>>(n, i, g.d_p, g.coef);
            count_launch();
        }
        cr = r_norm / r_norm_old;
    }

finished:
    if (prtlvl > PRINT_NONE) {
        const double rel = flexible ? (den_norm > 0 ? r_norm / den_norm : 0.0) : relres;
        if (iter > MaxIt) {
            printf("### WARNING: MaxIt = %lld reached with relative residual %e.\n",
                   (long long)MaxIt, rel);
        } else if (iter >= 0) {
            printf("Number of iterations = %lld with relative residual %e.\n",
                   (long long)iter, rel);
        }
        fflush(stdout);
    }
    if (relres_out) *relres_out = flexible ? (den_norm > 0 ? r_norm / den_norm : 0.0) : relres;
    HZB_CUDA(cudaStreamSynchronize(s));
    return iter >= MaxIt ? ERROR_SOLVER_MAXIT : iter;
}

}  // namespace hzb
