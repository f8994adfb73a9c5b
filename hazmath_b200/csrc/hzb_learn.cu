// hzb_learn.cu -- the method-generated loss for learned l1-Jacobi weights.
//
// For fine-level weights omega (one per row), the error propagation of one
// V(2,2) cycle is
//     E(omega) = S^2 C S^2,  S = I - W A,  W = diag(omega_i / l1_i),
//     C = I - P B_c R A     (B_c: the plain V-cycle below level 0),
// and the loss of an error vector e is the A-norm contraction of two cycles,
//     L(e) = ||E^2 e||_A^2 / ||e||_A^2.
// Its gradient follows from the adjoints S^T = I - A W and C^T = I - A P B_c R
// (B_c is symmetric: its pre and post smoothing are the same l1 sweeps):
//     g_final = 2 A e_final / ||e||_A^2,
//     through a sweep e_out = e_in - W A e_in:
//         dL/domega_i += -g_out_i (A e_in)_i / l1_i,   g_in = g_out - A W g_out,
//     through C: g_in = g_out - A P B_c R g_out.
// Training errors are those the plain method leaves: random vectors smoothed
// by three plain l1 sweeps, then two plain V-cycles, normalised in the A-norm.
// Everything runs in FP64 on the solver's stream with the cycle kernels.
#include <cmath>
#include "hzb_solver.cuh"
#include <vector>

namespace hzb {

__device__ __forceinline__ double hash_unit(unsigned long long seed, unsigned long long i) {
    unsigned long long x = seed * 0x9E3779B97F4A7C15ull + i * 0xBF58476D1CE4E5B9ull + 1;
    x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27; x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;   // U[-1,1)
}

__global__ void k_rand(int n, unsigned long long seed, double *e) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        e[i] = hash_unit(seed, (unsigned long long)i);
}

// e -= (omega_i / l1_i) * Ae_i   (omega == nullptr: plain weight 1)
__global__ void k_err_sweep(int n, const float *__restrict__ omega,
                            const double *__restrict__ l1, const double *__restrict__ Ae,
                            double *e) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const double w = (omega ? (double)omega[i] : 1.0) / l1[i];
        e[i] -= w * Ae[i];
    }
}

// adjoint of a sweep, first half: dom_i -= g_i Ae_i / l1_i ; t = W g
__global__ void k_err_sweep_adj(int n, const float *__restrict__ omega,
                                const double *__restrict__ l1,
                                const double *__restrict__ Ae,
                                const double *__restrict__ g, double *t, double *dom) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const double inv = 1.0 / l1[i];
        dom[i] -= g[i] * Ae[i] * inv;
        t[i] = (omega ? (double)omega[i] : 1.0) * inv * g[i];
    }
}

__global__ void k_sub(int n, const double *__restrict__ t, double *e) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        e[i] -= t[i];
}

// x *= f / den[0]
__global__ void k_scale_by(int n, const double *__restrict__ den, double f, double *x) {
    const double s = f / den[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        x[i] *= s;
}
__global__ void k_scale_rsqrt(int n, const double *__restrict__ num, double *x) {
    const double s = 1.0 / sqrt(num[0]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        x[i] *= s;
}
__global__ void k_to_float(int n, const double *__restrict__ d, double f, float *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x)
        out[i] = (float)(d[i] * f);
}

constexpr int LEARN_MAX_CYCLES = 16;

struct LearnWork {
    int n = 0;
    double *r = nullptr, *t = nullptr, *g = nullptr, *l1 = nullptr, *e = nullptr;
    double *dom = nullptr, *sc = nullptr, *part = nullptr;
    std::vector<double *> Ae;   // A e before each of the 4 sweeps of every cycle
    int alloc(int nn, int ncyc = 0) {
        n = nn;
        HZB_TRY(dalloc(&r, n)); HZB_TRY(dalloc(&t, n)); HZB_TRY(dalloc(&g, n));
        HZB_TRY(dalloc(&l1, n)); HZB_TRY(dalloc(&e, n)); HZB_TRY(dalloc(&dom, n));
        Ae.assign(4 * (size_t)ncyc, nullptr);
        for (auto &p : Ae) HZB_TRY(dalloc(&p, n));
        HZB_TRY(dalloc(&sc, 8));
        HZB_TRY(dalloc(&part, reduce_blocks(n) + 8));
        return SUCCESS;
    }
    ~LearnWork() {
        dfree(r); dfree(t); dfree(g); dfree(l1); dfree(e); dfree(dom); dfree(sc); dfree(part);
        for (auto &p : Ae) dfree(p);
    }
};

static AMG_param plain_cycle(hzb_solver *S) {
    AMG_param c = S->pc_cyc;
    c.maxit = 1;
    return c;
}

// x_1 = B_c b_1 on the levels below 0
static int coarse_apply(hzb_solver *S) {
    Level &L1 = S->lv[1];
    HZB_TRY(vzero<double>(L1.n, L1.x, S->s));
    if (S->nl == 2) return dense_gemv<double>(L1.n, S->Ainv, L1.b, L1.x, S->s);
    return cycle64(S, plain_cycle(S), 1);
}

// e <- e - P B_c R (A e)       (forward coarse correction)
static int coarse_correct(hzb_solver *S, LearnWork &w, double *e) {
    Level &L0 = S->lv[0], &L1 = S->lv[1];
    HZB_TRY(spmv<double>(L0.A64(), SPMV_Y, e, nullptr, w.r, 1.0, nullptr, S->s));
    HZB_TRY(restrict_level(S, 0, w.r, L1.b));
    HZB_TRY(coarse_apply(S));
    return prolong_level(S, 0, L1.x, e, -1.0);
}

// g <- g - A P B_c R g          (adjoint coarse correction)
static int coarse_correct_adj(hzb_solver *S, LearnWork &w, double *g) {
    Level &L0 = S->lv[0], &L1 = S->lv[1];
    HZB_TRY(restrict_level(S, 0, g, L1.b));
    HZB_TRY(coarse_apply(S));
    HZB_TRY(vzero<double>(L0.n, w.t, S->s));
    HZB_TRY(prolong_level(S, 0, L1.x, w.t, 1.0));
    return spmv<double>(L0.A64(), SPMV_AXPY, w.t, nullptr, g, -1.0, nullptr, S->s);
}

// out_dev[0] = e^T A e  (A e left in w.r)
static int anorm2(hzb_solver *S, LearnWork &w, const double *e, double *out_dev) {
    HZB_TRY(spmv<double>(S->lv[0].A64(), SPMV_Y, e, nullptr, w.r, 1.0, nullptr, S->s));
    return dot(S->lv[0].n, e, w.r, w.part, out_dev, S->s);
}

static int need_levels(hzb_solver *S) {
    if (S->nl < 2) {
        set_error_msg("learned weights need a hierarchy of at least two levels");
        return ERROR_INPUT_PAR;
    }
    const int sm = S->amg.smoother;
    if (sm != SMOOTHER_L1DIAG) {
        set_error_msg("learned weights apply to the l1-Jacobi smoother");
        return ERROR_AMG_SMOOTH_TYPE;
    }
    return SUCCESS;
}

// omega == nullptr: errors of the plain cycle; otherwise the two V-cycles
// use omega on the fine level (the errors the learned cycle leaves).
int learn_errors(hzb_solver *S, int ns, unsigned long long seed, double *E,
                 const float *omega, int ncyc) {
    if (ncyc < 0 || ncyc > LEARN_MAX_CYCLES) return ERROR_INPUT_PAR;
    HZB_TRY(need_levels(S));
    Level &L0 = S->lv[0];
    const int n = L0.n;
    cudaStream_t s = S->s;
    LearnWork w;
    HZB_TRY(w.alloc(n));
    HZB_TRY(l1_norms<double>(L0.A64(), w.l1, s));
    const bool was = S->omega_active;
    float *was_om = S->omega;
    const short was_graph = S->bp.use_graph;
    S->bp.use_graph = 0;   // omega's address is not part of a captured cycle
    S->omega = const_cast<float *>(omega);
    S->omega_active = omega != nullptr;
    const AMG_param cyc = plain_cycle(S);
    int rc = SUCCESS;
    const int g = grid_for(n);
    for (int k = 0; k < ns && !rc; ++k) {
        double *e = E + (size_t)k * n;
        k_rand<<<g, 256, 0, s>>>(n, seed + 7919ull * (unsigned long long)k, e);
        count_launch();
        for (int it = 0; it < 3 && !rc; ++it) {   // smooth it: plain l1 sweeps
            rc = spmv<double>(L0.A64(), SPMV_Y, e, nullptr, w.r, 1.0, nullptr, s);
            k_err_sweep<<<g, 256, 0, s>>>(n, nullptr, w.l1, w.r, e);
            count_launch();
        }
        for (int it = 0; it < ncyc && !rc; ++it) {   // cycles: e <- e - B A e
            rc = spmv<double>(L0.A64(), SPMV_Y, e, nullptr, w.g, 1.0, nullptr, s);
            if (!rc) rc = precond64(S, w.g, w.t, cyc);
            if (!rc) {
                k_sub<<<g, 256, 0, s>>>(n, w.t, e);
                count_launch();
            }
        }
        if (!rc) rc = anorm2(S, w, e, w.sc);
        if (!rc) {
            k_scale_rsqrt<<<g, 256, 0, s>>>(n, w.sc, e);
            count_launch();
        }
    }
    S->omega_active = was;
    S->omega = was_om;
    S->bp.use_graph = was_graph;
    if (!rc) HZB_CUDA(cudaStreamSynchronize(s));
    return rc;
}

int learn_loss_grad(hzb_solver *S, const float *omega, int ns, const double *E, int ncyc,
                    double *loss, float *domega) {
    if (ncyc < 1 || ncyc > LEARN_MAX_CYCLES) return ERROR_INPUT_PAR;
    HZB_TRY(need_levels(S));
    Level &L0 = S->lv[0];
    const int n = L0.n;
    const DCsr<double> A = L0.A64();
    cudaStream_t s = S->s;
    const int g = grid_for(n);
    const bool grad = domega != nullptr;   // without it: the loss alone
    LearnWork w;
    HZB_TRY(w.alloc(n, grad ? ncyc : 0));
    HZB_TRY(l1_norms<double>(A, w.l1, s));
    HZB_TRY(vzero<double>(n, w.dom, s));
    double total = 0.0;
    for (int k = 0; k < ns; ++k) {
        HZB_TRY(vcopy<double>(n, E + (size_t)k * n, w.e, s));
        HZB_TRY(anorm2(S, w, w.e, w.sc + 0));          // ||e||_A^2
        int q = 0;
        for (int cyc = 0; cyc < ncyc; ++cyc) {         // forward, storing A e_in
            for (int half = 0; half < 2; ++half) {
                if (half) HZB_TRY(coarse_correct(S, w, w.e));
                for (int j = 0; j < 2; ++j, ++q) {
                    double *Ae = grad ? w.Ae[q] : w.t;
                    HZB_TRY(spmv<double>(A, SPMV_Y, w.e, nullptr, Ae, 1.0, nullptr, s));
                    k_err_sweep<<<g, 256, 0, s>>>(n, omega, w.l1, Ae, w.e);
                    count_launch();
                }
            }
        }
        HZB_TRY(anorm2(S, w, w.e, w.sc + 1));          // ||E^k e||_A^2, A e in w.r
        if (!grad) {
            double h[2];
            HZB_CUDA(cudaMemcpyAsync(h, w.sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
            HZB_CUDA(cudaStreamSynchronize(s));
            total += h[1] / h[0];
            continue;
        }
        HZB_TRY(vcopy<double>(n, w.r, w.g, s));        // g = 2 A e / ||e0||_A^2
        k_scale_by<<<g, 256, 0, s>>>(n, w.sc + 0, 2.0, w.g);
        count_launch();
        for (int cyc = ncyc - 1; cyc >= 0; --cyc) {    // backward
            for (int j = 0; j < 2; ++j) {
                --q;
                k_err_sweep_adj<<<g, 256, 0, s>>>(n, omega, w.l1, w.Ae[q], w.g, w.t, w.dom);
                count_launch();
                HZB_TRY(spmv<double>(A, SPMV_AXPY, w.t, nullptr, w.g, -1.0, nullptr, s));
            }
            HZB_TRY(coarse_correct_adj(S, w, w.g));
            for (int j = 0; j < 2; ++j) {
                --q;
                k_err_sweep_adj<<<g, 256, 0, s>>>(n, omega, w.l1, w.Ae[q], w.g, w.t, w.dom);
                count_launch();
                HZB_TRY(spmv<double>(A, SPMV_AXPY, w.t, nullptr, w.g, -1.0, nullptr, s));
            }
        }
        double h[2];
        HZB_CUDA(cudaMemcpyAsync(h, w.sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        HZB_CUDA(cudaStreamSynchronize(s));
        total += h[1] / h[0];
    }
    // gradient of the mean over samples; the FP64 sum of the per-sample
    // gradients is divided by ns once
    if (grad) {
        k_to_float<<<g, 256, 0, s>>>(n, w.dom, 1.0 / ns, domega);
        count_launch();
        HZB_CUDA(cudaStreamSynchronize(s));
    }
    *loss = total / ns;
    return SUCCESS;
}

int cycle_contraction(hzb_solver *S, int ns, unsigned long long seed, double *loss) {
    if (ns < 1) return ERROR_INPUT_PAR;
    HZB_TRY(need_levels(S));
    Level &L0 = S->lv[0];
    const int n = L0.n;
    const DCsr<double> A = L0.A64();
    cudaStream_t s = S->s;
    const int g = grid_for(n);
    KrylovWork &kw = S->kw;   // r, z as the preconditioner's operands (its graph key)
    if (kw.n != n) HZB_TRY(kw.alloc(n));
    LearnWork w;
    HZB_TRY(w.alloc(n));
    HZB_TRY(l1_norms<double>(A, w.l1, s));
    double total = 0.0;
    for (int k = 0; k < ns; ++k) {
        k_rand<<<g, 256, 0, s>>>(n, seed + 7919ull * (unsigned long long)k, w.e);
        count_launch();
        for (int it = 0; it < 3; ++it) {   // plain l1 sweeps
            HZB_TRY(spmv<double>(A, SPMV_Y, w.e, nullptr, w.t, 1.0, nullptr, s));
            k_err_sweep<<<g, 256, 0, s>>>(n, nullptr, w.l1, w.t, w.e);
            count_launch();
        }
        for (int it = 0; it < 4; ++it) {   // e <- e - B A e, twice, then twice measured
            if (it == 2) HZB_TRY(anorm2(S, w, w.e, w.sc + 0));
            HZB_TRY(spmv<double>(A, SPMV_Y, w.e, nullptr, kw.r, 1.0, nullptr, s));
            HZB_TRY(solver_precond(S, kw.r, kw.z));
            k_sub<<<g, 256, 0, s>>>(n, kw.z, w.e);
            count_launch();
        }
        HZB_TRY(anorm2(S, w, w.e, w.sc + 1));
        double h[2];
        HZB_CUDA(cudaMemcpyAsync(h, w.sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        HZB_CUDA(cudaStreamSynchronize(s));
        total += h[1] / h[0];
    }
    *loss = total / ns;
    return SUCCESS;
}

// The contraction loss above is ||E^k e||_A^2 / ||e||_A^2 with e given, whose
// gradient dom accumulates d/domega of each sample's ratio with ||e||_A
// fixed (e does not depend on omega).

}  // namespace hzb
