// hzb_api.cu -- the exported C ABI: HAZmath drop-in entry points, the
// persistent solver handle and the kernel-level entry points.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include "hzb_solver.cuh"

using namespace hzb;

// ---------------------------------------------------------------------------
// parameters (src/utilities/parameters.c, src/utilities/data.c)
// ---------------------------------------------------------------------------
extern "C" void param_amg_init(AMG_param *p) {
    // parameters.c:158-205
    p->AMG_type = UA_AMG;
    p->print_level = PRINT_NONE;
    p->maxit = 1;
    p->tol = 1e-6;
    p->max_levels = 10;
    p->coarse_dof = 200;
    p->cycle_type = W_CYCLE;
    p->smoother = SMOOTHER_GS;
    p->presmooth_iter = 1;
    p->postsmooth_iter = 1;
    p->coarse_solver = SOLVER_DEFAULT;
    p->relaxation = 1.0;
    p->polynomial_degree = 2;
    p->coarse_scaling = OFF;
    p->amli_degree = 2;
    p->amli_coef = NULL;
    p->nl_amli_krylov_type = SOLVER_VFGMRES;
    p->fpwr = 1.0;
    p->aggregation_type = HEC;
    p->strong_coupled = 0.04;
    p->max_aggregation = 20;
    p->tentative_smooth = 0.67;
    p->smooth_filter = ON;
    p->Schwarz_levels = 0;
    p->Schwarz_mmsize = 200;
    p->Schwarz_maxlvl = -1;
    p->Schwarz_type = 1;
    p->Schwarz_blksolver = SOLVER_UMFPACK;
    p->HAZDIR = NULL;
    p->Schwarz_on_blk = NULL;
    p->Schwarz_patch_type = NULL;
    p->damping_param = 1.0;
    p->BSR_alpha = -1000.;
    p->BSR_omega = -1000.;
}

extern "C" void param_linear_solver_init(linear_itsolver_param *p) {
    // parameters.c:238-250
    p->linear_print_level = 0;
    p->linear_itsolver_type = SOLVER_VFGMRES;
    p->linear_precond_type = PREC_NULL;
    p->linear_stop_type = STOP_REL_RES;
    p->linear_maxit = 500;
    p->linear_restart = 100;
    p->linear_tol = 1e-6;
    p->HX_smooth_iter = 1;
}

extern "C" void precond_data_null(precond_data *d) {
    // data.c:22-55
    d->AMG_type = UA_AMG;
    d->print_level = PRINT_MIN;
    d->maxit = 100;
    d->max_levels = 20;
    d->tol = 1e-8;
    d->cycle_type = V_CYCLE;
    d->smoother = SMOOTHER_GS;
    d->presmooth_iter = 1;
    d->postsmooth_iter = 1;
    d->relaxation = 1.2;
    d->polynomial_degree = 2;
    d->coarse_solver = SOLVER_UMFPACK;
    d->coarse_scaling = OFF;
    d->amli_degree = 2;
    d->nl_amli_krylov_type = SOLVER_VFGMRES;
    d->fpwr = 1.0;
    d->amli_coef = NULL;
    d->mgl_data = NULL;
    d->A = NULL;
    d->A_nk = NULL;
    d->P_nk = NULL;
    d->R_nk = NULL;
    d->r = NULL;
    d->w = NULL;
}

extern "C" void param_amg_to_prec(precond_data *d, AMG_param *p) {
    // parameters.c:604-640
    d->AMG_type = p->AMG_type;
    d->print_level = p->print_level;
    d->maxit = p->maxit;
    d->max_levels = p->max_levels;
    d->tol = p->tol;
    d->cycle_type = p->cycle_type;
    d->smoother = p->smoother;
    d->presmooth_iter = p->presmooth_iter;
    d->postsmooth_iter = p->postsmooth_iter;
    d->coarse_solver = p->coarse_solver;
    d->relaxation = p->relaxation;
    d->polynomial_degree = p->polynomial_degree;
    d->coarse_scaling = p->coarse_scaling;
    d->amli_degree = p->amli_degree;
    d->nl_amli_krylov_type = p->nl_amli_krylov_type;
    d->fpwr = p->fpwr;
    if (p->amli_coef) {
        d->amli_coef = (REAL *)calloc(p->amli_degree + 1, sizeof(REAL));
        memcpy(d->amli_coef, p->amli_coef, (p->amli_degree + 1) * sizeof(REAL));
    }
}

extern "C" void param_prec_to_amg(AMG_param *p, precond_data *d) {
    // parameters.c:649-680 (tol, maxit, max_levels are not transferred)
    p->AMG_type = d->AMG_type;
    p->print_level = d->print_level;
    p->cycle_type = d->cycle_type;
    p->smoother = d->smoother;
    p->presmooth_iter = d->presmooth_iter;
    p->postsmooth_iter = d->postsmooth_iter;
    p->relaxation = d->relaxation;
    p->polynomial_degree = d->polynomial_degree;
    p->coarse_solver = d->coarse_solver;
    p->coarse_scaling = d->coarse_scaling;
    p->amli_degree = d->amli_degree;
    p->nl_amli_krylov_type = d->nl_amli_krylov_type;
    p->fpwr = d->fpwr;
    if (d->amli_coef) {
        p->amli_coef = (REAL *)calloc(d->amli_degree + 1, sizeof(REAL));
        memcpy(p->amli_coef, d->amli_coef, (d->amli_degree + 1) * sizeof(REAL));
    }
}

extern "C" void hzb_param_init(hzb_param *p) {
    memset(p, 0, sizeof(*p));
    p->precision = HZB_PREC_FP64;
    p->gs_schedule = HZB_GS_EXACT;
    p->matching = HZB_MATCH_EXACT;
    p->export_hierarchy = 1;
    p->use_omega = 0;
    p->omega = NULL;
    p->device = 0;
    p->fallback_check = 0;
    p->use_graph = 1;
}

extern "C" const char *hzb_last_error(void) { return hzb::last_error(); }

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
static AMG_param cycle_param_of(const AMG_param &amg) {
    // what precond_amg hands to mgcycle: defaults overwritten by the
    // precond_data copy of amgparam (precond.c:171-172)
    AMG_param c;
    param_amg_init(&c);
    precond_data d;
    precond_data_null(&d);
    AMG_param a = amg;
    a.amli_coef = NULL;
    param_amg_to_prec(&d, &a);
    param_prec_to_amg(&c, &d);
    c.maxit = amg.maxit;
    return c;
}

extern "C" INT hzb_create(hzb_solver **out, const AMG_param *amg,
                          const linear_itsolver_param *it, const hzb_param *bp) {
    *out = nullptr;
    hzb_solver *S = new (std::nothrow) hzb_solver();
    if (!S) return ERROR_ALLOC_MEM;
    if (amg) S->amg = *amg; else param_amg_init(&S->amg);
    if (it) S->it = *it; else param_linear_solver_init(&S->it);
    if (bp) S->bp = *bp; else hzb_param_init(&S->bp);
    S->pc_cyc = cycle_param_of(S->amg);
    cudaError_t e = cudaSetDevice(S->bp.device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&S->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&S->e1);
    if (e != cudaSuccess) {
        set_error(e, __FILE__, __LINE__);
        delete S;
        return ERROR_SOLVER_MISC;
    }
    *out = S;
    return SUCCESS;
}

extern "C" void hzb_destroy(hzb_solver *S) {
    if (!S) return;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    if (S->s) cudaStreamSynchronize(S->s);
    hzb::destroy(S);
    if (S->e0) cudaEventDestroy(S->e0);
    if (S->e1) cudaEventDestroy(S->e1);
    if (S->s) cudaStreamDestroy(S->s);
    delete S;
}

static int check_csr_host(int n, int nnz, const int *ia) {
    if (n <= 0 || nnz <= 0 || !ia) return ERROR_MAT_SIZE;
    if (ia[0] != 0 || ia[n] != nnz) return ERROR_DATA_STRUCTURE;
    return SUCCESS;
}

static int upload_omega(hzb_solver *S) {
    if (!(S->bp.use_omega && S->bp.omega)) return SUCCESS;
    const int n = S->lv[0].n;
    if (!S->omega) HZB_TRY(dalloc(&S->omega, n));
    HZB_CUDA(cudaMemcpyAsync(S->omega, S->bp.omega, sizeof(float) * n,
                             cudaMemcpyHostToDevice, S->s));
    S->omega_active = true;
    return SUCCESS;
}

extern "C" INT hzb_setup_device(hzb_solver *S, INT n, INT nnz, const INT *d_ia,
                                const INT *d_ja, const REAL *d_val) {
    if (!S || n <= 0 || nnz <= 0) return ERROR_MAT_SIZE;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    S->host_ia = nullptr; S->host_ja = nullptr; S->host_val = nullptr;
    HZB_TRY(hzb::setup(S, n, nnz, d_ia, d_ja, d_val, false));
    return upload_omega(S);
}

extern "C" INT hzb_setup_host(hzb_solver *S, const dCSRmat *A) {
    if (!S || !A) return ERROR_INPUT_PAR;
    if (A->row != A->col) return ERROR_MAT_SIZE;
    HZB_TRY(check_csr_host(A->row, A->nnz, A->IA));
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    HZB_TRY(hzb::setup(S, A->row, A->nnz, A->IA, A->JA, A->val, true));
    S->host_ia = A->IA; S->host_ja = A->JA; S->host_val = A->val;
    return upload_omega(S);
}

extern "C" INT hzb_set_omega_device(hzb_solver *S, const float *d_omega) {
    if (!S || S->nl == 0) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    if (!d_omega) { S->omega_active = false; return SUCCESS; }
    const int n = S->lv[0].n;
    if (!S->omega) HZB_TRY(dalloc(&S->omega, n));
    HZB_CUDA(cudaMemcpyAsync(S->omega, d_omega, sizeof(float) * n,
                             cudaMemcpyDeviceToDevice, S->s));
    S->omega_active = true;
    return SUCCESS;
}

extern "C" INT hzb_solve_device(hzb_solver *S, const REAL *d_b, REAL *d_x) {
    if (!S || S->nl == 0) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const long long l0 = hzb::launch_count();
    HZB_CUDA(cudaEventRecord(S->e0, S->s));
    double rel = 0.0, cond = 0.0;
    int it;
    const int prt = S->it.linear_print_level;
    // the preconditioner of linear_solver_dcsr_krylov_amg for the cycle type
    const int kind = pc_kind_of_cycle(S->pc_cyc.cycle_type);
    if (S->bp.precision == HZB_PREC_MIXED) {
        if (kind != PC_AMG) {
            set_error_msg("the mixed-precision solve runs V and W cycles (cycle_type 1, 2)");
            return ERROR_INPUT_PAR;
        }
        it = fcg_mixed(S, d_b, d_x, S->it.linear_tol, S->it.linear_maxit, prt, &rel);
    } else if (S->it.linear_itsolver_type == SOLVER_CG) {
        it = pcg(S, S->lv[0].A64(), d_b, d_x, kind, nullptr, S->it.linear_tol,
                 S->it.linear_maxit, S->it.linear_stop_type, prt, S->kw, &rel, &cond);
    } else if (S->it.linear_itsolver_type == SOLVER_VGMRES ||
               S->it.linear_itsolver_type == SOLVER_VFGMRES) {
        it = gmres(S, S->lv[0].A64(), d_b, d_x, kind, nullptr, S->it.linear_tol,
                   S->it.linear_maxit, S->it.linear_restart, S->it.linear_stop_type, prt,
                   S->it.linear_itsolver_type == SOLVER_VFGMRES, &rel);
    } else if (S->it.linear_itsolver_type == SOLVER_MinRes) {
        it = minres(S, S->lv[0].A64(), d_b, d_x, kind, nullptr, S->it.linear_tol,
                    S->it.linear_maxit, S->it.linear_stop_type, prt, &rel);
    } else {
        set_error_msg("Krylov types 1 (CG), 2 (MINRES), 3 (GMRES) and 4 (flexible GMRES) "
                      "are the ones solver_dcsr_linear_itsolver dispatches");
        return ERROR_SOLVER_TYPE;
    }
    HZB_CUDA(cudaEventRecord(S->e1, S->s));
    HZB_CUDA(cudaEventSynchronize(S->e1));
    if (it >= 0) {
        const int wc = check_waits(S);
        if (wc) it = wc;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, S->e0, S->e1);
    S->st.solve_seconds = ms * 1e-3;
    S->st.iterations = it;
    S->st.final_relres = rel;
    S->st.condest = cond;
    S->st.launches = (INT)(hzb::launch_count() - l0);
    return it;
}

extern "C" INT hzb_batch_setup_device(hzb_solver *S, INT nsys, const INT *off, INT n,
                                      INT nnz, const INT *d_ia, const INT *d_ja,
                                      const REAL *d_val) {
    if (!S || n <= 0 || nnz <= 0) return ERROR_MAT_SIZE;
    if (pc_kind_of_cycle(S->pc_cyc.cycle_type) != PC_AMG) {
        set_error_msg("batched solves run V and W cycles (cycle_type 1, 2)");
        return ERROR_INPUT_PAR;
    }
    if (S->amg.AMG_type == SA_AMG) {
        set_error_msg("batched solves run unsmoothed aggregation");
        return ERROR_INPUT_PAR;
    }
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    S->host_ia = nullptr; S->host_ja = nullptr; S->host_val = nullptr;
    HZB_CUDA(cudaEventRecord(S->e0, S->s));
    HZB_TRY(hzb::batch_setup(S, nsys, off, n, nnz, d_ia, d_ja, d_val));
    HZB_CUDA(cudaEventRecord(S->e1, S->s));
    HZB_CUDA(cudaEventSynchronize(S->e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, S->e0, S->e1);
    S->st.setup_seconds = ms * 1e-3;
    return upload_omega(S);
}

extern "C" INT hzb_batch_solve_device(hzb_solver *S, const REAL *d_b, REAL *d_x,
                                      INT *iters, REAL *relres, REAL *seconds) {
    if (!S || S->nl == 0 || !S->batch) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const long long l0 = hzb::launch_count();
    HZB_CUDA(cudaEventRecord(S->e0, S->s));
    const int it = hzb::batch_solve(S, d_b, d_x, S->it.linear_tol, S->it.linear_maxit, iters,
                                    relres, seconds);
    HZB_CUDA(cudaEventRecord(S->e1, S->s));
    HZB_CUDA(cudaEventSynchronize(S->e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, S->e0, S->e1);
    S->st.solve_seconds = ms * 1e-3;
    S->st.iterations = it;
    S->st.launches = (INT)(hzb::launch_count() - l0);
    return it;
}

extern "C" INT hzb_solve_host(hzb_solver *S, const REAL *b, REAL *x) {
    if (!S || S->nl == 0) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const int n = S->lv[0].n;
    double *db = nullptr, *dx = nullptr;
    HZB_TRY(dalloc(&db, n));
    int rc = dalloc(&dx, n);
    if (rc) { dfree(db); return rc; }
    cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyHostToDevice, S->s);
    cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, S->s);
    int it = hzb_solve_device(S, db, dx);
    cudaError_t e = cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, S->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->s);
    dfree(db);
    dfree(dx);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
    return it;
}

extern "C" INT hzb_precond_device(hzb_solver *S, const REAL *d_r, REAL *d_z) {
    if (!S || S->nl == 0) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    HZB_TRY(apply_precond(S, pc_kind_of_cycle(S->pc_cyc.cycle_type), nullptr, S->lv[0].n, d_r,
                          d_z));
    HZB_CUDA(cudaStreamSynchronize(S->s));
    return check_waits(S);
}

extern "C" INT hzb_time_kernel(hzb_solver *S, INT which, INT level, INT reps,
                               REAL *ms_per_launch, REAL *bytes_per_launch) {
    if (S && which >= HZB_K_BSR_RES && which <= HZB_K_BSR_GS) {
        cudaSetDevice(S->bp.device);
        StreamScope scope_(S->s);
        return hzb::bsr_time_kernel(S, which, level, reps, ms_per_launch, bytes_per_launch);
    }
    if (!S || level < 0 || level >= S->nl || reps < 1) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    Level &L = S->lv[level];
    const bool f32 = which == HZB_K_SPMV32 || which == HZB_K_L1_32;
    if (f32 && !L.val32) HZB_TRY(ensure_fp32(S));
    const double vb = f32 ? 4.0 : 8.0;
    // the FP32 kernels read the zero-free copy
    const double n = L.n, nnz = f32 ? L.nnz32 : L.nnz;
    double bytes = nnz * (vb + 4.0) + 4.0 * (n + 1);
    switch (which) {
    case HZB_K_SPMV64: case HZB_K_SPMV32: bytes += 2 * vb * n; break;     // x, y
    case HZB_K_RES64: bytes += 3 * vb * n; break;                        // x, b, w
    case HZB_K_L1_32: case HZB_K_L1_64: bytes += 3 * vb * n; break;      // x, b, xn
    case HZB_K_GS64:
        if (level >= S->nl - 1) return ERROR_INPUT_PAR;   // the coarsest is not smoothed
        bytes += 4 * vb * n;                                // b, 1/d, x read and written
        break;
    default: return ERROR_INPUT_PAR;
    }
    // the FP32 sweep of level 0 runs with the learned weights when the
    // solve does (as smooth32 passes them), and reads them
    const float *om = (which == HZB_K_L1_32 && level == 0 && S->omega_active) ? S->omega
                                                                             : nullptr;
    if (om) bytes += 4.0 * n;
    auto launch = [&]() -> int {
        switch (which) {
        case HZB_K_SPMV64:
            return spmv<double>(L.A64(), SPMV_Y, L.x, nullptr, L.w, 1.0, nullptr, S->s);
        case HZB_K_SPMV32:
            return spmv<float>(L.A32(), SPMV_Y, L.x32, nullptr, L.w32, 1.0f, nullptr, S->s);
        case HZB_K_RES64:
            return spmv<double>(L.A64(), SPMV_RES, L.x, L.b, L.w, 1.0, nullptr, S->s);
        case HZB_K_L1_32:
            return l1_sweep<float>(L.A32(), L.b32, L.x32, L.t32, om, S->s);
        case HZB_K_GS64:
            return time_gs_sweep(S, level);
        default:
            return l1_sweep<double>(L.A64(), L.b, L.x, L.t, nullptr, S->s);
        }
    };
    HZB_TRY(launch());
    HZB_CUDA(cudaEventRecord(S->e0, S->s));
    for (int r = 0; r < reps; ++r) HZB_TRY(launch());
    HZB_CUDA(cudaEventRecord(S->e1, S->s));
    HZB_CUDA(cudaEventSynchronize(S->e1));
    float ms = 0.f;
    HZB_CUDA(cudaEventElapsedTime(&ms, S->e0, S->e1));
    *ms_per_launch = ms / reps;
    *bytes_per_launch = bytes;
    return SUCCESS;
}

extern "C" INT hzb_get_stats(const hzb_solver *S, hzb_stats *st) {
    if (!S || !st) return ERROR_INPUT_PAR;
    *st = S->st;
    return SUCCESS;
}

extern "C" INT hzb_level_copy(const hzb_solver *S, INT l, INT *ia, INT *ja,
                              REAL *val, INT *agg) {
    if (!S || l < 0 || l >= S->nl) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const Level &L = S->lv[l];
    // the coarsest level is reported as the reference leaves it: transposed
    // when the direct coarse solver is used
    const int *sia = L.tia ? L.tia : L.ia, *sja = L.tia ? L.tja : L.ja;
    const double *sval = L.tia ? L.tval : L.val;
    if (ia) HZB_CUDA(cudaMemcpy(ia, sia, sizeof(int) * (L.n + 1), cudaMemcpyDeviceToHost));
    if (ja) HZB_CUDA(cudaMemcpy(ja, sja, sizeof(int) * L.nnz, cudaMemcpyDeviceToHost));
    if (val) HZB_CUDA(cudaMemcpy(val, sval, sizeof(double) * L.nnz, cudaMemcpyDeviceToHost));
    if (agg) {
        if (l < S->nl - 1)
            HZB_CUDA(cudaMemcpy(agg, L.agg, sizeof(int) * L.n, cudaMemcpyDeviceToHost));
        else
            for (int i = 0; i < L.n; ++i) agg[i] = -1;
    }
    return SUCCESS;
}

// ---------------------------------------------------------------------------
// drop-in: AMG_data life cycle and setup
// ---------------------------------------------------------------------------
extern "C" AMG_data *amg_data_create(SHORT max_levels) {
    // data.c:66-91
    if (max_levels < 1) max_levels = 1;
    AMG_data *mgl = (AMG_data *)calloc(max_levels, sizeof(AMG_data));
    for (int i = 0; i < max_levels; ++i) {
        mgl[i].max_levels = max_levels;
        mgl[i].num_levels = 0;
        mgl[i].near_kernel_dim = 0;
        mgl[i].near_kernel_basis = NULL;
        mgl[i].cycle_type = 0;
    }
    return mgl;
}

static void free_csr(dCSRmat *A) {
    free(A->IA); free(A->JA); free(A->val);
    A->IA = NULL; A->JA = NULL; A->val = NULL;
    A->row = A->col = A->nnz = 0;
}
static void free_vec(dvector *v) {
    free(v->val);
    v->val = NULL;
    v->row = 0;
}

extern "C" void amg_data_free(AMG_data *mgl, AMG_param *param) {
    // data.c:96-140 (the hierarchy handle in mgl[0].wdata is released too)
    if (!mgl) return;
    const int nl = mgl[0].num_levels > 1 ? mgl[0].num_levels : 1;
    for (int i = 0; i < nl; ++i) {
        free_csr(&mgl[i].A);
        free_csr(&mgl[i].P);
        free_csr(&mgl[i].R);
        free_csr(&mgl[i].M);
        free_vec(&mgl[i].b);
        free_vec(&mgl[i].x);
        free_vec(&mgl[i].w);
    }
    for (int i = 0; i < mgl->near_kernel_dim; ++i) {
        free(mgl->near_kernel_basis[i]);
        mgl->near_kernel_basis[i] = NULL;
    }
    free(mgl->near_kernel_basis);
    mgl->near_kernel_basis = NULL;
    if (mgl[0].wdata) {
        hzb_destroy((hzb_solver *)mgl[0].wdata);
        mgl[0].wdata = NULL;
    }
    if (param && param->cycle_type == AMLI_CYCLE) {
        free(param->amli_coef);
        param->amli_coef = NULL;
    }
}

static void print_complexity(const hzb_solver *S) {
    // message.c:105-147
    printf("-----------------------------------------------------------\n");
    printf("  Level   Num of rows   Num of nonzeros   Avg. NNZ / row   \n");
    printf("-----------------------------------------------------------\n");
    double gc = 0.0, oc = 0.0;
    for (int l = 0; l < S->nl; ++l) {
        const Level &L = S->lv[l];
        printf("%5lld %13lld %17lld %14.2f\n", (long long)l, (long long)L.n,
               (long long)L.nnz, (double)L.nnz / L.n);
        gc += L.n;
        oc += L.nnz;
    }
    printf("-----------------------------------------------------------\n");
    printf("  Grid complexity = %.3f  |", gc / S->lv[0].n);
    printf("  Operator complexity = %.3f\n", oc / S->lv[0].nnz);
    printf("-----------------------------------------------------------\n");
}

static int export_level(hzb_solver *S, AMG_data *mgl, int l) {
    const Level &L = S->lv[l];
    if (l > 0) {
        mgl[l].A.row = mgl[l].A.col = L.n;
        mgl[l].A.nnz = L.nnz;
        mgl[l].A.IA = (INT *)malloc(sizeof(INT) * (L.n + 1));
        mgl[l].A.JA = (INT *)malloc(sizeof(INT) * (L.nnz > 0 ? L.nnz : 1));
        mgl[l].A.val = (REAL *)malloc(sizeof(REAL) * (L.nnz > 0 ? L.nnz : 1));
        HZB_TRY(hzb_level_copy(S, l, mgl[l].A.IA, mgl[l].A.JA, mgl[l].A.val, NULL));
    }
    if (l < S->nl - 1 && L.sa) {
        // smoothed aggregation: P and R = P^T as stored, with their values
        dCSRmat &P = mgl[l].P, &R = mgl[l].R;
        const int nr = L.pnnz;
        P.row = L.n; P.col = L.nc; P.nnz = nr;
        R.row = L.nc; R.col = L.n; R.nnz = nr;
        P.IA = (INT *)malloc(sizeof(INT) * (L.n + 1));
        P.JA = (INT *)malloc(sizeof(INT) * (nr > 0 ? nr : 1));
        P.val = (REAL *)malloc(sizeof(REAL) * (nr > 0 ? nr : 1));
        R.IA = (INT *)malloc(sizeof(INT) * (L.nc + 1));
        R.JA = (INT *)malloc(sizeof(INT) * (nr > 0 ? nr : 1));
        R.val = (REAL *)malloc(sizeof(REAL) * (nr > 0 ? nr : 1));
        HZB_CUDA(cudaMemcpy(P.IA, L.pia, sizeof(int) * (L.n + 1), cudaMemcpyDeviceToHost));
        HZB_CUDA(cudaMemcpy(P.JA, L.pja, sizeof(int) * nr, cudaMemcpyDeviceToHost));
        HZB_CUDA(cudaMemcpy(P.val, L.pval, sizeof(double) * nr, cudaMemcpyDeviceToHost));
        HZB_CUDA(cudaMemcpy(R.IA, L.ria, sizeof(int) * (L.nc + 1), cudaMemcpyDeviceToHost));
        HZB_CUDA(cudaMemcpy(R.JA, L.rja, sizeof(int) * nr, cudaMemcpyDeviceToHost));
        HZB_CUDA(cudaMemcpy(R.val, L.rval, sizeof(double) * nr, cudaMemcpyDeviceToHost));
    } else if (l < S->nl - 1) {
        // P (n x nc, one unit entry per aggregated row) and R = P^T
        std::vector<int> agg(L.n), ria(L.nc + 1), rja(L.n);
        HZB_CUDA(cudaMemcpy(agg.data(), L.agg, sizeof(int) * L.n, cudaMemcpyDeviceToHost));
        HZB_CUDA(cudaMemcpy(ria.data(), L.ria, sizeof(int) * (L.nc + 1), cudaMemcpyDeviceToHost));
        const int nr = ria[L.nc];
        HZB_CUDA(cudaMemcpy(rja.data(), L.rja, sizeof(int) * nr, cudaMemcpyDeviceToHost));
        dCSRmat &P = mgl[l].P;
        P.row = L.n; P.col = L.nc; P.nnz = nr;
        P.IA = (INT *)malloc(sizeof(INT) * (L.n + 1));
        P.JA = (INT *)malloc(sizeof(INT) * (nr > 0 ? nr : 1));
        P.val = (REAL *)malloc(sizeof(REAL) * (nr > 0 ? nr : 1));
        for (int i = 0, k = 0; i < L.n; ++i) {
            P.IA[i] = k;
            if (agg[i] >= 0) { P.JA[k] = agg[i]; P.val[k] = 1.0; ++k; }
            P.IA[i + 1] = k;
        }
        dCSRmat &R = mgl[l].R;
        R.row = L.nc; R.col = L.n; R.nnz = nr;
        R.IA = (INT *)malloc(sizeof(INT) * (L.nc + 1));
        R.JA = (INT *)malloc(sizeof(INT) * (nr > 0 ? nr : 1));
        R.val = (REAL *)malloc(sizeof(REAL) * (nr > 0 ? nr : 1));
        memcpy(R.IA, ria.data(), sizeof(int) * (L.nc + 1));
        memcpy(R.JA, rja.data(), sizeof(int) * nr);
        for (int k = 0; k < nr; ++k) R.val[k] = 1.0;
    }
    return SUCCESS;
}

// amg_setup_ua / amg_setup_sa: the device hierarchy hangs off mgl[0].wdata
static SHORT amg_setup_common(AMG_data *mgl, AMG_param *param, SHORT type) {
    if (!mgl || !param) return ERROR_INPUT_PAR;
    hzb_param bp;
    hzb_param_init(&bp);
    if (mgl[0].wdata) {   // re-setup: drop the previous device hierarchy
        hzb_destroy((hzb_solver *)mgl[0].wdata);
        mgl[0].wdata = NULL;
    }
    hzb_solver *S = nullptr;
    INT rc = hzb_create(&S, param, NULL, &bp);
    if (rc) return (SHORT)rc;
    S->amg.AMG_type = type;   // the entry point decides, as in the reference
    S->caller_amg = param;
    rc = hzb_setup_host(S, &mgl[0].A);
    if (rc) { hzb_destroy(S); return (SHORT)rc; }
    const int nl = S->nl;
    const int m = S->lv[0].n;
    mgl[0].near_kernel_dim = 1;
    mgl[0].near_kernel_basis = (REAL **)calloc(1, sizeof(REAL *));
    mgl[0].near_kernel_basis[0] = (REAL *)malloc(sizeof(REAL) * m);
    for (int i = 0; i < m; ++i) mgl[0].near_kernel_basis[0][i] = 1.0;
    mgl[0].Schwarz_levels = param->Schwarz_levels;
    for (int l = 0; l < nl && l < mgl[0].max_levels; ++l) {
        if (bp.export_hierarchy) {
            rc = export_level(S, mgl, l);
            if (rc) { hzb_destroy(S); return (SHORT)rc; }
        }
        const int mm = S->lv[l].n;
        if (l == 0) {
            if (!mgl[0].b.val) { mgl[0].b.row = mm; mgl[0].b.val = (REAL *)calloc(mm, sizeof(REAL)); }
            if (!mgl[0].x.val) { mgl[0].x.row = mm; mgl[0].x.val = (REAL *)calloc(mm, sizeof(REAL)); }
            mgl[0].w.row = mm;
            mgl[0].w.val = (REAL *)calloc(mm, sizeof(REAL));
        } else {
            mgl[l].num_levels = nl;
            mgl[l].b.row = mm; mgl[l].b.val = (REAL *)calloc(mm, sizeof(REAL));
            mgl[l].x.row = mm; mgl[l].x.val = (REAL *)calloc(mm, sizeof(REAL));
            const int nw = param->cycle_type == NL_AMLI_CYCLE ? 3 * mm : 2 * mm;
            mgl[l].w.row = nw; mgl[l].w.val = (REAL *)calloc(nw, sizeof(REAL));
            mgl[l].cycle_type = param->cycle_type;
        }
    }
    mgl[0].num_levels = nl;
    mgl[0].wdata = S;
    if (param->cycle_type == AMLI_CYCLE) {
        // amg_setup_ua.c:1276-1281: the polynomial for lambda in [0.5, 2]
        param->amli_coef = (REAL *)calloc(param->amli_degree + 1, sizeof(REAL));
        hzb::amli_coefficients(2.0, 0.5, param->amli_degree, param->amli_coef);
    }
    if (param->print_level > PRINT_NONE) {
        if (param->print_level >= PRINT_SOME) print_complexity(S);
        printf("%s aggregation setup costs %.4f seconds.\n",
               type == SA_AMG ? "Smoothed" : "Unsmoothed", S->st.setup_seconds);
    }
    return SUCCESS;
}

extern "C" SHORT amg_setup_ua(AMG_data *mgl, AMG_param *param) {
    // amg_setup_ua.c:53 -> amg_setup_unsmoothP_unsmoothR (:1228-1452)
    return amg_setup_common(mgl, param, UA_AMG);
}

extern "C" SHORT amg_setup_sa(AMG_data *mgl, AMG_param *param) {
    // amg_setup_ua.c:76 -> amg_setup_smoothP_smoothR (:1461-1700)
    return amg_setup_common(mgl, param, SA_AMG);
}

extern "C" INT hzb_level_prolongation(const hzb_solver *S, INT l, INT *ia, INT *ja,
                                      REAL *val, INT *nnz) {
    if (!S || l < 0 || l >= S->nl - 1) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const Level &L = S->lv[l];
    if (nnz) *nnz = L.sa ? L.pnnz : 0;
    if (!L.sa) return SUCCESS;
    if (ia) HZB_CUDA(cudaMemcpy(ia, L.pia, sizeof(int) * (L.n + 1), cudaMemcpyDeviceToHost));
    if (ja) HZB_CUDA(cudaMemcpy(ja, L.pja, sizeof(int) * L.pnnz, cudaMemcpyDeviceToHost));
    if (val) HZB_CUDA(cudaMemcpy(val, L.pval, sizeof(double) * L.pnnz, cudaMemcpyDeviceToHost));
    return SUCCESS;
}

static hzb_solver *handle_of(AMG_data *mgl) {
    return mgl ? (hzb_solver *)mgl[0].wdata : nullptr;
}

extern "C" void mgcycle(AMG_data *mgl, AMG_param *param) {
    // mgcycle.c:245-415 on mgl[0].b / mgl[0].x (host arrays)
    hzb_solver *S = handle_of(mgl);
    if (!S || !param) return;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    Level &L0 = S->lv[0];
    cudaMemcpyAsync(L0.b, mgl[0].b.val, sizeof(double) * L0.n, cudaMemcpyHostToDevice, S->s);
    cudaMemcpyAsync(L0.x, mgl[0].x.val, sizeof(double) * L0.n, cudaMemcpyHostToDevice, S->s);
    if (cycle64(S, *param) == SUCCESS)
        cudaMemcpyAsync(mgl[0].x.val, L0.x, sizeof(double) * L0.n, cudaMemcpyDeviceToHost, S->s);
    cudaStreamSynchronize(S->s);
}

// The cycle parameters a precond_* function builds from its precond_data
// (param_amg_init, then param_prec_to_amg; maxit from the data).  AMLI
// coefficients the data carries move into the handle.
static AMG_param pc_param_of(hzb_solver *S, precond_data *pcd) {
    AMG_param cyc;
    param_amg_init(&cyc);
    param_prec_to_amg(&cyc, pcd);
    cyc.maxit = pcd->maxit;
    S->amli_coef.clear();
    if (cyc.amli_coef) {
        S->amli_coef.assign(cyc.amli_coef, cyc.amli_coef + cyc.amli_degree + 1);
        free(cyc.amli_coef);
        cyc.amli_coef = NULL;
    }
    return cyc;
}

// z = B r on host arrays with the device preconditioner of the kind
static void precond_host(REAL *r, REAL *z, void *data, int kind) {
    precond_data *pcdata = (precond_data *)data;
    hzb_solver *S = pcdata ? handle_of(pcdata->mgl_data) : nullptr;
    if (!S) return;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const int n = S->lv[0].n;
    if (!S->pr) {
        if (dalloc(&S->pr, n) || dalloc(&S->pz, n)) return;
    }
    S->pc_cyc = pc_param_of(S, pcdata);
    cudaMemcpyAsync(S->pr, r, sizeof(double) * n, cudaMemcpyHostToDevice, S->s);
    if (apply_precond(S, kind, nullptr, n, S->pr, S->pz) == SUCCESS)
        cudaMemcpyAsync(z, S->pz, sizeof(double) * n, cudaMemcpyDeviceToHost, S->s);
    cudaStreamSynchronize(S->s);
}

extern "C" void precond_amg(REAL *r, REAL *z, void *data) {
    // precond.c:164-184 with host arrays r, z
    precond_host(r, z, data, PC_AMG);
}

extern "C" void precond_amli(REAL *r, REAL *z, void *data) {
    // precond.c:232-250
    precond_host(r, z, data, PC_AMLI);
}

extern "C" void precond_nl_amli(REAL *r, REAL *z, void *data) {
    // precond.c:301-320 (the whole hierarchy of the handle)
    precond_host(r, z, data, PC_NLAMLI);
}

extern "C" void precond_amg_add(REAL *r, REAL *z, void *data) {
    // precond.c:336-355
    precond_host(r, z, data, PC_ADD);
}

// One cycle of a kind on mgl[0].b / mgl[0].x (host arrays) with param as
// given; the device hierarchy of mgl[0] is the whole of it, so only
// level 0 (and, for nl_amli, all levels) can be asked for.
static void cycle_host(AMG_data *mgl, AMG_param *param, int kind, INT level) {
    hzb_solver *S = handle_of(mgl);
    if (!S || !param) return;
    if (level != 0) {
        printf("### ERROR: the device hierarchy runs cycles from level 0 of mgl[0]\n");
        return;
    }
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    Level &L0 = S->lv[0];
    if (cycles_prepare(S, kind, *param) != SUCCESS) return;
    // the coarse-level Krylov solves of the nonlinear AMLI cycle precondition
    // with precond_nl_amli on parameters rebuilt from param (mgcycle.c:620)
    S->pc_cyc = cycle_param_of(*param);
    cudaMemcpyAsync(L0.b, mgl[0].b.val, sizeof(double) * L0.n, cudaMemcpyHostToDevice, S->s);
    cudaMemcpyAsync(L0.x, mgl[0].x.val, sizeof(double) * L0.n, cudaMemcpyHostToDevice, S->s);
    int rc;
    if (kind == PC_AMLI) rc = amli64(S, *param, S->amli_coef.data(), 0);
    else if (kind == PC_ADD) rc = add_cycle64(S, *param);
    else rc = nl_amli64(S, *param, 0);
    if (rc == SUCCESS)
        cudaMemcpyAsync(mgl[0].x.val, L0.x, sizeof(double) * L0.n, cudaMemcpyDeviceToHost, S->s);
    cudaStreamSynchronize(S->s);
}

extern "C" void amli(AMG_data *mgl, AMG_param *param, INT level) {
    // mgcycle.c:430-555
    cycle_host(mgl, param, PC_AMLI, level);
}

extern "C" void nl_amli(AMG_data *mgl, AMG_param *param, INT level, INT num_levels) {
    // mgcycle.c:561-690
    hzb_solver *S = handle_of(mgl);
    if (S && num_levels != S->nl) {
        printf("### ERROR: the device hierarchy has %d levels\n", S->nl);
        return;
    }
    cycle_host(mgl, param, PC_NLAMLI, level);
}

extern "C" void mgcycle_add(AMG_data *mgl, AMG_param *param) {
    // mgcycle.c:700-820
    cycle_host(mgl, param, PC_ADD, 0);
}

extern "C" void amg_amli_coef(const REAL lambda_max, const REAL lambda_min, const INT degree,
                              REAL *coef) {
    // parameters.c:714-775
    if (hzb::amli_coefficients(lambda_max, lambda_min, degree, coef) != SUCCESS)
        printf("### ERROR HAZMATH DANGER: Wrong AMLI degree %lld!\n", (long long)degree);
}

// ---------------------------------------------------------------------------
// drop-in: Krylov entry points
// ---------------------------------------------------------------------------
// device copy of a host matrix for operators that are not the setup matrix
struct TmpCsr {
    int *ia = nullptr, *ja = nullptr;
    double *val = nullptr;
    void release() { dfree(ia); dfree(ja); dfree(val); }
    ~TmpCsr() { release(); }
};

static int upload_csr(const dCSRmat *A, TmpCsr &T, DCsr<double> &D, cudaStream_t s) {
    HZB_TRY(dalloc(&T.ia, A->row + 1));
    HZB_TRY(dalloc(&T.ja, A->nnz));
    HZB_TRY(dalloc(&T.val, A->nnz));
    HZB_CUDA(cudaMemcpyAsync(T.ia, A->IA, sizeof(int) * (A->row + 1), cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(T.ja, A->JA, sizeof(int) * A->nnz, cudaMemcpyHostToDevice, s));
    HZB_CUDA(cudaMemcpyAsync(T.val, A->val, sizeof(double) * A->nnz, cudaMemcpyHostToDevice, s));
    D.n = A->row; D.nnz = A->nnz; D.ia = T.ia; D.ja = T.ja; D.val = T.val;
    HZB_TRY(bundle_capacity(D.n, D.ia, s, &D.bundle_cap));
    return SUCCESS;
}

// A Krylov method (SOLVER_CG, SOLVER_MinRes, SOLVER_GCG, SOLVER_VGMRES, SOLVER_VFGMRES) on host
// arrays with the caller's preconditioner: the setup's own AMG runs on the
// device, any other pc->fct is called on host copies.
static INT krylov_host(dCSRmat *A, dvector *b, dvector *u, precond *pc, REAL tol,
                       INT MaxIt, SHORT stop_type, SHORT prtlvl, double *condest, int type,
                       int restart) {
    if (!A || !b || !u || A->row != b->row || A->row != u->row) return ERROR_MAT_SIZE;
    HZB_TRY(check_csr_host(A->row, A->nnz, A->IA));
    hzb_solver *S = nullptr, *own = nullptr;
    int kind = PC_NONE;
    HostPrecond hp;
    const int dev_kind = !pc ? -1
                         : pc->fct == precond_amg ? PC_AMG
                         : pc->fct == precond_amli ? PC_AMLI
                         : pc->fct == precond_nl_amli ? PC_NLAMLI
                         : pc->fct == precond_amg_add ? PC_ADD : -1;
    if (dev_kind >= 0 && pc->data && handle_of(((precond_data *)pc->data)->mgl_data)) {
        S = handle_of(((precond_data *)pc->data)->mgl_data);
        S->pc_cyc = pc_param_of(S, (precond_data *)pc->data);
        kind = dev_kind;
    } else {
        HZB_TRY(hzb_create(&own, NULL, NULL, NULL));
        S = own;
        if (pc && pc->fct) {
            kind = PC_HOST;
            hp.fct = pc->fct;
            hp.data = pc->data;
            hp.h_r = (double *)malloc(sizeof(double) * A->row);
            hp.h_z = (double *)malloc(sizeof(double) * A->row);
        }
    }
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    int rc = SUCCESS;
    DCsr<double> D;
    TmpCsr T;
    double *db = nullptr, *du = nullptr;
    KrylovWork w;
    const bool same = kind != PC_NONE && kind != PC_HOST && S->host_ia == A->IA && S->host_ja == A->JA &&
                      S->host_val == A->val && S->lv[0].n == A->row;
    if (same) D = S->lv[0].A64();
    else rc = upload_csr(A, T, D, S->s);
    if (!rc) rc = dalloc(&db, A->row);
    if (!rc) rc = dalloc(&du, A->row);
    if (!rc) rc = w.alloc(A->row);
    INT it = rc;
    if (!rc) {
        cudaMemcpyAsync(db, b->val, sizeof(double) * A->row, cudaMemcpyHostToDevice, S->s);
        cudaMemcpyAsync(du, u->val, sizeof(double) * A->row, cudaMemcpyHostToDevice, S->s);
        double rel = 0.0;
        if (type == SOLVER_CG)
            it = pcg(S, D, db, du, kind, &hp, tol, MaxIt, stop_type, prtlvl, w, &rel, condest);
        else if (type == SOLVER_GCG)
            it = gcg(S, D, db, du, kind, &hp, tol, MaxIt, stop_type, prtlvl, &rel);
        else if (type == SOLVER_MinRes)
            it = minres(S, D, db, du, kind, &hp, tol, MaxIt, stop_type, prtlvl, &rel);
        else
            it = gmres(S, D, db, du, kind, &hp, tol, MaxIt, restart, stop_type, prtlvl,
                       type == SOLVER_VFGMRES, &rel);
        if (it >= 0 && S->nl > 0) {
            const int wc = check_waits(S);
            if (wc) it = wc;
        }
        if (it != ERROR_SOLVER_MISC) {
            cudaMemcpyAsync(u->val, du, sizeof(double) * A->row, cudaMemcpyDeviceToHost, S->s);
            if (cudaStreamSynchronize(S->s) != cudaSuccess) it = ERROR_SOLVER_MISC;
        }
    }
    // everything allocated on the handle's stream goes before the stream
    w.release();
    T.release();
    dfree(db);
    dfree(du);
    free(hp.h_r);
    free(hp.h_z);
    if (own) hzb_destroy(own);
    return it;
}

extern "C" INT dcsr_pcg(dCSRmat *A, dvector *b, dvector *u, precond *pc,
                        const REAL tol, const INT MaxIt, const SHORT stop_type,
                        const SHORT prtlvl) {
    // krylov.c:122-398
    return krylov_host(A, b, u, pc, tol, MaxIt, stop_type, prtlvl, nullptr, SOLVER_CG, 0);
}

extern "C" INT dcsr_pvgmres(dCSRmat *A, dvector *b, dvector *x, precond *pc,
                            const REAL tol, const INT MaxIt, const SHORT restart,
                            const SHORT stop_type, const SHORT prtlvl) {
    // krylov.c:4612-4930
    return krylov_host(A, b, x, pc, tol, MaxIt, stop_type, prtlvl, nullptr, SOLVER_VGMRES,
                       restart);
}

extern "C" INT dcsr_pvfgmres(dCSRmat *A, dvector *b, dvector *x, precond *pc,
                             const REAL tol, const INT MaxIt, const SHORT restart,
                             const SHORT stop_type, const SHORT prtlvl) {
    // krylov.c:5974-6250
    return krylov_host(A, b, x, pc, tol, MaxIt, stop_type, prtlvl, nullptr, SOLVER_VFGMRES,
                       restart);
}

extern "C" INT dcsr_pminres(dCSRmat *A, dvector *b, dvector *u, precond *pc, const REAL tol,
                            const INT MaxIt, const SHORT stop_type, const SHORT prtlvl) {
    // krylov.c:2449-2840
    return krylov_host(A, b, u, pc, tol, MaxIt, stop_type, prtlvl, nullptr, SOLVER_MinRes, 0);
}

extern "C" INT dcsr_pgcg(dCSRmat *A, dvector *b, dvector *u, precond *pc, const REAL tol,
                         const INT MaxIt, const SHORT stop_type, const SHORT prtlvl) {
    // krylov.c:2309-2420
    return krylov_host(A, b, u, pc, tol, MaxIt, stop_type, prtlvl, nullptr, SOLVER_GCG, 0);
}

// the banner solver_dcsr_linear_itsolver prints for a Krylov type
static void krylov_banner(SHORT prtlvl, SHORT type) {
    if (prtlvl <= PRINT_NONE) return;
    printf("**********************************************************\n");
    if (type == SOLVER_CG) printf(" --> using Conjugate Gradient Method:\n");
    else if (type == SOLVER_MinRes) printf(" --> using MINRES Method:\n");
    else if (type == SOLVER_VGMRES) printf(" --> using GMRES Method:\n");
    else printf(" --> using Flexible GMRES Method:\n");
}

extern "C" INT solver_dcsr_linear_itsolver(dCSRmat *A, dvector *b, dvector *x,
                                           precond *pc,
                                           linear_itsolver_param *itparam) {
    // itsolver.c:135-229
    const SHORT prtlvl = itparam->linear_print_level;
    const SHORT type = itparam->linear_itsolver_type;
    if (itparam->linear_tol < SMALLREAL)
        printf("### HAZMATH WARNING: Convergence tolerance for iterative solver is too small!\n");
    if (itparam->linear_maxit <= 0)
        printf("### HAZMATH WARNING: Max number of iterations should be a POSITIVE integer!\n");
    if (type != SOLVER_CG && type != SOLVER_MinRes && type != SOLVER_VGMRES &&
        type != SOLVER_VFGMRES) {
        printf("### ERROR: Unknown itertive solver type %lld!\n", (long long)type);
        return ERROR_SOLVER_TYPE;
    }
    krylov_banner(prtlvl, type);
    double cond = 0.0;
    INT it = krylov_host(A, b, x, pc, itparam->linear_tol, itparam->linear_maxit,
                         itparam->linear_stop_type, prtlvl, &cond, type,
                         itparam->linear_restart);
    if (type == SOLVER_CG) printf("Estimated condition number = %13.6e\n", cond);
    if (type == SOLVER_MinRes) printf(" NOTHING IMPLEMENTED FOR MINRES\n");   // itsolver.c:176
    return it;
}

extern "C" INT hzb_solver_dcsr_krylov_amg(dCSRmat *A, dvector *b, dvector *x,
                                          linear_itsolver_param *itparam,
                                          AMG_param *amgparam, const hzb_param *bp) {
    // itsolver.c:846-931
    if (!A || !b || !x || !itparam || !amgparam) return ERROR_INPUT_PAR;
    const SHORT prtlvl = itparam->linear_print_level;
    if (A->row != A->col || b->row != A->row || x->row != A->row) return ERROR_MAT_SIZE;
    hzb_param dflt;
    hzb_param_init(&dflt);
    if (!bp) bp = &dflt;
    if (prtlvl > PRINT_NONE)
        printf("\n Calling %s AMG ...\n", amgparam->AMG_type == SA_AMG ? "SA" : "UA");
    hzb_solver *S = nullptr;
    INT rc = hzb_create(&S, amgparam, itparam, bp);
    if (rc) return rc;
    S->caller_amg = amgparam;
    rc = hzb_setup_host(S, A);
    if (rc) { hzb_destroy(S); return rc; }
    if (amgparam->print_level > PRINT_NONE) {
        if (amgparam->print_level >= PRINT_SOME) print_complexity(S);
        printf("%s aggregation setup costs %.4f seconds.\n",
               amgparam->AMG_type == SA_AMG ? "Smoothed" : "Unsmoothed", S->st.setup_seconds);
    }
    const SHORT type = itparam->linear_itsolver_type;
    if (bp->precision != HZB_PREC_MIXED && type != SOLVER_CG && type != SOLVER_MinRes &&
        type != SOLVER_VGMRES && type != SOLVER_VFGMRES) {
        printf("### ERROR: Unknown itertive solver type %lld!\n", (long long)type);
        hzb_destroy(S);
        return ERROR_SOLVER_TYPE;
    }
    krylov_banner(prtlvl, bp->precision == HZB_PREC_MIXED ? SOLVER_CG : type);
    INT it = hzb_solve_host(S, b->val, x->val);
    if (bp->precision != HZB_PREC_MIXED && type == SOLVER_CG)
        printf("Estimated condition number = %13.6e\n", S->st.condest);
    if (bp->precision != HZB_PREC_MIXED && type == SOLVER_MinRes)
        printf(" NOTHING IMPLEMENTED FOR MINRES\n");
    if (prtlvl >= PRINT_MIN) {
        printf("AMG_Krylov method totally costs %.4f seconds.\n",
               S->st.setup_seconds + S->st.solve_seconds);
        printf("**********************************************************\n");
    }
    hzb_destroy(S);
    return it;
}

extern "C" INT linear_solver_dcsr_krylov_amg(dCSRmat *A, dvector *b, dvector *x,
                                             linear_itsolver_param *itparam,
                                             AMG_param *amgparam) {
    return hzb_solver_dcsr_krylov_amg(A, b, x, itparam, amgparam, NULL);
}

// ---------------------------------------------------------------------------
// block (BSR) matrices: amg_setup_ua_bsr, precond_dbsr_amg and
// solver_dbsr_linear_itsolver behind linear_solver_dbsr_krylov_amg
// (amg_setup_ua.c:145, precond.c:1311-1339, itsolver.c:232-305, 2104-2200)
// ---------------------------------------------------------------------------
static int check_bsr_host(const dBSRmat *A) {
    if (!A || !A->IA || !A->JA || !A->val) return ERROR_INPUT_PAR;
    if (A->ROW != A->COL || A->ROW <= 0 || A->NNZ <= 0) return ERROR_MAT_SIZE;
    if (A->IA[0] != 0 || A->IA[A->ROW] != A->NNZ) return ERROR_DATA_STRUCTURE;
    if (A->storage_manner != 0) {
        set_error_msg("blocks are stored row by row (storage_manner 0)");
        return ERROR_INPUT_PAR;
    }
    return SUCCESS;
}

// precond_dbsr_amg rebuilds its cycle parameters from param_amg_init with
// these fields of the caller's AMG_param (precond.c:1322-1330): the coarse
// solver and tolerance stay at their defaults
static AMG_param bsr_cycle_param_of(const AMG_param &amg) {
    AMG_param c;
    param_amg_init(&c);
    c.cycle_type = amg.cycle_type;
    c.smoother = amg.smoother;
    c.presmooth_iter = amg.presmooth_iter;
    c.postsmooth_iter = amg.postsmooth_iter;
    c.relaxation = amg.relaxation;
    c.coarse_scaling = amg.coarse_scaling;
    c.tentative_smooth = amg.tentative_smooth;
    c.maxit = amg.maxit;   // precdata.maxit: the cycles per application
    return c;
}

extern "C" INT hzb_bsr_setup_host(hzb_solver *S, const dBSRmat *A) {
    if (!S) return ERROR_INPUT_PAR;
    HZB_TRY(check_bsr_host(A));
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    S->bsr_cyc = bsr_cycle_param_of(S->amg);
    return hzb::bsr_setup(S, A->ROW, A->NNZ, A->nb, A->IA, A->JA, A->val);
}

extern "C" INT hzb_bsr_setup_device(hzb_solver *S, INT nrow, INT nnzb, INT nb,
                                    const INT *d_ia, const INT *d_ja, const REAL *d_val) {
    if (!S || !d_ia || !d_ja || !d_val) return ERROR_INPUT_PAR;
    if (nrow <= 0 || nnzb <= 0) return ERROR_MAT_SIZE;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    S->bsr_cyc = bsr_cycle_param_of(S->amg);
    return hzb::bsr_setup(S, nrow, nnzb, nb, d_ia, d_ja, d_val);
}

extern "C" INT hzb_bsr_level(const hzb_solver *S, INT l, dBSRmat *out, INT *agg) {
    if (!S || !S->bsr || !out) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    int nrow = 0, nnzb = 0;
    HZB_TRY(hzb::bsr_level_copy(S, l, &nrow, &nnzb, out->IA, out->JA, out->val, agg));
    out->ROW = out->COL = nrow;
    out->NNZ = nnzb;
    out->nb = hzb::bsr_block_size(S);
    out->storage_manner = 0;
    return SUCCESS;
}

extern "C" INT hzb_bsr_precond_device(hzb_solver *S, const REAL *d_r, REAL *d_z) {
    if (!S || !S->bsr) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    HZB_TRY(hzb::bsr_precond(S, d_r, d_z));
    HZB_CUDA(cudaStreamSynchronize(S->s));
    return hzb::check_waits(S);
}

extern "C" INT hzb_bsr_solve_device(hzb_solver *S, const REAL *d_b, REAL *d_x) {
    if (!S || !S->bsr) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const long long l0 = hzb::launch_count();
    HZB_CUDA(cudaEventRecord(S->e0, S->s));
    double rel = 0.0, cond = 0.0;
    int it;
    const int prt = S->it.linear_print_level;
    const DCsr<double> A = bsr_scalar_A(S);
    switch (S->it.linear_itsolver_type) {
    case SOLVER_CG:   // dbsr_pcg_w_cond_est
        it = pcg(S, A, d_b, d_x, PC_BSR, nullptr, S->it.linear_tol, S->it.linear_maxit,
                 S->it.linear_stop_type, prt, S->kw, &rel, &cond);
        break;
    case SOLVER_VGMRES:
    case SOLVER_VFGMRES:   // dbsr_pvgmres / dbsr_pvfgmres
        it = gmres(S, A, d_b, d_x, PC_BSR, nullptr, S->it.linear_tol, S->it.linear_maxit,
                   S->it.linear_restart, S->it.linear_stop_type, prt,
                   S->it.linear_itsolver_type == SOLVER_VFGMRES, &rel);
        break;
    default:
        set_error_msg("Krylov types 1 (CG), 3 (GMRES) and 4 (flexible GMRES) are the ones "
                      "solver_dbsr_linear_itsolver dispatches");
        return ERROR_SOLVER_TYPE;
    }
    HZB_CUDA(cudaEventRecord(S->e1, S->s));
    HZB_CUDA(cudaEventSynchronize(S->e1));
    if (it >= 0) {
        const int wc = check_waits(S);
        if (wc) it = wc;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, S->e0, S->e1);
    S->st.solve_seconds = ms * 1e-3;
    S->st.iterations = it;
    S->st.final_relres = rel;
    S->st.condest = cond;
    S->st.launches = (INT)(hzb::launch_count() - l0);
    return it;
}

// host vectors through device copies; op 0 solves, 1 applies the
// preconditioner
static INT bsr_host_call(hzb_solver *S, const REAL *in, REAL *out, int op) {
    if (!S || !S->bsr) return ERROR_INPUT_PAR;
    cudaSetDevice(S->bp.device);
    StreamScope scope_(S->s);
    const int n = bsr_scalar_A(S).n;
    double *di = nullptr, *dout = nullptr;
    HZB_TRY(dalloc(&di, n));
    int rc = dalloc(&dout, n);
    if (rc) { dfree(di); return rc; }
    cudaMemcpyAsync(di, in, sizeof(double) * n, cudaMemcpyHostToDevice, S->s);
    if (op == 0) cudaMemcpyAsync(dout, out, sizeof(double) * n, cudaMemcpyHostToDevice, S->s);
    const int it = op == 0 ? hzb_bsr_solve_device(S, di, dout)
                           : hzb_bsr_precond_device(S, di, dout);
    cudaError_t e = cudaMemcpyAsync(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, S->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->s);
    dfree(di);
    dfree(dout);
    if (e != cudaSuccess) { set_error(e, __FILE__, __LINE__); return ERROR_SOLVER_MISC; }
    return it;
}

extern "C" INT hzb_bsr_solve_host(hzb_solver *S, const REAL *b, REAL *x) {
    return bsr_host_call(S, b, x, 0);
}

extern "C" INT hzb_bsr_precond_host(hzb_solver *S, const REAL *r, REAL *z) {
    return bsr_host_call(S, r, z, 1);
}

extern "C" INT linear_solver_dbsr_krylov_amg(dBSRmat *A, dvector *b, dvector *x,
                                             linear_itsolver_param *itparam,
                                             AMG_param *amgparam) {
    if (!A || !b || !x || !itparam || !amgparam) return ERROR_INPUT_PAR;
    HZB_TRY(check_bsr_host(A));
    if (b->row != A->ROW * A->nb || x->row != A->ROW * A->nb) return ERROR_MAT_SIZE;
    const SHORT prtlvl = itparam->linear_print_level;
    hzb_solver *S = nullptr;
    INT rc = hzb_create(&S, amgparam, itparam, NULL);
    if (rc) return rc;
    rc = hzb_bsr_setup_host(S, A);
    if (rc) { hzb_destroy(S); return rc; }
    if (prtlvl >= PRINT_MIN) printf("BSR AMG setup costs %.4f seconds.\n", S->st.setup_seconds);
    // solver_dbsr_linear_itsolver (itsolver.c:232-305)
    if (itparam->linear_tol < SMALLREAL)
        printf("### HAZMATH WARNING: Convergence tolerance for iterative solver is too small!\n");
    if (itparam->linear_maxit <= 0)
        printf("### HAZMATH WARNING: Max number of iterations should be a POSITIVE integer!\n");
    const SHORT type = itparam->linear_itsolver_type;
    if (type != SOLVER_CG && type != SOLVER_VGMRES && type != SOLVER_VFGMRES) {
        printf("### ERROR: Unknown itertive solver type %lld!\n", (long long)type);
        hzb_destroy(S);
        return ERROR_SOLVER_TYPE;
    }
    krylov_banner(prtlvl, type);
    const INT it = hzb_bsr_solve_host(S, b->val, x->val);
    if (type == SOLVER_CG) printf("Estimated condition number = %13.6e\n", S->st.condest);
    if (prtlvl >= PRINT_SOME && it >= 0) {   // itsolver.c:298-303
        printf("Iterative method costs %.4f seconds.\n", S->st.solve_seconds);
        printf("**********************************************************\n");
    }
    if (prtlvl >= PRINT_MIN)
        printf("BSR Krylov method costs %.4f seconds.\n",
               S->st.setup_seconds + S->st.solve_seconds);
    hzb_destroy(S);
    return it;
}

extern "C" INT linear_solver_amg(dCSRmat *A, dvector *b, dvector *x, AMG_param *param) {
    // itsolver.c:524-630 + amg_solve (amg_solve.c:109-160)
    if (!A || !b || !x || !param) return ERROR_INPUT_PAR;
    if (A->row != A->col) {
        printf("### ERROR: A is not a square matrix!\n");
        return ERROR_MAT_SIZE;
    }
    if (A->nnz <= 0) {
        printf("### ERROR: A has no nonzero entries!\n");
        return ERROR_MAT_SIZE;
    }
    const SHORT prtlvl = param->print_level;
    if (prtlvl > PRINT_NONE)
        printf("\n Calling %s AMG ...\n", param->AMG_type == SA_AMG ? "SA" : "UA");
    hzb_solver *S = nullptr;
    INT rc = hzb_create(&S, param, NULL, NULL);
    if (rc) return rc;
    S->caller_amg = param;
    rc = hzb_setup_host(S, A);
    if (rc) { hzb_destroy(S); return rc; }
    const int n = A->row;
    Level &L0 = S->lv[0];
    KrylovWork &w = S->kw;
    cudaStream_t s = S->s;
    cudaMemcpyAsync(L0.b, b->val, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(L0.x, x->val, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    double sumb = 0.0, absres0, absres, relres1 = BIGREAL;
    dot(n, L0.b, L0.b, w.part, w.sc, s);
    cudaMemcpy(w.h_sc, w.sc, sizeof(double), cudaMemcpyDeviceToHost);
    sumb = sqrt(w.h_sc[0]);
    absres0 = sumb;
    const INT MaxIt = param->maxit;
    int iter = 0;
    if (prtlvl >= PRINT_SOME) {
        printf("-----------------------------------------------------------\n");
        printf("It Num |   ||r||/||b||   |     ||r||      |  Conv. Factor\n");
        printf("-----------------------------------------------------------\n");
        printf("%6lld | %13.6e   | %13.6e  |     -.-- \n", 0LL, 1.0, sumb);
    }
    while ((++iter <= MaxIt) & (sumb > SMALLREAL)) {
        if (cycle64(S, *param)) { iter = ERROR_SOLVER_MISC; break; }
        spmv<double>(L0.A64(), SPMV_RES, L0.x, L0.b, w.r, 1.0, nullptr, s);
        dot(n, w.r, w.r, w.part, w.sc, s);
        cudaMemcpyAsync(w.h_sc, w.sc, sizeof(double), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        absres = sqrt(w.h_sc[0]);
        relres1 = absres / sumb;
        if (prtlvl >= PRINT_SOME)
            printf("%6lld | %13.6e   | %13.6e  | %10.4f\n", (long long)iter, relres1,
                   absres, absres / absres0);
        absres0 = absres;
        if (relres1 < param->tol) break;
    }
    if (prtlvl > PRINT_NONE && iter >= 0) {
        if (iter > MaxIt)
            printf("### HAZMATH WARNING: Max iter %lld reached with rel. resid. %e.\n",
                   (long long)MaxIt, relres1);
        else
            printf("Num_iter(krylov.c) = %lld with relative residual %e.\n",
                   (long long)iter, relres1);
    }
    cudaMemcpyAsync(x->val, L0.x, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    hzb_destroy(S);
    return iter;
}

// ---------------------------------------------------------------------------
// python_wrapper_krylov_amg (wrapper.c:36-99)
// ---------------------------------------------------------------------------
static std::string trim(const std::string &v) {
    size_t a = 0, b = v.size();
    while (a < b && isspace((unsigned char)v[a])) ++a;
    while (b > a && (isspace((unsigned char)v[b - 1]) || v[b - 1] == ';')) --b;
    return v.substr(a, b - a);
}

// The AMG and linear-solver keys of HAZmath's input.dat (input.c:445-676).
static void read_input_dat(const char *path, AMG_param *amg,
                           linear_itsolver_param *it) {
    FILE *f = fopen(path, "r");
    if (!f) return;
    char line[1024];
    while (fgets(line, sizeof line, f)) {
        std::string s(line);
        size_t c = s.find('%');
        if (c != std::string::npos) s = s.substr(0, c);
        size_t eq = s.find('=');
        if (eq == std::string::npos) continue;
        std::string k = trim(s.substr(0, eq)), v = trim(s.substr(eq + 1));
        if (v.empty()) continue;
        const char *cv = v.c_str();
        if (k == "print_level") { it->linear_print_level = (SHORT)atoi(cv); amg->print_level = (SHORT)atoi(cv); }
        else if (k == "linear_itsolver_type") it->linear_itsolver_type = (SHORT)atoi(cv);
        else if (k == "linear_itsolver_maxit") it->linear_maxit = atoi(cv);
        else if (k == "linear_itsolver_tol") it->linear_tol = atof(cv);
        else if (k == "linear_stop_type") it->linear_stop_type = (SHORT)atoi(cv);
        else if (k == "linear_restart") it->linear_restart = atoi(cv);
        else if (k == "linear_precond_type") it->linear_precond_type = (SHORT)atoi(cv);
        else if (k == "AMG_type") amg->AMG_type = (v == "SA") ? SA_AMG : UA_AMG;
        else if (k == "AMG_cycle_type") amg->cycle_type = (v == "W") ? W_CYCLE : V_CYCLE;
        else if (k == "AMG_levels") amg->max_levels = (SHORT)atoi(cv);
        else if (k == "AMG_tol") amg->tol = atof(cv);
        else if (k == "AMG_maxit") amg->maxit = atoi(cv);
        else if (k == "AMG_smoother") {
            if (v == "JACOBI") amg->smoother = SMOOTHER_JACOBI;
            else if (v == "GS") amg->smoother = SMOOTHER_GS;
            else if (v == "SGS") amg->smoother = SMOOTHER_SGS;
            else if (v == "SOR") amg->smoother = SMOOTHER_SOR;
            else if (v == "SSOR") amg->smoother = SMOOTHER_SSOR;
            else if (v == "GSOR") amg->smoother = SMOOTHER_GSOR;
            else if (v == "SGSOR") amg->smoother = SMOOTHER_SGSOR;
            else if (v == "L1DIAG") amg->smoother = SMOOTHER_L1DIAG;
        }
        else if (k == "AMG_presmooth_iter") amg->presmooth_iter = (SHORT)atoi(cv);
        else if (k == "AMG_postsmooth_iter") amg->postsmooth_iter = (SHORT)atoi(cv);
        else if (k == "AMG_relaxation") amg->relaxation = atof(cv);
        else if (k == "AMG_coarse_dof") amg->coarse_dof = atoi(cv);
        else if (k == "AMG_coarse_solver") amg->coarse_solver = (SHORT)atoi(cv);
        else if (k == "AMG_coarse_scaling") amg->coarse_scaling = (v == "ON") ? ON : OFF;
        else if (k == "AMG_aggregation_type") amg->aggregation_type = (SHORT)atoi(cv);
        else if (k == "AMG_strong_coupled") amg->strong_coupled = atof(cv);
        else if (k == "AMG_max_aggregation") amg->max_aggregation = atoi(cv);
    }
    fclose(f);
}

extern "C" void python_wrapper_krylov_amg(INT *n, INT *nnz, INT *ia, INT *ja,
                                          REAL *a, REAL *b, REAL *u, REAL *tol,
                                          INT *maxit, INT *print_lvl) {
    AMG_param amg;
    linear_itsolver_param it;
    param_linear_solver_init(&it);
    param_amg_init(&amg);
    // UA-AMG preconditioned CG defaults of the HAZmath solver examples
    it.linear_itsolver_type = SOLVER_CG;
    it.linear_precond_type = PREC_AMG;
    amg.cycle_type = V_CYCLE;
    amg.aggregation_type = HEM;
    amg.strong_coupled = 0.0;
    amg.max_levels = 20;
    amg.coarse_dof = 2000;
    amg.coarse_solver = SOLVER_UMFPACK;
    read_input_dat("./input.dat", &amg, &it);
    amg.print_level = (SHORT)*print_lvl;
    it.linear_tol = *tol;
    it.linear_print_level = (SHORT)*print_lvl;
    it.linear_maxit = *maxit;
    dCSRmat mat;
    mat.row = *n; mat.col = *n; mat.nnz = *nnz;
    mat.IA = ia; mat.JA = ja; mat.val = a;
    dvector rhs, sol;
    rhs.row = *n; rhs.val = b;
    sol.row = *n; sol.val = u;
    linear_solver_dcsr_krylov_amg(&mat, &rhs, &sol, &it, &amg);
}

// ---------------------------------------------------------------------------
// kernel-level entry points on device arrays (parity tests)
// ---------------------------------------------------------------------------
static DCsr<double> view(INT n, INT nnz, const INT *ia, const INT *ja, const REAL *val,
                         cudaStream_t s, int *rc) {
    DCsr<double> A;
    A.n = n; A.nnz = nnz; A.ia = ia; A.ja = ja; A.val = val;
    *rc = bundle_capacity(n, ia, s, &A.bundle_cap);
    return A;
}

extern "C" INT hzb_dcsr_mxv_device(INT n, INT nnz, const INT *ia, const INT *ja,
                                   const REAL *val, const REAL *x, REAL *y) {
    int rc;
    DCsr<double> A = view(n, nnz, ia, ja, val, 0, &rc);
    if (rc) return rc;
    HZB_TRY(spmv<double>(A, SPMV_Y, x, nullptr, y, 1.0, nullptr, 0));
    HZB_CUDA(cudaDeviceSynchronize());
    return SUCCESS;
}

extern "C" INT hzb_dcsr_aAxpy_device(REAL alpha, INT n, INT nnz, const INT *ia,
                                     const INT *ja, const REAL *val, const REAL *x,
                                     REAL *y) {
    int rc;
    DCsr<double> A = view(n, nnz, ia, ja, val, 0, &rc);
    if (rc) return rc;
    HZB_TRY(spmv<double>(A, SPMV_AXPY, x, nullptr, y, alpha, nullptr, 0));
    HZB_CUDA(cudaDeviceSynchronize());
    return SUCCESS;
}

extern "C" INT hzb_smoother_device(SHORT smoother, SHORT forward, INT sweeps,
                                   REAL relax, INT n, INT nnz, const INT *ia,
                                   const INT *ja, const REAL *val, const REAL *b,
                                   REAL *x) {
    hzb_solver *S = nullptr;
    AMG_param amg;
    param_amg_init(&amg);
    amg.smoother = smoother;
    amg.presmooth_iter = (SHORT)sweeps;
    amg.postsmooth_iter = (SHORT)sweeps;
    amg.relaxation = relax;
    HZB_TRY(hzb_create(&S, &amg, NULL, NULL));
    int rc = SUCCESS;
    {
    StreamScope scope_(S->s);
    S->lv.emplace_back();
    Level &L = S->lv[0];
    L.n = n; L.nnz = nnz; L.own_A = false;
    L.ia = const_cast<int *>(ia); L.ja = const_cast<int *>(ja);
    L.val = const_cast<double *>(val);
    L.b = const_cast<double *>(b);
    L.x = x;
    S->nl = 1;
    rc = bundle_capacity(n, ia, S->s, &L.bundle_cap);
    if (!rc) rc = dalloc(&L.t, n);
    if (!rc) rc = level_smoother_data(S, L);
    if (!rc) rc = smooth64(S, 0, forward != 0, amg);
    if (!rc && cudaStreamSynchronize(S->s) != cudaSuccess) rc = ERROR_SOLVER_MISC;
    L.b = nullptr;   // not owned
    L.x = nullptr;
    }
    hzb_destroy(S);
    return rc;
}

extern "C" INT hzb_aggregation_hem_device(INT n, INT nnz, const INT *ia,
                                          const INT *ja, const REAL *val,
                                          REAL strong_coupled, INT *agg,
                                          INT *num_aggregates) {
    cudaStream_t s = 0;
    int *nia = nullptr, *nja = nullptr, *work = nullptr, *tmp = nullptr;
    double *nval = nullptr;
    int rc = SUCCESS, nnnz = 0;
    DCsr<double> A;
    A.n = n; A.nnz = nnz; A.ia = ia; A.ja = ja; A.val = val;
    if ((rc = dalloc(&nia, n + 1)) || (rc = dalloc(&nja, nnz)) ||
        (rc = dalloc(&nval, nnz)) || (rc = dalloc(&work, n)) ||
        (rc = dalloc(&tmp, scan_tmp_size(n + 1)))) goto done;
    rc = strength_graph(A, strong_coupled, nia, nja, nval, &nnnz, tmp, s);
    if (!rc) rc = hem_exact(n, nia, nja, nval, agg, num_aggregates, work, s);
done:
    dfree(nia); dfree(nja); dfree(nval); dfree(work); dfree(tmp);
    return rc;
}

extern "C" INT hzb_rap_agg_device(INT n, INT nnz, const INT *ia, const INT *ja,
                                  const REAL *val, INT nc, const INT *agg,
                                  INT *rap_nnz, INT **rap_ia, INT **rap_ja,
                                  REAL **rap_val) {
    cudaStream_t s = 0;
    int *ria = nullptr, *rja = nullptr, *tmp = nullptr;
    int rc = SUCCESS;
    DCsr<double> A;
    A.n = n; A.nnz = nnz; A.ia = ia; A.ja = ja; A.val = val;
    if (n < 1 || nnz < 0 || nc < 1 || nc > n || !ia || !ja || !val || !agg) {
        set_error_msg("hzb_rap_agg_device: need n >= 1, nnz >= 0, 1 <= nc <= n");
        return ERROR_INPUT_PAR;
    }
    if ((rc = dalloc(&ria, nc + 1)) || (rc = dalloc(&rja, n)) ||
        (rc = dalloc(&tmp, scan_tmp_size(n + 1)))) goto done;
    rc = check_rap_inputs(n, nnz, ia, ja, nc, agg, ria, s);
    if (!rc) rc = restriction_pattern(n, nc, agg, ria, rja, tmp, s);
    if (!rc) rc = rap_agg(A, nc, agg, ria, rja, rap_ia, rap_ja, rap_val, rap_nnz, s);
done:
    dfree(ria); dfree(rja); dfree(tmp);
    return rc;
}

extern "C" INT hzb_assemble_p1_kuhn_device(INT N, const REAL *d_kcell, const REAL *K,
                                           INT *d_ia, INT *d_ja, REAL *d_val, INT *nnz) {
    // mesh_cube_init (mesh_cube_anydim.c:30-128) + call_assembly
    // (examples/elliptic_p1/supporting_elliptic_p1.h:537-647) + set_essential_bc
    if (!d_ia) return ERROR_INPUT_PAR;
    return hzb::assemble_kuhn_p1(N, d_kcell, K, d_ia, d_ja, d_val, nnz, 0);
}

extern "C" void hzb_free_device(void *p) {
    if (p) cudaFree(p);
}

extern "C" INT hzb_copy_to_host(void *dst, const void *src, size_t bytes) {
    HZB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return SUCCESS;
}
