/*
 * ref_harness.c -- test infrastructure only.
 *
 * A thin ctypes-facing shim over the reference HAZmath library compiled from
 * its own sources by oracle/build_ref.sh.  It is the checker that pins the C
 * restatement (oracle/hzoracle.c) and produces the golden fixtures under
 * tests/golden/.  Nothing in the product links or loads it.
 *
 * The UA-AMG-PCG path is driven the way linear_solver_dcsr_krylov_amg
 * (src/solver/itsolver.c:846-931) drives it, except that dcsr_pcg
 * (src/solver/krylov.c:122) is called directly instead of
 * dcsr_pcg_w_cond_est: without LAPACK the latter exits the process with
 * status 252 after a converged solve (krylov.c:704, message.c:295); its
 * iterates are the same.
 */
#include "hazmath.h"
#include <time.h>

static AMG_data *g_mgl = NULL;
static AMG_param g_amg;
static dCSRmat g_A;            /* caller's matrix, wrapped (not owned) */
static precond_data g_pcdata;
static precond g_pc;
/* the preconditioner linear_solver_dcsr_krylov_amg (itsolver.c:899-917)
 * picks for the cycle type of the last setup */
static void (*g_fct)(REAL *, REAL *, void *) = precond_amg;
static double *g_hist = NULL;  /* ||r|| seen by each preconditioner call */
static int g_hist_cap = 0, g_hist_n = 0;
static double g_setup_s = 0.0, g_solve_s = 0.0;

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* iparam: [0] max_levels [1] coarse_dof [2] cycle_type [3] smoother
 *         [4] presmooth [5] postsmooth [6] coarse_solver [7] aggregation_type
 *         [8] max_aggregation [9] coarse_scaling [10] print_level [11] amg maxit
 *         [12] amli_degree [13] nl_amli_krylov_type [14] AMG_type
 *         [15] smooth_filter
 * dparam: [0] strong_coupled [1] relaxation [2] amg tol [3] tentative_smooth */
static void fill_param(AMG_param *p, const int *ip, const double *dp)
{
    param_amg_init(p);
    p->max_levels = (SHORT)ip[0];
    p->coarse_dof = ip[1];
    p->cycle_type = (SHORT)ip[2];
    p->smoother = (SHORT)ip[3];
    p->presmooth_iter = (SHORT)ip[4];
    p->postsmooth_iter = (SHORT)ip[5];
    p->coarse_solver = (SHORT)ip[6];
    p->aggregation_type = (SHORT)ip[7];
    p->max_aggregation = ip[8];
    p->coarse_scaling = (SHORT)ip[9];
    p->print_level = (SHORT)ip[10];
    p->maxit = ip[11];
    p->amli_degree = (SHORT)ip[12];
    p->nl_amli_krylov_type = (SHORT)ip[13];
    p->AMG_type = (SHORT)ip[14];
    p->smooth_filter = (SHORT)ip[15];
    p->tentative_smooth = dp[3];
    p->strong_coupled = dp[0];
    p->relaxation = dp[1];
    p->tol = dp[2];
}

void ref_free(void)
{
    if (g_mgl) {
        amg_data_free(g_mgl, &g_amg);
        free(g_mgl);
        g_mgl = NULL;
    }
}

int ref_setup(int n, int nnz, int *ia, int *ja, double *val,
              const int *iparam, const double *dparam)
{
    ref_free();
    fill_param(&g_amg, iparam, dparam);
    g_A.row = n; g_A.col = n; g_A.nnz = nnz;
    g_A.IA = ia; g_A.JA = ja; g_A.val = val;
    g_mgl = amg_data_create(g_amg.max_levels);
    g_mgl[0].A = dcsr_create(n, n, nnz);
    dcsr_cp(&g_A, &g_mgl[0].A);
    g_mgl[0].b = dvec_create(n);
    g_mgl[0].x = dvec_create(n);
    double t0 = now_s();
    /* linear_solver_dcsr_krylov_amg's choice (itsolver.c:870-885) */
    SHORT status = g_amg.AMG_type == SA_AMG ? amg_setup_sa(g_mgl, &g_amg)
                                            : amg_setup_ua(g_mgl, &g_amg);
    g_setup_s = now_s() - t0;
    precond_data_null(&g_pcdata);
    param_amg_to_prec(&g_pcdata, &g_amg);
    g_pcdata.max_levels = g_mgl[0].num_levels;
    g_pcdata.mgl_data = g_mgl;
    g_pc.data = &g_pcdata;
    switch (g_amg.cycle_type) {
    case AMLI_CYCLE: g_fct = precond_amli; break;
    case NL_AMLI_CYCLE: g_fct = precond_nl_amli; break;
    case ADD_CYCLE: g_fct = precond_amg_add; break;
    default: g_fct = precond_amg; break;
    }
    g_pc.fct = g_fct;
    return status;
}

double ref_setup_seconds(void) { return g_setup_s; }
double ref_solve_seconds(void) { return g_solve_s; }
double ref_strong_coupled(void) { return g_amg.strong_coupled; }
int ref_num_levels(void) { return g_mgl ? g_mgl[0].num_levels : 0; }

/* out: [0] rows [1] nnz of A_l [2] columns of P_l (0 on the coarsest)
 *      [3] nnz of P_l [4] nnz of R_l                                        */
void ref_level_info(int l, int *out)
{
    dCSRmat *A = &g_mgl[l].A, *P = &g_mgl[l].P, *R = &g_mgl[l].R;
    out[0] = A->row; out[1] = A->nnz;
    out[2] = P->IA ? P->col : 0; out[3] = P->IA ? P->nnz : 0;
    out[4] = R->IA ? R->nnz : 0;
}

void ref_level_A(int l, int *ia, int *ja, double *val)
{
    dCSRmat *A = &g_mgl[l].A;
    memcpy(ia, A->IA, sizeof(int) * (A->row + 1));
    memcpy(ja, A->JA, sizeof(int) * A->nnz);
    memcpy(val, A->val, sizeof(double) * A->nnz);
}

/* aggregate map recovered from P: P(i, agg[i]) = 1, or -1 for an empty row */
void ref_level_agg(int l, int *agg)
{
    dCSRmat *P = &g_mgl[l].P;
    for (int i = 0; i < P->row; ++i)
        agg[i] = (P->IA[i + 1] > P->IA[i]) ? P->JA[P->IA[i]] : -1;
}

/* P of level l with its values (smoothed aggregation) */
void ref_level_P(int l, int *ia, int *ja, double *val)
{
    dCSRmat *P = &g_mgl[l].P;
    memcpy(ia, P->IA, sizeof(int) * (P->row + 1));
    memcpy(ja, P->JA, sizeof(int) * P->nnz);
    memcpy(val, P->val, sizeof(double) * P->nnz);
}

void ref_level_R(int l, int *ia, int *ja)
{
    dCSRmat *R = &g_mgl[l].R;
    memcpy(ia, R->IA, sizeof(int) * (R->row + 1));
    memcpy(ja, R->JA, sizeof(int) * R->nnz);
}

/* one application of the setup's preconditioner (precond_amg, precond.c:164,
 * or the one of its cycle type) */
void ref_precond(double *r, double *z) { g_fct(r, z, &g_pcdata); }

static void hist_precond(REAL *r, REAL *z, void *data)
{
    if (g_hist_n < g_hist_cap) {
        REAL s = 0.0;
        for (int i = 0; i < g_mgl[0].A.row; ++i) s += r[i] * r[i];
        g_hist[g_hist_n] = sqrt(s);
    }
    g_hist_n++;
    g_fct(r, z, data);
}

/* PCG with the AMG preconditioner; hist receives ||r|| at every
 * preconditioner call (r_0, r_1, ...), nhist the number of calls.          */
int ref_pcg(double *b, double *x, double tol, int maxit, int stop_type,
            int print_level, double *hist, int hist_cap, int *nhist)
{
    dvector bb, xx;
    bb.row = g_A.row; bb.val = b;
    xx.row = g_A.row; xx.val = x;
    g_hist = hist; g_hist_cap = hist ? hist_cap : 0; g_hist_n = 0;
    precond pc = g_pc;
    pc.fct = hist ? hist_precond : g_fct;
    double t0 = now_s();
    int it = dcsr_pcg(&g_A, &bb, &xx, &pc, tol, maxit, (SHORT)stop_type,
                      (SHORT)print_level);
    g_solve_s = now_s() - t0;
    if (nhist) *nhist = g_hist_n;
    g_hist = NULL; g_hist_cap = 0;
    return it;
}

/* Variable-restart GMRES (type 3: dcsr_pvgmres, krylov.c:4612) or its
 * flexible form (type 4: dcsr_pvfgmres, krylov.c:5974) with the AMG
 * preconditioner, as solver_dcsr_linear_itsolver (itsolver.c:135) calls
 * them; hist as for ref_pcg.                                               */
int ref_gmres(int type, double *b, double *x, double tol, int maxit, int restart,
              int stop_type, int print_level, double *hist, int hist_cap, int *nhist)
{
    dvector bb, xx;
    bb.row = g_A.row; bb.val = b;
    xx.row = g_A.row; xx.val = x;
    g_hist = hist; g_hist_cap = hist ? hist_cap : 0; g_hist_n = 0;
    precond pc = g_pc;
    pc.fct = hist ? hist_precond : g_fct;
    double t0 = now_s();
    int it = type == 4
        ? dcsr_pvfgmres(&g_A, &bb, &xx, &pc, tol, maxit, (SHORT)restart, (SHORT)stop_type,
                        (SHORT)print_level)
        : dcsr_pvgmres(&g_A, &bb, &xx, &pc, tol, maxit, (SHORT)restart, (SHORT)stop_type,
                       (SHORT)print_level);
    g_solve_s = now_s() - t0;
    if (nhist) *nhist = g_hist_n;
    g_hist = NULL; g_hist_cap = 0;
    return it;
}

/* Preconditioned MINRES (dcsr_pminres, krylov.c:2449) with the setup's
 * preconditioner (use_pc != 0) or none; hist as for ref_pcg.              */
int ref_minres(double *b, double *x, double tol, int maxit, int stop_type, int use_pc,
               double *hist, int hist_cap, int *nhist)
{
    dvector bb, xx;
    bb.row = g_A.row; bb.val = b;
    xx.row = g_A.row; xx.val = x;
    g_hist = hist; g_hist_cap = hist ? hist_cap : 0; g_hist_n = 0;
    precond pc = g_pc;
    pc.fct = hist ? hist_precond : g_fct;
    double t0 = now_s();
    int it = dcsr_pminres(&g_A, &bb, &xx, use_pc ? &pc : NULL, tol, maxit, (SHORT)stop_type, 0);
    g_solve_s = now_s() - t0;
    if (nhist) *nhist = g_hist_n;
    g_hist = NULL; g_hist_cap = 0;
    return it;
}

/* Generalized CG (dcsr_pgcg, krylov.c:2309) with the setup's
 * preconditioner; hist as for ref_pcg.                                     */
int ref_gcg(double *b, double *x, double tol, int maxit, int print_level, double *hist,
            int hist_cap, int *nhist)
{
    dvector bb, xx;
    bb.row = g_A.row; bb.val = b;
    xx.row = g_A.row; xx.val = x;
    g_hist = hist; g_hist_cap = hist ? hist_cap : 0; g_hist_n = 0;
    precond pc = g_pc;
    pc.fct = hist ? hist_precond : g_fct;
    double t0 = now_s();
    int it = dcsr_pgcg(&g_A, &bb, &xx, &pc, tol, maxit, 1, (SHORT)print_level);
    g_solve_s = now_s() - t0;
    if (nhist) *nhist = g_hist_n;
    g_hist = NULL; g_hist_cap = 0;
    return it;
}

/* amg_amli_coef (parameters.c:714) */
void ref_amli_coef(double lambda_max, double lambda_min, int degree, double *coef)
{
    amg_amli_coef(lambda_max, lambda_min, degree, coef);
}

/* ---- kernel-level entry points on caller arrays -------------------------- */
static dCSRmat wrap(int n, int m, int nnz, int *ia, int *ja, double *val)
{
    dCSRmat A;
    A.row = n; A.col = m; A.nnz = nnz; A.IA = ia; A.JA = ja; A.val = val;
    return A;
}

void ref_mxv(int n, int nnz, int *ia, int *ja, double *val, double *x, double *y)
{
    dCSRmat A = wrap(n, n, nnz, ia, ja, val);
    dcsr_mxv(&A, x, y);
}

void ref_aAxpy(double alpha, int n, int nnz, int *ia, int *ja, double *val,
               double *x, double *y)
{
    dCSRmat A = wrap(n, n, nnz, ia, ja, val);
    dcsr_aAxpy(alpha, &A, x, y);
}

/* forward != 0: the pre-smoothing call of mgcycle (mgcycle.c:289);
 * forward == 0: the post-smoothing call (mgcycle.c:397).                   */
void ref_smooth(int smoother, int forward, int sweeps, double relax, int n,
                int nnz, int *ia, int *ja, double *val, double *b, double *x)
{
    dCSRmat A = wrap(n, n, nnz, ia, ja, val);
    dvector bb, xx;
    bb.row = n; bb.val = b; xx.row = n; xx.val = x;
    int i0 = forward ? 0 : n - 1, i1 = forward ? n - 1 : 0, s = forward ? 1 : -1;
    /* the argument pattern of dcsr_presmoothing / dcsr_postsmoothing,
     * with istart = 0, iend = n-1, istep = +1 (pre) or -1 (post) */
    const int is = 0, ie = n - 1, st = forward ? 1 : -1;
    switch (smoother) {
    case SMOOTHER_JACOBI: smoother_dcsr_jacobi(&xx, i0, i1, s, &A, &bb, sweeps); break;
    case SMOOTHER_GS: smoother_dcsr_gs(&xx, i0, i1, s, &A, &bb, sweeps); break;
    case SMOOTHER_SGS: smoother_dcsr_sgs(&xx, &A, &bb, sweeps); break;
    case SMOOTHER_SOR: smoother_dcsr_sor(&xx, i0, i1, s, &A, &bb, sweeps, relax); break;
    case SMOOTHER_L1DIAG: smoother_dcsr_L1diag(&xx, i0, i1, s, &A, &bb, sweeps); break;
    case SMOOTHER_SSOR:
        if (forward) {
            smoother_dcsr_sor(&xx, is, ie, st, &A, &bb, sweeps, relax);
            smoother_dcsr_sor(&xx, ie, is, -st, &A, &bb, sweeps, relax);
        } else {
            smoother_dcsr_sor(&xx, is, ie, -st, &A, &bb, sweeps, relax);
            smoother_dcsr_sor(&xx, ie, is, st, &A, &bb, sweeps, relax);
        }
        break;
    case SMOOTHER_GSOR:
        if (forward) {
            smoother_dcsr_gs(&xx, is, ie, st, &A, &bb, sweeps);
            smoother_dcsr_sor(&xx, ie, is, -st, &A, &bb, sweeps, relax);
        } else {
            smoother_dcsr_sor(&xx, is, ie, -st, &A, &bb, sweeps, relax);
            smoother_dcsr_gs(&xx, ie, is, st, &A, &bb, sweeps);
        }
        break;
    case SMOOTHER_SGSOR:
        if (forward) {
            smoother_dcsr_gs(&xx, is, ie, st, &A, &bb, sweeps);
            smoother_dcsr_gs(&xx, ie, is, -st, &A, &bb, sweeps);
            smoother_dcsr_sor(&xx, is, ie, st, &A, &bb, sweeps, relax);
            smoother_dcsr_sor(&xx, ie, is, -st, &A, &bb, sweeps, relax);
        } else {
            smoother_dcsr_sor(&xx, is, ie, -st, &A, &bb, sweeps, relax);
            smoother_dcsr_sor(&xx, ie, is, st, &A, &bb, sweeps, relax);
            smoother_dcsr_gs(&xx, is, ie, -st, &A, &bb, sweeps);
            smoother_dcsr_gs(&xx, ie, is, st, &A, &bb, sweeps);
        }
        break;
    default: break;
    }
}

/* Galerkin product for aggregation, dcsr_rap_agg (sparse.c:2557); two calls:
 * first with ia_out only (sizes), then with all outputs.                     */
static dCSRmat g_rap = {0};
int ref_rap_agg(int n, int nnz, int *ia, int *ja, double *val, int nc,
                const int *agg, int *rap_ia, int *rap_ja, double *rap_val)
{
    if (!rap_ja) {
        dCSRmat A = wrap(n, n, nnz, ia, ja, val), P, R;
        int np = 0;
        for (int i = 0; i < n; ++i) np += agg[i] >= 0;
        P = dcsr_create(n, nc, np);
        for (int i = 0, k = 0; i < n; ++i) {
            P.IA[i] = k;
            if (agg[i] >= 0) { P.JA[k] = agg[i]; P.val[k] = 1.0; ++k; }
        }
        P.IA[n] = np;
        dcsr_trans(&P, &R);
        if (g_rap.IA) dcsr_free(&g_rap);
        dcsr_rap_agg(&R, &A, &P, &g_rap);
        dcsr_free(&P); dcsr_free(&R);
        memcpy(rap_ia, g_rap.IA, sizeof(int) * (nc + 1));
        return g_rap.nnz;
    }
    memcpy(rap_ja, g_rap.JA, sizeof(int) * g_rap.nnz);
    memcpy(rap_val, g_rap.val, sizeof(double) * g_rap.nnz);
    return g_rap.nnz;
}

/* srand() in this process: the reference's HEC aggregation draws its row
 * order from rand() (iarray_shuffle, array.c:302) */
void ref_srand(unsigned seed) { srand(seed); }

/* ---- UA-AMG for BSR matrices: amg_setup_ua_bsr (amg_setup_ua.c:145),
 * precond_dbsr_amg (precond.c:1311) and linear_solver_dbsr_krylov_amg
 * (itsolver.c:2104), on one global hierarchy.  ip/dp as fill_param.       */
static AMG_data_bsr *g_bmgl = NULL;
static AMG_param g_bamg;
static dBSRmat g_bA;
static precond_data_bsr g_bpd;

static dBSRmat wrap_bsr(int nrow, int nnzb, int nb, int *ia, int *ja, double *val)
{
    dBSRmat A;
    A.ROW = nrow; A.COL = nrow; A.NNZ = nnzb; A.nb = nb; A.storage_manner = 0;
    A.IA = ia; A.JA = ja; A.val = val;
    return A;
}

void ref_bsr_free(void)
{
    if (g_bmgl) {
        amg_data_bsr_free(g_bmgl);
        g_bmgl = NULL;
    }
}

int ref_bsr_setup(int nrow, int nnzb, int nb, int *ia, int *ja, double *val,
                  const int *iparam, const double *dparam)
{
    ref_bsr_free();
    fill_param(&g_bamg, iparam, dparam);
    g_bA = wrap_bsr(nrow, nnzb, nb, ia, ja, val);
    g_bmgl = amg_data_bsr_create(g_bamg.max_levels);
    g_bmgl[0].A = dbsr_create(nrow, nrow, nnzb, nb, 0);
    g_bmgl[0].b = dvec_create(nrow * nb);
    g_bmgl[0].x = dvec_create(nrow * nb);
    dbsr_cp(&g_bA, &g_bmgl[0].A);
    double t0 = now_s();
    SHORT status = amg_setup_ua_bsr(g_bmgl, &g_bamg);
    g_setup_s = now_s() - t0;
    /* the preconditioner data of linear_solver_dbsr_krylov_amg */
    memset(&g_bpd, 0, sizeof(g_bpd));
    g_bpd.print_level = g_bamg.print_level;
    g_bpd.maxit = g_bamg.maxit;
    g_bpd.tol = g_bamg.tol;
    g_bpd.cycle_type = g_bamg.cycle_type;
    g_bpd.smoother = g_bamg.smoother;
    g_bpd.presmooth_iter = g_bamg.presmooth_iter;
    g_bpd.postsmooth_iter = g_bamg.postsmooth_iter;
    g_bpd.relaxation = g_bamg.relaxation;
    g_bpd.coarse_solver = g_bamg.coarse_solver;
    g_bpd.coarse_scaling = g_bamg.coarse_scaling;
    g_bpd.amli_degree = g_bamg.amli_degree;
    g_bpd.amli_coef = g_bamg.amli_coef;
    g_bpd.tentative_smooth = g_bamg.tentative_smooth;
    g_bpd.max_levels = g_bmgl[0].num_levels;
    g_bpd.mgl_data = g_bmgl;
    g_bpd.A = &g_bA;
    return status;
}

int ref_bsr_num_levels(void) { return g_bmgl ? g_bmgl[0].num_levels : 0; }

/* out: ROW, NNZ of level l */
void ref_bsr_level_info(int l, int *out)
{
    out[0] = g_bmgl[l].A.ROW;
    out[1] = g_bmgl[l].A.NNZ;
}

void ref_bsr_level_A(int l, int *ia, int *ja, double *val)
{
    const dBSRmat *A = &g_bmgl[l].A;
    memcpy(ia, A->IA, sizeof(int) * (A->ROW + 1));
    memcpy(ja, A->JA, sizeof(int) * A->NNZ);
    memcpy(val, A->val, sizeof(double) * A->NNZ * A->nb * A->nb);
}

/* block aggregate of every row of level l (the column of its P block, -1
 * for an empty row) */
void ref_bsr_level_agg(int l, int *agg)
{
    const dBSRmat *P = &g_bmgl[l].P;
    for (int i = 0; i < P->ROW; ++i)
        agg[i] = P->IA[i + 1] > P->IA[i] ? P->JA[P->IA[i]] : -1;
}

void ref_bsr_precond(double *r, double *z) { precond_dbsr_amg(r, z, &g_bpd); }

/* linear_solver_dbsr_krylov_amg (itsolver.c:2104) on its own hierarchy:
 * amg_setup_ua_bsr, precond_dbsr_amg, then the Krylov method of
 * solver_dbsr_linear_itsolver (type 1, 3 or 4).  Type 1 calls dbsr_pcg:
 * dbsr_pcg_w_cond_est takes the same iterates and adds a LAPACK condition
 * estimate, and this build has no LAPACK.                                   */
int ref_bsr_krylov_amg(int nrow, int nnzb, int nb, int *ia, int *ja, double *val,
                       double *b, double *x, int type, double tol, int maxit,
                       int stop_type, int restart, const int *iparam,
                       const double *dparam)
{
    int st = ref_bsr_setup(nrow, nnzb, nb, ia, ja, val, iparam, dparam);
    if (st < 0) return st;
    precond pc;
    pc.data = &g_bpd;
    pc.fct = precond_dbsr_amg;
    dvector bv, xv;
    bv.row = nrow * nb; bv.val = b;
    xv.row = nrow * nb; xv.val = x;
    double t0 = now_s();
    int it_n;
    switch (type) {
    case 1: it_n = dbsr_pcg(&g_bA, &bv, &xv, &pc, tol, maxit, (SHORT)stop_type, 0); break;
    case 3: it_n = dbsr_pvgmres(&g_bA, &bv, &xv, &pc, tol, maxit, (SHORT)restart,
                                (SHORT)stop_type, 0); break;
    case 4: it_n = dbsr_pvfgmres(&g_bA, &bv, &xv, &pc, tol, maxit, (SHORT)restart,
                                 (SHORT)stop_type, 0); break;
    default: it_n = ERROR_SOLVER_TYPE; break;
    }
    g_solve_s = now_s() - t0;
    ref_bsr_free();
    return it_n;
}
