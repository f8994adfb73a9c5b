/*
 * hzoracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * A plain-C restatement of HAZmath's UA-AMG preconditioned CG path, written
 * from the reference's behaviour (each function cites the reference
 * file:line it follows), and of the configurations around it: VMB and HEC
 * aggregation (with the C library's rand() stream), smoothed aggregation,
 * the block (BSR) setup and cycle, the AMLI / nonlinear AMLI / additive
 * cycles, GCG, MINRES and (flexible) GMRES.  It is the checker for the CUDA
 * library: only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 * It is pinned against the reference itself (oracle/_ref, built by
 * oracle/build_ref.sh) through the golden fixtures in tests/golden/.
 *
 * Build: see oracle/Makefile (gcc -O3 -ffp-contract=off, no FMA), so that
 * every sum and product is rounded separately, in the reference's order.
 *
 * One deliberate difference: the coarsest level is solved by a dense
 * Cholesky factorisation (the product's method) instead of the reference's
 * sparse LDL^T with identity permutation (src/solver/hazmath_direct.c:633);
 * both are direct solves and agree to rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SMALLREAL 1e-20
#define BIGREAL 1e20
#define UNPT (-1)

typedef struct {
    int n, m, nnz;
    int *ia, *ja;
    double *val;
} ocsr;

/* a preconditioner z = B r for the Krylov restatements (NULL: B = I) */
typedef void (*or_pcfn)(const double *in, double *out, void *ctx);

static void ocsr_free(ocsr *A)
{
    free(A->ia); free(A->ja); free(A->val);
    memset(A, 0, sizeof(*A));
}

/* ---------------------------------------------------------------------------
 * Sparse kernels (src/utilities/sparse.c)
 * ------------------------------------------------------------------------- */

/* dcsr_mxv sparse.c:1456-1590: y_i = sum_k a_k x_{ja_k}, starting at 0.0,
 * CSR order (the unrolled cases keep that order). */
void or_mxv(int n, const int *ia, const int *ja, const double *a,
            const double *x, double *y)
{
    for (int i = 0; i < n; ++i) {
        double t = 0.0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) t += a[k] * x[ja[k]];
        y[i] = t;
    }
}

/* dcsr_aAxpy sparse.c:1693-1735: y += alpha A x with the alpha = +-1 cases
 * adding/subtracting the row sum directly. */
void or_aAxpy(double alpha, int n, const int *ia, const int *ja,
              const double *a, const double *x, double *y)
{
    for (int i = 0; i < n; ++i) {
        double t = 0.0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) t += a[k] * x[ja[k]];
        if (alpha == 1.0) y[i] += t;
        else if (alpha == -1.0) y[i] -= t;
        else y[i] += t * alpha;
    }
}

/* dcsr_mxv_agg sparse.c:1663-1678 applied to R: y_c = sum of x over the
 * fine rows of the aggregate, in R's (ascending) order, from 0.0 */
static void or_restrict(int nc, const int *ria, const int *rja,
                        const double *x, double *y)
{
    for (int c = 0; c < nc; ++c) {
        double t = 0.0;
        for (int k = ria[c]; k < ria[c + 1]; ++k) t += x[rja[k]];
        y[c] = t;
    }
}

/* dcsr_aAxpy_agg sparse.c:1748-1785 applied to P (one unit entry per
 * non-empty row, agg[i] < 0 for an empty row) */
static void or_prolong(double alpha, int n, const int *agg, const double *xc,
                       double *x)
{
    for (int i = 0; i < n; ++i) {
        double t = 0.0;
        if (agg[i] >= 0) t += xc[agg[i]];
        if (alpha == 1.0) x[i] += t;
        else if (alpha == -1.0) x[i] -= t;
        else x[i] += t * alpha;
    }
}

/* dcsr_getdiag sparse.c:2168-2188: first diagonal entry of each row (0.0 if
 * none: the reference's dvec_alloc leaves calloc'd zeros) */
static void or_getdiag(int n, const int *ia, const int *ja, const double *a,
                       double *d)
{
    for (int i = 0; i < n; ++i) {
        d[i] = 0.0;
        for (int k = ia[i]; k < ia[i + 1]; ++k)
            if (ja[k] == i) { d[i] = a[k]; break; }
    }
}

/* ---------------------------------------------------------------------------
 * Aggregation (src/solver/amg_setup_ua.c)
 * ------------------------------------------------------------------------- */

/* construct_strongly_coupled amg_setup_ua.c:375-455: keep a_ij if j == i, or
 * a_ij^2 >= theta^2 |a_ii a_jj| and a_ij < 0; input column order. */
int or_strength(int n, const int *ia, const int *ja, const double *a,
                double theta, int *nia, int *nja, double *nval)
{
    double *d = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    or_getdiag(n, ia, ja, a, d);
    const double th2 = theta * theta;
    int idx = 0;
    for (int i = 0; i < n; ++i) {
        nia[i] = idx;
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            int j = ja[k];
            double v = a[k];
            if (j == i || ((v * v) >= th2 * fabs(d[i] * d[j]) && v < 0.0)) {
                nja[idx] = j; nval[idx] = v; ++idx;
            }
        }
    }
    nia[n] = idx;
    free(d);
    return idx;
}

/* heavy_edg amg_setup_ua.c:864-893: start at position n0, walk to n1, keep
 * the first strictly larger weight seen. */
static int or_heavy(const double *w, const int *id, int n0, int n1)
{
    int step = (n0 > n1) ? -1 : 1;
    int best = id[n0];
    double bw = w[n0];
    for (int j = n0; j != n1 + step; j += step)
        if (w[j] > bw && id[j] >= 0) { bw = w[j]; best = id[j]; }
    return best;
}

/* aggregation_hem amg_setup_ua.c:913-1050 on the strength graph.
 * Returns the number of aggregates, or -1 for the "isolated point on the
 * second pass" case where the reference calls exit(17). */
int or_hem(int n, const int *ia, const int *ja, const double *a, int *mask)
{
    int maxdeg = 1;
    for (int k = 0; k < n; ++k) {
        int l = ia[k + 1] - ia[k];
        if (l > maxdeg) maxdeg = l;
        mask[k] = (l > 1) ? -1 : -2;      /* pass 0: only a diagonal -> -2 */
    }
    double *w = (double *)malloc(sizeof(double) * maxdeg);
    int *iw = (int *)malloc(sizeof(int) * maxdeg);
    int *cnt = (int *)calloc(n > 0 ? n : 1, sizeof(int));
    int nc = 0;
    for (int k = 0; k < n; ++k) {         /* pass 1: heavy edge matching */
        if (mask[k] != -1) continue;
        int iz = 0;
        for (int p = ia[k]; p < ia[k + 1]; ++p) {
            int j = ja[p];
            if (mask[j] < 0 && j != k) { w[iz] = fabs(a[p]); iw[iz] = j; ++iz; }
        }
        if (iz) {
            int pick = or_heavy(w, iw, iz - 1, 0);
            mask[k] = nc; mask[pick] = nc; cnt[nc] += 2; ++nc;
        }
    }
    int status = nc;
    for (int k = 0; k < n; ++k) {         /* pass 2: attach leftovers */
        if (mask[k] != -1) continue;
        int iz = 0;
        for (int p = ia[k]; p < ia[k + 1]; ++p) {
            int kc = mask[ja[p]];
            if (kc >= 0) { w[iz] = (double)(-cnt[kc]); iw[iz] = kc; ++iz; }
        }
        if (!iz) { status = -1; break; }
        int kc = or_heavy(w, iw, 0, iz - 1);
        mask[k] = kc; cnt[kc]++;
    }
    for (int k = 0; k < n; ++k)           /* pass 3 */
        if (mask[k] < 0) mask[k] = UNPT;
    free(w); free(iw); free(cnt);
    return status;
}

/* dcsr_trans sparse.c:770-862 on P: R rows list fine indices ascending */
static void or_trans_agg(int n, int nc, const int *agg, int *ria, int *rja)
{
    memset(ria, 0, sizeof(int) * (nc + 1));
    for (int i = 0; i < n; ++i) if (agg[i] >= 0) ria[agg[i] + 1]++;
    for (int c = 0; c < nc; ++c) ria[c + 1] += ria[c];
    int *pos = (int *)malloc(sizeof(int) * (nc > 0 ? nc : 1));
    memcpy(pos, ria, sizeof(int) * nc);
    for (int i = 0; i < n; ++i) if (agg[i] >= 0) rja[pos[agg[i]]++] = i;
    free(pos);
}

/* dcsr_rap_agg sparse.c:2557-2690.  Row c of A_c: slot 0 is the diagonal
 * (starting at 0.0 and accumulated), further columns in first-encounter
 * order over (fine row i in R row c, ascending) x (A row i, CSR order) x
 * (P row of the column); a new column takes the entry's value, a known one
 * adds it.  Rows of P with agg < 0 contribute nothing. */
int or_rap_agg(int n, const int *ia, const int *ja, const double *a, int nc,
               const int *agg, const int *ria, const int *rja, ocsr *Ac)
{
    int *slot = (int *)malloc(sizeof(int) * (nc > 0 ? nc : 1));
    for (int c = 0; c < nc; ++c) slot[c] = -1;
    /* symbolic */
    int *cia = (int *)malloc(sizeof(int) * (nc + 1));
    int cnt = 0;
    for (int c = 0; c < nc; ++c) {
        int rb = cnt;
        cia[c] = rb;
        slot[c] = cnt++;
        for (int q = ria[c]; q < ria[c + 1]; ++q) {
            int i = rja[q];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                int cc = agg[ja[k]];
                if (cc < 0) continue;
                if (slot[cc] < rb) slot[cc] = cnt++;
            }
        }
    }
    cia[nc] = cnt;
    int *cja = (int *)malloc(sizeof(int) * (cnt > 0 ? cnt : 1));
    double *cv = (double *)malloc(sizeof(double) * (cnt > 0 ? cnt : 1));
    for (int c = 0; c < nc; ++c) slot[c] = -1;
    cnt = 0;
    for (int c = 0; c < nc; ++c) {
        int rb = cnt;
        slot[c] = cnt;
        cja[cnt] = c; cv[cnt] = 0.0; ++cnt;
        for (int q = ria[c]; q < ria[c + 1]; ++q) {
            int i = rja[q];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                int cc = agg[ja[k]];
                if (cc < 0) continue;
                if (slot[cc] < rb) {
                    slot[cc] = cnt; cja[cnt] = cc; cv[cnt] = a[k]; ++cnt;
                } else {
                    cv[slot[cc]] += a[k];
                }
            }
        }
    }
    free(slot);
    Ac->n = Ac->m = nc; Ac->nnz = cnt; Ac->ia = cia; Ac->ja = cja; Ac->val = cv;
    return cnt;
}

/* ---------------------------------------------------------------------------
 * Smoothers (src/solver/smoother.c) and their mgcycle dispatch
 * ------------------------------------------------------------------------- */

/* smoother_dcsr_jacobi smoother.c:35-100 (w = 1, t from old u) */
static void or_jacobi(int n, const int *ia, const int *ja, const double *a,
                      const double *b, double *u, int sweeps, double *t,
                      double *d)
{
    const double w = 1.0;
    for (int i = 0; i < n; ++i) d[i] = 0.0;
    while (sweeps--) {
        for (int i = 0; i < n; ++i) {
            t[i] = b[i];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                if (ja[k] != i) t[i] -= a[k] * u[ja[k]];
                else d[i] = a[k];
            }
        }
        for (int i = 0; i < n; ++i)
            if (fabs(d[i]) > SMALLREAL) u[i] = (1 - w) * u[i] + w * t[i] / d[i];
    }
}

/* smoother_dcsr_gs smoother.c:109-190: in place, d = 1/a_ii kept from the
 * last row that had a usable diagonal */
static void or_gs(int n, const int *ia, const int *ja, const double *a,
                  const double *b, double *u, int sweeps, int forward)
{
    double d = 0.0;
    while (sweeps--) {
        for (int s = 0; s < n; ++s) {
            int i = forward ? s : n - 1 - s;
            double t = b[i];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                if (ja[k] != i) t -= a[k] * u[ja[k]];
                else if (fabs(a[k]) > SMALLREAL) d = 1.e+0 / a[k];
            }
            u[i] = t * d;
        }
    }
}

/* smoother_dcsr_sgs smoother.c:196-250 (backward sweep from n-2) */
static void or_sgs(int n, const int *ia, const int *ja, const double *a,
                   const double *b, double *u, int sweeps)
{
    double d = 0.0;
    while (sweeps--) {
        for (int i = 0; i < n; ++i) {
            double t = b[i];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                if (ja[k] != i) t -= a[k] * u[ja[k]];
                else d = a[k];
            }
            if (fabs(d) > SMALLREAL) u[i] = t / d;
        }
        for (int i = n - 2; i >= 0; --i) {
            double t = b[i];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                if (ja[k] != i) t -= a[k] * u[ja[k]];
                else d = a[k];
            }
            if (fabs(d) > SMALLREAL) u[i] = t / d;
        }
    }
}

/* smoother_dcsr_sor smoother.c:257-318 */
static void or_sor(int n, const int *ia, const int *ja, const double *a,
                   const double *b, double *u, int sweeps, int forward,
                   double w)
{
    double d = 0.0;
    while (sweeps--) {
        for (int s = 0; s < n; ++s) {
            int i = forward ? s : n - 1 - s;
            double t = b[i];
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                if (ja[k] != i) t -= a[k] * u[ja[k]];
                else d = a[k];
            }
            if (fabs(d) > SMALLREAL) u[i] = w * (t / d) + (1 - w) * u[i];
        }
    }
}

/* smoother_dcsr_L1diag smoother.c:324-390; omega (may be NULL) scales the
 * update for the learned form: u_i += omega_i * t_i / d_i, which is the
 * reference for omega == NULL. */
static void or_l1(int n, const int *ia, const int *ja, const double *a,
                  const double *b, double *u, int sweeps, double *t,
                  double *d, const float *omega)
{
    while (sweeps--) {
        for (int i = 0; i < n; ++i) {
            t[i] = b[i]; d[i] = 0.0;
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                t[i] -= a[k] * u[ja[k]];
                d[i] += fabs(a[k]);
            }
        }
        for (int i = 0; i < n; ++i)
            if (fabs(d[i]) > SMALLREAL) {
                if (omega) u[i] += (double)omega[i] * (t[i] / d[i]);
                else u[i] += t[i] / d[i];
            }
    }
}

/* smoother ids as in include/macro.h */
enum { S_JACOBI = 1, S_GS = 2, S_SGS = 3, S_SOR = 5, S_SSOR = 6, S_GSOR = 7,
       S_SGSOR = 8, S_L1 = 10 };

/* dcsr_presmoothing / dcsr_postsmoothing mgcycle.c:76-240 */
int or_smooth(int smoother, int pre, int sweeps, double relax, int n,
              const int *ia, const int *ja, const double *a, const double *b,
              double *u, const float *omega)
{
    double *t = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    double *d = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    int fw = pre ? 1 : 0;
    int rc = 0;
    switch (smoother) {
    case S_JACOBI: or_jacobi(n, ia, ja, a, b, u, sweeps, t, d); break;
    case S_GS: or_gs(n, ia, ja, a, b, u, sweeps, fw); break;
    case S_SGS: or_sgs(n, ia, ja, a, b, u, sweeps); break;
    case S_SOR: or_sor(n, ia, ja, a, b, u, sweeps, fw, relax); break;
    case S_SSOR:   /* forward then backward in both calls (mgcycle.c:100, :187) */
        or_sor(n, ia, ja, a, b, u, sweeps, 1, relax);
        or_sor(n, ia, ja, a, b, u, sweeps, 0, relax);
        break;
    case S_GSOR:
        if (pre) { or_gs(n, ia, ja, a, b, u, sweeps, 1); or_sor(n, ia, ja, a, b, u, sweeps, 0, relax); }
        else { or_sor(n, ia, ja, a, b, u, sweeps, 1, relax); or_gs(n, ia, ja, a, b, u, sweeps, 0); }
        break;
    case S_SGSOR:
        if (pre) {
            or_gs(n, ia, ja, a, b, u, sweeps, 1); or_gs(n, ia, ja, a, b, u, sweeps, 0);
            or_sor(n, ia, ja, a, b, u, sweeps, 1, relax); or_sor(n, ia, ja, a, b, u, sweeps, 0, relax);
        } else {
            or_sor(n, ia, ja, a, b, u, sweeps, 1, relax); or_sor(n, ia, ja, a, b, u, sweeps, 0, relax);
            or_gs(n, ia, ja, a, b, u, sweeps, 1); or_gs(n, ia, ja, a, b, u, sweeps, 0);
        }
        break;
    case S_L1: or_l1(n, ia, ja, a, b, u, sweeps, t, d, omega); break;
    default: rc = -31;
    }
    free(t); free(d);
    return rc;
}

/* ---------------------------------------------------------------------------
 * Dense Cholesky for the coarsest level
 * ------------------------------------------------------------------------- */
static int or_chol(int n, double *L)  /* lower factor in place, row-major */
{
    for (int j = 0; j < n; ++j) {
        double s = L[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) s -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
        if (!(s > 0.0)) return -22;
        s = sqrt(s);
        L[(size_t)j * n + j] = s;
        for (int i = j + 1; i < n; ++i) {
            double t = L[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) t -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
            L[(size_t)i * n + j] = t / s;
        }
    }
    return 0;
}

static void or_chol_solve(int n, const double *L, const double *b, double *x)
{
    for (int i = 0; i < n; ++i) {
        double t = b[i];
        for (int k = 0; k < i; ++k) t -= L[(size_t)i * n + k] * x[k];
        x[i] = t / L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double t = x[i];
        for (int k = i + 1; k < n; ++k) t -= L[(size_t)k * n + i] * x[k];
        x[i] = t / L[(size_t)i * n + i];
    }
}

/* ---------------------------------------------------------------------------
 * Hierarchy, setup and cycle
 * ------------------------------------------------------------------------- */
#define OR_MAXLVL 20

typedef struct {
    /* parameters (AMG_param subset) */
    int max_levels, coarse_dof, cycle_type, smoother, pre, post;
    int coarse_solver, aggregation_type, coarse_scaling, amg_maxit;
    double strong_coupled, relaxation;
    /* hierarchy */
    int nl;
    ocsr A[OR_MAXLVL];
    int *agg[OR_MAXLVL];
    int nc[OR_MAXLVL];
    int *ria[OR_MAXLVL], *rja[OR_MAXLVL];
    double *b[OR_MAXLVL], *x[OR_MAXLVL], *w[OR_MAXLVL];
    double *Lc;      /* dense Cholesky factor of the coarsest level */
    const float *omega; /* learned fine-level weights (NULL: plain) */
} or_amg;

static or_amg g_or;

void or_free(void)
{
    for (int l = 0; l < g_or.nl; ++l) {
        ocsr_free(&g_or.A[l]);
        free(g_or.agg[l]); free(g_or.ria[l]); free(g_or.rja[l]);
        free(g_or.b[l]); free(g_or.x[l]); free(g_or.w[l]);
    }
    free(g_or.Lc);
    memset(&g_or, 0, sizeof(g_or));
}

/* same parameter vectors as the reference harness (oracle/ref_harness.c) */
int or_setup(int n, int nnz, const int *ia, const int *ja, const double *val,
             const int *ip, const double *dp)
{
    or_free();
    or_amg *G = &g_or;
    G->max_levels = ip[0]; G->coarse_dof = ip[1]; G->cycle_type = ip[2];
    G->smoother = ip[3]; G->pre = ip[4]; G->post = ip[5];
    G->coarse_solver = ip[6]; G->aggregation_type = ip[7];
    G->coarse_scaling = ip[9]; G->amg_maxit = ip[11];
    G->strong_coupled = dp[0]; G->relaxation = dp[1];
    if (G->aggregation_type != 5) return -32;   /* HEM only in the oracle */
    ocsr *A0 = &G->A[0];
    A0->n = A0->m = n; A0->nnz = nnz;
    A0->ia = (int *)malloc(sizeof(int) * (n + 1));
    A0->ja = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    A0->val = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    memcpy(A0->ia, ia, sizeof(int) * (n + 1));
    memcpy(A0->ja, ja, sizeof(int) * nnz);
    memcpy(A0->val, val, sizeof(double) * nnz);
    /* amg_setup_ua.c:1233 min_cdof is a SHORT */
    const short min_cdof = (short)(G->coarse_dof > 1 ? G->coarse_dof : 1);
    int lvl = 0;
    while (G->A[lvl].n > min_cdof && lvl < G->max_levels - 1) {
        ocsr *A = &G->A[lvl];
        int m = A->n;
        int *nia = (int *)malloc(sizeof(int) * (m + 1));
        int *nja = (int *)malloc(sizeof(int) * (A->nnz > 0 ? A->nnz : 1));
        double *nv = (double *)malloc(sizeof(double) * (A->nnz > 0 ? A->nnz : 1));
        or_strength(m, A->ia, A->ja, A->val, G->strong_coupled, nia, nja, nv);
        int *agg = (int *)malloc(sizeof(int) * (m > 0 ? m : 1));
        int nagg = or_hem(m, nia, nja, nv, agg);
        free(nia); free(nja); free(nv);
        if (nagg < 0) { free(agg); return -33; }
        /* adaptive threshold, amg_setup_ua.c:1325-1328 */
        if (nagg * 4 > m) G->strong_coupled /= 2;
        else if (nagg * 1.25 < m) G->strong_coupled *= 2;
        if (nagg < 1) { free(agg); break; }       /* P.col < MIN_CDOF */
        G->agg[lvl] = agg;
        G->nc[lvl] = nagg;
        G->ria[lvl] = (int *)malloc(sizeof(int) * (nagg + 1));
        G->rja[lvl] = (int *)malloc(sizeof(int) * (m > 0 ? m : 1));
        or_trans_agg(m, nagg, agg, G->ria[lvl], G->rja[lvl]);
        or_rap_agg(m, A->ia, A->ja, A->val, nagg, agg, G->ria[lvl], G->rja[lvl],
                   &G->A[lvl + 1]);
        ++lvl;
    }
    G->nl = lvl + 1;
    for (int l = 0; l < G->nl; ++l) {
        int m = G->A[l].n > 0 ? G->A[l].n : 1;
        G->b[l] = (double *)calloc(m, sizeof(double));
        G->x[l] = (double *)calloc(m, sizeof(double));
        G->w[l] = (double *)calloc(m, sizeof(double));
    }
    /* coarsest: dense factorisation (coarse_solver 32) */
    if (G->coarse_solver == 32) {
        ocsr *C = &G->A[G->nl - 1];
        /* amg_setup_ua.c:1392-1398: the coarsest matrix is replaced by its
         * transpose with ascending column indices (dcsr_transz, p = NULL)
         * before the factorisation */
        {
            int m = C->n, nz = C->nnz;
            int *tia = (int *)calloc(m + 1, sizeof(int));
            int *tja = (int *)malloc(sizeof(int) * (nz > 0 ? nz : 1));
            double *tv = (double *)malloc(sizeof(double) * (nz > 0 ? nz : 1));
            for (int k = 0; k < nz; ++k) tia[C->ja[k] + 1]++;
            for (int i = 0; i < m; ++i) tia[i + 1] += tia[i];
            int *pos = (int *)malloc(sizeof(int) * (m > 0 ? m : 1));
            memcpy(pos, tia, sizeof(int) * m);
            for (int i = 0; i < m; ++i)
                for (int k = C->ia[i]; k < C->ia[i + 1]; ++k) {
                    int q = pos[C->ja[k]]++;
                    tja[q] = i; tv[q] = C->val[k];
                }
            free(pos);
            free(C->ia); free(C->ja); free(C->val);
            C->ia = tia; C->ja = tja; C->val = tv;
        }
        int m = C->n;
        G->Lc = (double *)calloc((size_t)m * m > 0 ? (size_t)m * m : 1, sizeof(double));
        for (int i = 0; i < m; ++i)
            for (int k = C->ia[i]; k < C->ia[i + 1]; ++k)
                G->Lc[(size_t)i * m + C->ja[k]] += C->val[k];
        if (or_chol(m, G->Lc)) return -22;
    }
    return 0;
}

int or_num_levels(void) { return g_or.nl; }
double or_strong_coupled(void) { return g_or.strong_coupled; }
void or_level_info(int l, int *out)
{
    out[0] = g_or.A[l].n; out[1] = g_or.A[l].nnz;
    out[2] = (l < g_or.nl - 1) ? g_or.nc[l] : 0;
}
void or_level_A(int l, int *ia, int *ja, double *val)
{
    ocsr *A = &g_or.A[l];
    memcpy(ia, A->ia, sizeof(int) * (A->n + 1));
    memcpy(ja, A->ja, sizeof(int) * A->nnz);
    memcpy(val, A->val, sizeof(double) * A->nnz);
}
void or_level_agg(int l, int *agg)
{
    memcpy(agg, g_or.agg[l], sizeof(int) * g_or.A[l].n);
}
void or_set_omega(const float *omega) { g_or.omega = omega; }

static int or_pcg_core(const ocsr *A, const double *b, double *u, int use_pc,
                       double tol, int maxit, int stop_type, double *hist,
                       int hist_cap, int *nhist);
static double or_dot(int n, const double *x, const double *y);
static double or_norm2(int n, const double *x);
static double or_norminf(int n, const double *x);
void or_precond(const double *r, double *z);

/* coarse_itsolver mgcycle.c:34-52: unpreconditioned CG to ctol, maxit 20n */
static void or_coarse_cg(const ocsr *A, const double *b, double *x, double ctol)
{
    or_pcg_core(A, b, x, 0, ctol, 20 * A->n, 1, NULL, 0, NULL);
}

/* mgcycle mgcycle.c:245-415 (V and W cycles; precond_amg passes tol=1e-6,
 * so the coarse CG runs to 1e-8) */
static void or_mgcycle_from(int l0)
{
    or_amg *G = &g_or;
    const int nl = G->nl;
    int num_lvl[OR_MAXLVL] = {0};
    int l = l0;
    double alpha = 1.0;
    const double ctol = 1e-6 * 1e-2;
forward:
    while (l < nl - 1) {
        ocsr *A = &G->A[l];
        num_lvl[l]++;
        or_smooth(G->smoother, 1, G->pre, G->relaxation, A->n, A->ia, A->ja,
                  A->val, G->b[l], G->x[l], l == 0 ? G->omega : NULL);
        memcpy(G->w[l], G->b[l], sizeof(double) * A->n);
        or_aAxpy(-1.0, A->n, A->ia, A->ja, A->val, G->x[l], G->w[l]);
        or_restrict(G->nc[l], G->ria[l], G->rja[l], G->w[l], G->b[l + 1]);
        ++l;
        memset(G->x[l], 0, sizeof(double) * G->A[l].n);
    }
    {
        ocsr *C = &G->A[nl - 1];
        if (G->coarse_solver == 32) or_chol_solve(C->n, G->Lc, G->b[nl - 1], G->x[nl - 1]);
        else or_coarse_cg(C, G->b[nl - 1], G->x[nl - 1], ctol);
    }
    while (l > l0) {
        --l;
        ocsr *A = &G->A[l];
        if (G->coarse_scaling == 1) {
            ocsr *Ac = &G->A[l + 1];
            double num = 0.0, den = 0.0;
            for (int i = 0; i < Ac->n; ++i) num += G->x[l + 1][i] * G->b[l + 1][i];
            /* dcsr_vmv sparse.c:1797-1815 */
            for (int i = 0; i < Ac->n; ++i) {
                double t = 0.0;
                for (int k = Ac->ia[i]; k < Ac->ia[i + 1]; ++k)
                    t += Ac->val[k] * G->x[l + 1][Ac->ja[k]];
                den += G->x[l + 1][i] * t;
            }
            alpha = num / den;
            if (alpha > 2.0) alpha = 2.0;
        }
        or_prolong(alpha, A->n, G->agg[l], G->x[l + 1], G->x[l]);
        or_smooth(G->smoother, 0, G->post, G->relaxation, A->n, A->ia, A->ja,
                  A->val, G->b[l], G->x[l], l == 0 ? G->omega : NULL);
        if (num_lvl[l] < G->cycle_type) break;
        else num_lvl[l] = 0;
    }
    if (l > l0) goto forward;
}

void or_mgcycle(void) { or_mgcycle_from(0); }

/* the cycle on the levels from l0 down (x_l0 = 0, b_l0 = b) */
void or_cycle_from(int l0, const double *b, double *x)
{
    int m = g_or.A[l0].n;
    memcpy(g_or.b[l0], b, sizeof(double) * m);
    memset(g_or.x[l0], 0, sizeof(double) * m);
    if (l0 == g_or.nl - 1) {
        ocsr *C = &g_or.A[l0];
        if (g_or.coarse_solver == 32) or_chol_solve(C->n, g_or.Lc, g_or.b[l0], g_or.x[l0]);
        else or_coarse_cg(C, g_or.b[l0], g_or.x[l0], 1e-8);
    } else {
        or_mgcycle_from(l0);
    }
    memcpy(x, g_or.x[l0], sizeof(double) * m);
}

/* the coarsest-level solve of the recursive cycles: the direct solver, or
 * coarse_itsolver to ctol */
static void or_coarse_solve(int l, double ctol)
{
    ocsr *C = &g_or.A[l];
    if (g_or.coarse_solver == 32) or_chol_solve(C->n, g_or.Lc, g_or.b[l], g_or.x[l]);
    else or_coarse_cg(C, g_or.b[l], g_or.x[l], ctol);
}

/* sum_i x_i (A x)_i, dcsr_vmv sparse.c:1797-1815 */
static double or_vmv(const ocsr *A, const double *x)
{
    double den = 0.0;
    for (int i = 0; i < A->n; ++i) {
        double t = 0.0;
        for (int k = A->ia[i]; k < A->ia[i + 1]; ++k) t += A->val[k] * x[A->ja[k]];
        den += x[i] * t;
    }
    return den;
}

/* amli mgcycle.c:430-555 from `level` with b, x of that level in place:
 * smoothing, residual, restriction, then degree + 1 recursive coarse cycles
 * combined by the polynomial's coefficients (b1 = A1 e1 + (c_{d-i}/c_d) r1),
 * e1 scaled by c_d, optional scaling alpha <= 2, prolongation, smoothing.
 * r1[l] keeps the restricted residual of level l. */
static double *g_r1[OR_MAXLVL];

static void or_amli(int level, const double *coef, int degree, double tol)
{
    or_amg *G = &g_or;
    ocsr *A0 = &G->A[level];
    if (level >= G->nl - 1) { or_coarse_solve(level, tol * 1e-4); return; }
    ocsr *A1 = &G->A[level + 1];
    const int m0 = A0->n, m1 = A1->n;
    double *b0 = G->b[level], *e0 = G->x[level], *r = G->w[level];
    double *b1 = G->b[level + 1], *e1 = G->x[level + 1];
    double *r1 = g_r1[level + 1];
    or_smooth(G->smoother, 1, G->pre, G->relaxation, m0, A0->ia, A0->ja, A0->val, b0, e0,
              level == 0 ? G->omega : NULL);
    memcpy(r, b0, sizeof(double) * m0);
    or_aAxpy(-1.0, m0, A0->ia, A0->ja, A0->val, e0, r);
    or_restrict(G->nc[level], G->ria[level], G->rja[level], r, b1);
    memcpy(r1, b1, sizeof(double) * m1);
    for (int i = 1; i <= degree; ++i) {
        memset(e1, 0, sizeof(double) * m1);
        or_amli(level + 1, coef, degree, tol);
        or_mxv(m1, A1->ia, A1->ja, A1->val, e1, b1);
        const double c = coef[degree - i] / coef[degree];   /* array_axpy array.c:357 */
        if (c == 1.0) for (int k = 0; k < m1; ++k) b1[k] += r1[k];
        else if (c == -1.0) for (int k = 0; k < m1; ++k) b1[k] -= r1[k];
        else for (int k = 0; k < m1; ++k) b1[k] += c * r1[k];
    }
    memset(e1, 0, sizeof(double) * m1);
    or_amli(level + 1, coef, degree, tol);
    for (int k = 0; k < m1; ++k) e1[k] *= coef[degree];   /* array_ax */
    double alpha = 1.0;
    if (G->coarse_scaling == 1) {
        alpha = or_dot(m1, e1, r1) / or_vmv(A1, e1);
        if (alpha > 2.0) alpha = 2.0;
    }
    or_prolong(alpha, m0, G->agg[level], e1, e0);
    or_smooth(G->smoother, 0, G->post, G->relaxation, m0, A0->ia, A0->ja, A0->val, b0, e0,
              level == 0 ? G->omega : NULL);
}

/* mgcycle_add mgcycle.c:700-820: the fine residual first (from x), then on
 * every level smoothing and restriction of the fine residual / the level's
 * b, the coarsest solve, and prolongations only (no post-smoothing) */
static void or_add_cycle(double tol)
{
    or_amg *G = &g_or;
    const int nl = G->nl;
    ocsr *A0 = &G->A[0];
    memcpy(G->w[0], G->b[0], sizeof(double) * A0->n);
    or_aAxpy(-1.0, A0->n, A0->ia, A0->ja, A0->val, G->x[0], G->w[0]);
    int l = 0;
    while (l < nl - 1) {
        ocsr *A = &G->A[l];
        or_smooth(G->smoother, 1, G->pre, G->relaxation, A->n, A->ia, A->ja, A->val,
                  G->b[l], G->x[l], l == 0 ? G->omega : NULL);
        or_restrict(G->nc[l], G->ria[l], G->rja[l], l == 0 ? G->w[0] : G->b[l], G->b[l + 1]);
        ++l;
        memset(G->x[l], 0, sizeof(double) * G->A[l].n);
    }
    or_coarse_solve(nl - 1, tol * 1e-2);
    while (l > 0) {
        --l;
        double alpha = 1.0;
        if (G->coarse_scaling == 1) {
            ocsr *Ac = &G->A[l + 1];
            alpha = or_dot(Ac->n, G->x[l + 1], G->b[l + 1]) / or_vmv(Ac, G->x[l + 1]);
            if (alpha > 2.0) alpha = 2.0;
        }
        or_prolong(alpha, G->A[l].n, G->agg[l], G->x[l + 1], G->x[l]);
    }
}

/* precond_amli / precond_amg_add precond.c:232-250, 336-355: maxit cycles
 * of the kind (3 AMLI, 5 additive) from x = 0 on b = r */
int or_precond_cycle(int kind, const double *coef, int degree, double tol, const double *r,
                     double *z)
{
    const int m = g_or.A[0].n;
    if (kind != 3 && kind != 5) return -1;
    for (int l = 1; l < g_or.nl; ++l)
        g_r1[l] = (double *)malloc(sizeof(double) * (g_or.A[l].n > 0 ? g_or.A[l].n : 1));
    memcpy(g_or.b[0], r, sizeof(double) * m);
    memset(g_or.x[0], 0, sizeof(double) * m);
    for (int i = 0; i < g_or.amg_maxit; ++i) {
        if (kind == 3) or_amli(0, coef, degree, tol);
        else or_add_cycle(tol);
    }
    memcpy(z, g_or.x[0], sizeof(double) * m);
    for (int l = 1; l < g_or.nl; ++l) { free(g_r1[l]); g_r1[l] = NULL; }
    return 0;
}

/* y' A x, dcsr_vmv sparse.c:1797-1815 */
static double or_vmv2(const ocsr *A, const double *x, const double *y)
{
    double value = 0.0;
    for (int i = 0; i < A->n; ++i) {
        double t = 0.0;
        for (int k = A->ia[i]; k < A->ia[i + 1]; ++k) t += A->val[k] * x[A->ja[k]];
        value += y[i] * t;
    }
    return value;
}

/* dcsr_pgcg krylov.c:2309-2420 with the preconditioner of the last setup's
 * cycle type (1 V/W, 3 AMLI with coef, 5 additive): a steepest-descent
 * step, then each new direction B r A-orthogonalised against all earlier
 * ones (beta_i = -(p_i' A Br) / (p_i' A p_i)); the relative residual is
 * ||r|| / ||b||, checked from the second step on.  hist: ||r|| handed to each
 * preconditioner call. */
typedef struct { int kind, degree; const double *coef; double amg_tol; } or_cycle_pc;

static void or_pc_cycle(const double *in, double *out, void *ctx)
{
    const or_cycle_pc *c = (const or_cycle_pc *)ctx;
    if (c->kind == 1) or_precond(in, out);
    else or_precond_cycle(c->kind, c->coef, c->degree, c->amg_tol, in, out);
}

static int or_gcg_on(const ocsr *A, or_pcfn pc, void *pcctx, const double *b, double *u,
                     double tol, int maxit, double *hist, int hist_cap, int *nhist);

int or_gcg(const double *b, double *u, double tol, int maxit, int kind, const double *coef,
           int degree, double amg_tol, double *hist, int hist_cap, int *nhist)
{
    or_cycle_pc c = {kind, degree, coef, amg_tol};
    return or_gcg_on(&g_or.A[0], or_pc_cycle, &c, b, u, tol, maxit, hist, hist_cap, nhist);
}

static int or_gcg_on(const ocsr *A, or_pcfn pc, void *pcctx, const double *b, double *u,
                     double tol, int maxit, double *hist, int hist_cap, int *nhist)
{
    const int m = A->n;
    int nh = 0, iter = 0;
    double *r = (double *)malloc(sizeof(double) * m);
    double *Br = (double *)malloc(sizeof(double) * m);
    double *p = (double *)malloc(sizeof(double) * (size_t)m * (maxit > 0 ? maxit : 1));
    double *beta = (double *)malloc(sizeof(double) * (maxit > 0 ? maxit : 1));
#define OR_GCG_PC(in, out)                                                      \
    do {                                                                         \
        if (hist && nh < hist_cap) hist[nh] = or_norm2(m, in);                  \
        ++nh;                                                                    \
        if (pc) pc(in, out, pcctx);                                              \
        else memcpy(out, in, sizeof(double) * m);                                \
    } while (0)
    const double normb = or_norm2(m, b);
    memcpy(r, b, sizeof(double) * m);
    or_aAxpy(-1.0, m, A->ia, A->ja, A->val, u, r);
    OR_GCG_PC(r, p);
    double alpha = or_dot(m, r, p) / or_vmv2(A, p, p);
    for (int i = 0; i < m; ++i) u[i] += alpha * p[i];
    or_aAxpy(-1.0 * alpha, m, A->ia, A->ja, A->val, p, r);
    double relres = or_norm2(m, r) / normb;
    for (iter = 1; iter < maxit; ++iter) {
        OR_GCG_PC(r, Br);
        double *pk = p + (size_t)iter * m;
        memcpy(pk, Br, sizeof(double) * m);
        for (int i = 0; i < iter; ++i) {
            const double *pi = p + (size_t)i * m;
            beta[i] = (-1.0) * (or_vmv2(A, Br, pi) / or_vmv2(A, pi, pi));
            for (int k = 0; k < m; ++k) pk[k] += beta[i] * pi[k];   /* array_axpy */
        }
        alpha = or_dot(m, r, pk) / or_vmv2(A, pk, pk);
        for (int k = 0; k < m; ++k) u[k] += alpha * pk[k];
        or_aAxpy(-1.0 * alpha, m, A->ia, A->ja, A->val, pk, r);
        relres = or_norm2(m, r) / normb;
        if (relres < tol) break;
    }
#undef OR_GCG_PC
    free(r); free(Br); free(p); free(beta);
    if (nhist) *nhist = nh;
    return iter > maxit ? -48 : iter;
}

/* array_axpy array.c:357-373: y += a x with a = +-1 as plain sums (x may be y) */
static void or_axpy(int n, double a, const double *x, double *y)
{
    if (a == 1.0) for (int i = 0; i < n; ++i) y[i] += x[i];
    else if (a == -1.0) for (int i = 0; i < n; ++i) y[i] -= x[i];
    else for (int i = 0; i < n; ++i) y[i] += a * x[i];
}

/* dcsr_pvgmres krylov.c:4612-4930 (flexible = 0) and dcsr_pvfgmres
 * krylov.c:5974-6280 (flexible = 1), right-preconditioned by the V/W cycle
 * of the last setup: restart cycles of modified Gram-Schmidt Arnoldi with
 * Givens rotations; the restart length shrinks by 3 (not below 3) while the
 * last cycle's convergence rate is in [0.174, 0.99], returns to `restart`
 * otherwise; a converged cycle is checked on the true residual and
 * restarted from it if that check fails.  hist: ||v|| of every vector handed
 * to the preconditioner. */
/* r = b - A x: CSR (dcsr_aAxpy(-1): the row sum subtracted) or, for the
 * scalar expansion of a block matrix, the products subtracted one by one
 * (dbsr_aAxpy(-1) negates, adds and negates back) */
static void or_resid_of(const ocsr *A, int block, const double *b, const double *x,
                        double *r)
{
    memcpy(r, b, sizeof(double) * A->n);
    if (!block) { or_aAxpy(-1.0, A->n, A->ia, A->ja, A->val, x, r); return; }
    for (int i = 0; i < A->n; ++i)
        for (int k = A->ia[i]; k < A->ia[i + 1]; ++k) r[i] -= A->val[k] * x[A->ja[k]];
}

static void or_pc_vcycle(const double *in, double *out, void *ctx)
{
    (void)ctx;
    or_precond(in, out);
}

static int or_gmres_on(int flexible, const ocsr *A, int block, or_pcfn pc, void *pcctx,
                       const double *b, double *x, double tol, int MaxIt, int restart,
                       int stop_type, double *hist, int hist_cap, int *nhist);

int or_gmres(int flexible, const double *b, double *x, double tol, int MaxIt, int restart,
             int stop_type, double *hist, int hist_cap, int *nhist)
{
    return or_gmres_on(flexible, &g_or.A[0], 0, or_pc_vcycle, NULL, b, x, tol, MaxIt, restart,
                       stop_type, hist, hist_cap, nhist);
}

static int or_gmres_on(int flexible, const ocsr *A, int block, or_pcfn pc, void *pcctx,
                       const double *b, double *x, double tol, int MaxIt, int restart,
                       int stop_type, double *hist, int hist_cap, int *nhist)
{
    const int n = A->n;
    const double cr_max = 0.99, cr_min = 0.174, epsmac = SMALLREAL;
    int nh = 0, iter = 0, i = 0, Restart = restart;
    const int R1 = restart + 1;
    double *r = (double *)calloc(n, sizeof(double));
    double *w = (double *)calloc(n, sizeof(double));
    double *rs = (double *)calloc(R1, sizeof(double));
    double *c = (double *)calloc(R1, sizeof(double));
    double *sn = (double *)calloc(R1, sizeof(double));
    double *pv = (double *)calloc((size_t)R1 * n, sizeof(double));
    double *zv = (double *)calloc((size_t)R1 * n, sizeof(double));
    double *hh = (double *)calloc((size_t)R1 * R1, sizeof(double));
#define P(k) (pv + (size_t)(k) * n)
#define Z(k) (zv + (size_t)(k) * n)
#define H(a, b_) hh[(size_t)(a) * R1 + (b_)]
#define OR_PC(in, out)                                                          \
    do {                                                                         \
        if (hist && nh < hist_cap) hist[nh] = or_norm2(n, in);                  \
        ++nh;                                                                    \
        if (pc) pc(in, out, pcctx);                                              \
        else memcpy(out, in, sizeof(double) * n);                                \
    } while (0)
    double cr = 1.0, r_norm_old = 0.0, r_norm, relres = BIGREAL, absres0 = BIGREAL;
    double absres, normu, den_norm = 1.0, epsilon = 0.0, b_norm = 0.0;
    or_resid_of(A, block, b, x, P(0));
    if (flexible) {
        b_norm = or_norm2(n, b);
        r_norm = or_norm2(n, P(0));
        den_norm = b_norm > 0.0 ? b_norm : r_norm;
        epsilon = tol * den_norm;
        if (r_norm < epsilon || r_norm < 1e-3 * tol) goto done;
    } else {
        r_norm = or_norm2(n, P(0));
        switch (stop_type) {
        case 1: absres0 = r_norm > SMALLREAL ? r_norm : SMALLREAL; relres = r_norm / absres0;
            break;
        case 2: {
            OR_PC(P(0), r);
            double rb = sqrt(or_dot(n, P(0), r));
            absres0 = rb > SMALLREAL ? rb : SMALLREAL;
            relres = rb / absres0;
            break;
        }
        default:
            normu = or_norm2(n, x);
            if (normu < SMALLREAL) normu = SMALLREAL;
            absres0 = r_norm;
            relres = absres0 / normu;
        }
        if (relres < tol || absres0 < 1e-3 * tol) goto done;
    }
    while (iter < MaxIt) {
        rs[0] = r_norm_old = r_norm;
        if (flexible && r_norm == 0.0) goto done;
        if (cr > cr_max || iter == 0) Restart = restart;
        else if (cr < cr_min) { /* keep */ }
        else Restart = (Restart - 3 > 3) ? Restart - 3 : restart;
        const double t0 = 1.0 / r_norm;
        for (int k = 0; k < n; ++k) P(0)[k] *= t0;
        i = 0;
        while (i < Restart && iter < MaxIt) {
            ++i; ++iter;
            double *zi = flexible ? Z(i - 1) : r;
            OR_PC(P(i - 1), zi);
            or_mxv(n, A->ia, A->ja, A->val, zi, P(i));
            for (int j = 0; j < i; ++j) {
                H(j, i - 1) = or_dot(n, P(j), P(i));
                or_axpy(n, -H(j, i - 1), P(j), P(i));
            }
            double t = or_norm2(n, P(i));
            H(i, i - 1) = t;
            if (t != 0.0) {
                t = 1.0 / t;
                for (int k = 0; k < n; ++k) P(i)[k] *= t;
            }
            for (int j = 1; j < i; ++j) {
                t = H(j - 1, i - 1);
                H(j - 1, i - 1) = sn[j - 1] * H(j, i - 1) + c[j - 1] * t;
                H(j, i - 1) = -sn[j - 1] * t + c[j - 1] * H(j, i - 1);
            }
            t = H(i, i - 1) * H(i, i - 1);
            t += H(i - 1, i - 1) * H(i - 1, i - 1);
            double gamma = sqrt(t);
            if (gamma == 0.0) gamma = epsmac;
            c[i - 1] = H(i - 1, i - 1) / gamma;
            sn[i - 1] = H(i, i - 1) / gamma;
            rs[i] = -sn[i - 1] * rs[i - 1];
            rs[i - 1] = c[i - 1] * rs[i - 1];
            H(i - 1, i - 1) = sn[i - 1] * H(i, i - 1) + c[i - 1] * H(i - 1, i - 1);
            if (flexible) {
                r_norm = fabs(rs[i]);
                if (r_norm <= epsilon) break;
            } else {
                absres = r_norm = fabs(rs[i]);
                relres = absres / absres0;
                if (relres < tol) break;
            }
        }
        rs[i - 1] = rs[i - 1] / H(i - 1, i - 1);
        for (int k = i - 2; k >= 0; --k) {
            double t = 0.0;
            for (int j = k + 1; j < i; ++j) t -= H(k, j) * rs[j];
            t += rs[k];
            rs[k] = t / H(k, k);
        }
        int conv;
        if (flexible) {
            memcpy(r, Z(i - 1), sizeof(double) * n);
            for (int k = 0; k < n; ++k) r[k] *= rs[i - 1];
            for (int j = i - 2; j >= 0; --j) or_axpy(n, rs[j], Z(j), r);
            or_axpy(n, 1.0, r, x);
            conv = r_norm <= epsilon;
        } else {
            memcpy(w, P(i - 1), sizeof(double) * n);
            for (int k = 0; k < n; ++k) w[k] *= rs[i - 1];
            for (int j = i - 2; j >= 0; --j) or_axpy(n, rs[j], P(j), w);
            OR_PC(w, r);
            or_axpy(n, 1.0, r, x);
            conv = relres < tol;
        }
        if (conv) {
            or_resid_of(A, block, b, x, r);
            r_norm = or_norm2(n, r);
            double dn = flexible ? den_norm : absres0;
            switch (stop_type) {
            case 1: relres = r_norm / dn; break;
            case 2: {
                double *dst = flexible ? P(0) : w;
                OR_PC(r, dst);
                relres = sqrt(or_dot(n, dst, r)) / dn;
                break;
            }
            default:
                normu = or_norm2(n, x);
                if (normu < SMALLREAL) normu = SMALLREAL;
                relres = r_norm / normu;
            }
            if (flexible ? relres <= tol : relres < tol) break;
            memcpy(P(0), r, sizeof(double) * n);
            i = 0;
        }
        for (int j = i; j > 0; --j) {
            rs[j - 1] = -sn[j - 1] * rs[j];
            rs[j] = c[j - 1] * rs[j];
        }
        if (i) or_axpy(n, rs[i] - 1.0, P(i), P(i));
        for (int j = i - 1; j > 0; --j) or_axpy(n, rs[j], P(j), P(i));
        if (i) {
            or_axpy(n, rs[0] - 1.0, P(0), P(0));
            or_axpy(n, 1.0, P(i), P(0));
        }
        cr = r_norm / r_norm_old;
    }
done:
#undef P
#undef Z
#undef H
#undef OR_PC
    free(r); free(w); free(rs); free(c); free(sn); free(pv); free(zv); free(hh);
    if (nhist) *nhist = nh;
    return iter >= MaxIt ? -48 : iter;
}

/* dcsr_pminres krylov.c:2449-2840: preconditioned MINRES by the three-term
 * recurrence of A-orthonormal directions p (with t = A p, z = B A p), with
 * the reference's checks: a zero solution (ERROR_SOLVER_SOLSTAG), stagnation
 * (restart from the true residual, at most 20 times, ERROR_SOLVER_STAG) and
 * false convergence (restart, at most 20 times, ERROR_SOLVER_TOLSMALL).
 * hist: ||v|| of every vector preconditioned. */
static int or_minres_on(const ocsr *A, or_pcfn pc, void *pcctx, const double *b, double *u,
                        double tol, int MaxIt, int stop_type, double *hist, int hist_cap,
                        int *nhist)
{
    const int m = A->n;
    const double maxdiff = tol * 1e-4;
    int iter = 0, stag = 1, more_step = 1, nh = 0;
    double absres0 = BIGREAL, absres = BIGREAL, normr0 = BIGREAL, relres = BIGREAL;
    double normu2 = 0.0, normp, alpha = 0.0;
    double *w = (double *)calloc((size_t)11 * m, sizeof(double));
    double *p0 = w, *p1 = w + m, *p2 = p1 + m, *z0 = p2 + m, *z1 = z0 + m;
    double *t0 = z1 + m, *t1 = t0 + m, *t = t1 + m, *tp = t + m, *tz = tp + m, *r = tz + m;
#define OR_M_PC(in, out)                                                        \
    do {                                                                         \
        if (hist && nh < hist_cap) hist[nh] = or_norm2(m, in);                  \
        ++nh;                                                                    \
        if (pc) pc(in, out, pcctx);                                              \
        else memcpy(out, in, sizeof(double) * m);                                \
    } while (0)
#define OR_M_MEASURE()                                                          \
    do {                                                                         \
        if (stop_type == 2) {                                                    \
            OR_M_PC(r, t);                                                       \
            absres = sqrt(fabs(or_dot(m, r, t)));                                \
            relres = absres / normr0;                                            \
        } else {                                                                 \
            absres = sqrt(or_dot(m, r, r));                                      \
            relres = absres / (stop_type == 3 ? normu2 : normr0);                \
        }                                                                        \
    } while (0)
#define OR_M_RESTART(use_abs)                                                   \
    do {                                                                         \
        memset(p0, 0, sizeof(double) * m);                                       \
        OR_M_PC(r, p1);                                                          \
        or_mxv(m, A->ia, A->ja, A->val, p1, tp);                                 \
        OR_M_PC(tp, tz);                                                         \
        normp = or_dot(m, tz, tp);                                               \
        normp = sqrt((use_abs) ? fabs(normp) : normp);                           \
        memcpy(t, p1, sizeof(double) * m);                                       \
        memset(t0, 0, sizeof(double) * m);                                       \
        memset(z0, 0, sizeof(double) * m);                                       \
        memset(t1, 0, sizeof(double) * m);                                       \
        memset(z1, 0, sizeof(double) * m);                                       \
        memset(p1, 0, sizeof(double) * m);                                       \
        or_axpy(m, 1 / normp, t, p1);                                            \
        or_axpy(m, 1 / normp, tp, t1);                                           \
        or_axpy(m, 1 / normp, tz, z1);                                           \
    } while (0)
    or_resid_of(A, 0, b, u, r);
    OR_M_PC(r, p1);
    if (stop_type == 2) {
        absres0 = sqrt(or_dot(m, r, p1));
        normr0 = absres0 > SMALLREAL ? absres0 : SMALLREAL;
        relres = absres0 / normr0;
    } else if (stop_type == 3) {
        absres0 = or_norm2(m, r);
        normu2 = or_norm2(m, u);
        if (normu2 < SMALLREAL) normu2 = SMALLREAL;
        relres = absres0 / normu2;
    } else {
        absres0 = or_norm2(m, r);
        normr0 = absres0 > SMALLREAL ? absres0 : SMALLREAL;
        relres = absres0 / normr0;
    }
    if (relres < tol || absres0 < 1e-3 * tol) goto done;
    or_mxv(m, A->ia, A->ja, A->val, p1, tp);
    OR_M_PC(tp, tz);
    normp = sqrt(fabs(or_dot(m, tz, tp)));
    memcpy(t, p1, sizeof(double) * m);
    memset(p1, 0, sizeof(double) * m);
    or_axpy(m, 1 / normp, t, p1);
    memset(t0, 0, sizeof(double) * m);
    memcpy(z0, t0, sizeof(double) * m);
    memcpy(t1, t0, sizeof(double) * m);
    memcpy(z1, t0, sizeof(double) * m);
    or_axpy(m, 1.0 / normp, tp, t1);
    or_axpy(m, 1.0 / normp, tz, z1);
    while (iter++ < MaxIt) {
        alpha = or_dot(m, r, z1);
        or_axpy(m, alpha, p1, u);
        or_axpy(m, -alpha, t1, r);
        or_mxv(m, A->ia, A->ja, A->val, z1, t);
        const double alpha1 = or_dot(m, z1, t);
        or_mxv(m, A->ia, A->ja, A->val, z0, t);
        const double alpha0 = or_dot(m, z1, t);
        memcpy(p2, z1, sizeof(double) * m);
        or_axpy(m, -alpha1, p1, p2);
        or_axpy(m, -alpha0, p0, p2);
        or_mxv(m, A->ia, A->ja, A->val, p2, tp);
        OR_M_PC(tp, tz);
        normp = sqrt(fabs(or_dot(m, tz, tp)));
        if (normp < 1e-14) { iter--; break; }
        memcpy(t, p2, sizeof(double) * m);
        memset(p2, 0, sizeof(double) * m);
        or_axpy(m, 1 / normp, t, p2);
        memcpy(p0, p1, sizeof(double) * m);
        memcpy(p1, p2, sizeof(double) * m);
        memcpy(t0, t1, sizeof(double) * m);
        memcpy(z0, z1, sizeof(double) * m);
        memset(t1, 0, sizeof(double) * m);
        memcpy(z1, t1, sizeof(double) * m);
        or_axpy(m, 1 / normp, tp, t1);
        or_axpy(m, 1 / normp, tz, z1);
        normu2 = or_norm2(m, u);
        OR_M_MEASURE();
        if (or_norminf(m, u) <= SMALLREAL) { iter = -43; break; }
        double normuu = or_norm2(m, p1);
        normuu = fabs(alpha) * (normuu / normu2);
        if (normuu < maxdiff) {
            or_resid_of(A, 0, b, u, r);
            OR_M_MEASURE();
            if (relres < tol) break;
            if (stag >= 20) { iter = -42; break; }
            ++stag;
            OR_M_RESTART(1);
        }
        if (relres < tol) {
            or_resid_of(A, 0, b, u, r);
            OR_M_MEASURE();
            if (relres < tol) break;
            if (more_step >= 20) { iter = -44; break; }
            ++more_step;
            OR_M_RESTART(0);
        }
        absres0 = absres;
    }
done:
#undef OR_M_PC
#undef OR_M_MEASURE
#undef OR_M_RESTART
    free(w);
    if (nhist) *nhist = nh;
    return iter > MaxIt ? -48 : iter;
}

int or_minres(const double *b, double *x, double tol, int maxit, int stop_type, int use_pc,
              double *hist, int hist_cap, int *nhist)
{
    return or_minres_on(&g_or.A[0], use_pc ? or_pc_vcycle : NULL, NULL, b, x, tol, maxit,
                        stop_type, hist, hist_cap, nhist);
}

/* nl_amli mgcycle.c:561-690 from absolute level a with nrem levels left
 * (the reference shifts mgl and counts levels from there): smoothing,
 * residual, restriction; below the second-coarsest level the coarse
 * correction is amli_degree + 1 steps of GCG (nl_amli_krylov_type 5) or
 * flexible GMRES(30) on the next level, to tol 1e-4 * amg tol, from zero,
 * preconditioned by precond_nl_amli there (one cycle); the second-coarsest
 * level calls the cycle once on the coarsest, which solves directly or by
 * coarse_itsolver to the same tolerance */
typedef struct { int a, nrem, degree, krylov; double tol; } or_nl_ctx;
static double *g_uH[OR_MAXLVL], *g_bH[OR_MAXLVL];

static void or_nl_amli(int a, int nrem, int degree, int krylov, double tol);

static void or_pc_nl_amli(const double *in, double *out, void *ctx)
{
    const or_nl_ctx *c = (const or_nl_ctx *)ctx;
    const int m = g_or.A[c->a].n;
    memcpy(g_or.b[c->a], in, sizeof(double) * m);
    memset(g_or.x[c->a], 0, sizeof(double) * m);
    or_nl_amli(c->a, c->nrem, c->degree, c->krylov, c->tol);
    memcpy(out, g_or.x[c->a], sizeof(double) * m);
}

static void or_nl_amli(int a, int nrem, int degree, int krylov, double tol)
{
    or_amg *G = &g_or;
    const double ktol = tol * 1e-4;
    if (!(0 < nrem - 1)) { or_coarse_solve(a, ktol); return; }
    ocsr *A0 = &G->A[a], *A1 = &G->A[a + 1];
    const int m0 = A0->n, m1 = A1->n;
    or_smooth(G->smoother, 1, G->pre, G->relaxation, m0, A0->ia, A0->ja, A0->val, G->b[a],
              G->x[a], a == 0 ? G->omega : NULL);
    memcpy(G->w[a], G->b[a], sizeof(double) * m0);
    or_aAxpy(-1.0, m0, A0->ia, A0->ja, A0->val, G->x[a], G->w[a]);
    or_restrict(G->nc[a], G->ria[a], G->rja[a], G->w[a], G->b[a + 1]);
    memset(G->x[a + 1], 0, sizeof(double) * m1);
    if (nrem - 2 == 0) {
        or_nl_amli(a + 1, nrem - 1, degree, krylov, tol);
    } else {
        double *bH = g_bH[a + 1], *uH = g_uH[a + 1];
        memcpy(bH, G->b[a + 1], sizeof(double) * m1);
        memcpy(uH, G->x[a + 1], sizeof(double) * m1);
        or_nl_ctx c = {a + 1, nrem - 1, degree, krylov, tol};
        if (krylov == 5)
            or_gcg_on(A1, or_pc_nl_amli, &c, bH, uH, ktol, degree + 1, NULL, 0, NULL);
        else
            or_gmres_on(1, A1, 0, or_pc_nl_amli, &c, bH, uH, ktol, degree + 1, 30, 1, NULL, 0,
                        NULL);
        memcpy(G->b[a + 1], bH, sizeof(double) * m1);
        memcpy(G->x[a + 1], uH, sizeof(double) * m1);
    }
    or_prolong(1.0, m0, G->agg[a], G->x[a + 1], G->x[a]);
    or_smooth(G->smoother, 0, G->post, G->relaxation, m0, A0->ia, A0->ja, A0->val, G->b[a],
              G->x[a], a == 0 ? G->omega : NULL);
}

/* precond_nl_amli precond.c:301-320: maxit cycles from x = 0 */
int or_precond_nl_amli(int degree, int krylov, double tol, const double *r, double *z)
{
    const int m = g_or.A[0].n;
    for (int l = 1; l < g_or.nl; ++l) {
        g_uH[l] = (double *)calloc(g_or.A[l].n > 0 ? g_or.A[l].n : 1, sizeof(double));
        g_bH[l] = (double *)calloc(g_or.A[l].n > 0 ? g_or.A[l].n : 1, sizeof(double));
    }
    memcpy(g_or.b[0], r, sizeof(double) * m);
    memset(g_or.x[0], 0, sizeof(double) * m);
    for (int i = 0; i < g_or.amg_maxit; ++i) or_nl_amli(0, g_or.nl, degree, krylov, tol);
    memcpy(z, g_or.x[0], sizeof(double) * m);
    for (int l = 1; l < g_or.nl; ++l) { free(g_uH[l]); free(g_bH[l]); g_uH[l] = g_bH[l] = NULL; }
    return 0;
}

int or_hier_level(int l, int *n, const int **ia, const int **ja, const double **a,
                  const int **agg, const int **ria, const int **rja, int *nc)
{
    if (l < 0 || l >= g_or.nl) return -1;
    *n = g_or.A[l].n; *ia = g_or.A[l].ia; *ja = g_or.A[l].ja; *a = g_or.A[l].val;
    *agg = g_or.agg[l]; *ria = g_or.ria[l]; *rja = g_or.rja[l]; *nc = g_or.nc[l];
    return 0;
}

/* precond_amg precond.c:164-184 */
void or_precond(const double *r, double *z)
{
    int m = g_or.A[0].n;
    memcpy(g_or.b[0], r, sizeof(double) * m);
    memset(g_or.x[0], 0, sizeof(double) * m);
    for (int i = 0; i < g_or.amg_maxit; ++i) or_mgcycle();
    memcpy(z, g_or.x[0], sizeof(double) * m);
}

/* array_norm2 / array_dotprod / array_norminf array.c:448-541 */
static double or_dot(int n, const double *x, const double *y)
{
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}
static double or_norm2(int n, const double *x) { return sqrt(or_dot(n, x, x)); }
static double or_norminf(int n, const double *x)
{
    double s = 0.0;
    for (int i = 0; i < n; ++i) { double v = fabs(x[i]); if (v > s) s = v; }
    return s;
}

/* residual measure for the three stopping types (krylov.c:157-170 etc.) */
static double or_resid(int stop_type, int n, const double *r, double *z,
                       int use_pc, double *absres)
{
    (void)z;
    if (stop_type == 2) {
        if (use_pc) or_precond(r, z); else memcpy(z, r, sizeof(double) * n);
        *absres = sqrt(fabs(or_dot(n, z, r)));
    } else {
        *absres = or_norm2(n, r);
    }
    return *absres;
}

/* dcsr_pcg krylov.c:122-398, including checks I-III and the restarts */
static int or_pcg_core(const ocsr *A, const double *b, double *u, int use_pc,
                       double tol, int maxit, int stop_type, double *hist,
                       int hist_cap, int *nhist)
{
    const int n = A->n;
    const double maxdiff = tol * 1e-4;
    int iter = 0, stag = 1, more_step = 1;
    double absres0 = BIGREAL, absres = BIGREAL, relres = BIGREAL;
    double normu = BIGREAL, normr0 = BIGREAL;
    double alpha, beta, temp1, temp2;
    int nh = 0;
    double *p = (double *)calloc(4 * (size_t)(n > 0 ? n : 1), sizeof(double));
    double *z = p + n, *r = z + n, *t = r + n;
#define PC_APPLY() do { \
        if (hist && nh < hist_cap) hist[nh] = or_norm2(n, r); \
        ++nh; \
        if (use_pc) or_precond(r, z); else memcpy(z, r, sizeof(double) * n); \
    } while (0)

    memcpy(r, b, sizeof(double) * n);
    or_aAxpy(-1.0, n, A->ia, A->ja, A->val, u, r);
    PC_APPLY();
    switch (stop_type) {
    case 1: absres0 = or_norm2(n, r); normr0 = absres0 > SMALLREAL ? absres0 : SMALLREAL;
        relres = absres0 / normr0; break;
    case 2: absres0 = sqrt(or_dot(n, r, z)); normr0 = absres0 > SMALLREAL ? absres0 : SMALLREAL;
        relres = absres0 / normr0; break;
    case 3: absres0 = or_norm2(n, r); normu = or_norm2(n, u);
        if (normu < SMALLREAL) normu = SMALLREAL;
        relres = absres0 / normu; break;
    default: goto done;
    }
    if (relres < tol || absres0 < 1e-3 * tol) goto done;
    memcpy(p, z, sizeof(double) * n);
    temp1 = or_dot(n, z, r);
    while (iter++ < maxit) {
        or_mxv(n, A->ia, A->ja, A->val, p, t);
        temp2 = or_dot(n, t, p);
        alpha = temp1 / temp2;
        for (int i = 0; i < n; ++i) u[i] += alpha * p[i];
        for (int i = 0; i < n; ++i) r[i] += (-alpha) * t[i];
        or_resid(stop_type, n, r, z, use_pc, &absres);
        relres = absres / (stop_type == 3 ? normu : normr0);
        if (or_norminf(n, u) <= SMALLREAL) { iter = -43; break; }
        normu = or_norm2(n, u);
        double reldiff = fabs(alpha) * or_norm2(n, p) / normu;
        if ((stag <= 20) & (reldiff < maxdiff)) {
            memcpy(r, b, sizeof(double) * n);
            or_aAxpy(-1.0, n, A->ia, A->ja, A->val, u, r);
            or_resid(stop_type, n, r, z, use_pc, &absres);
            relres = absres / (stop_type == 3 ? normu : normr0);
            if (relres < tol) break;
            if (stag >= 20) { iter = -42; break; }
            memset(p, 0, sizeof(double) * n);
            ++stag;
        }
        if (relres < tol) {
            memcpy(r, b, sizeof(double) * n);
            or_aAxpy(-1.0, n, A->ia, A->ja, A->val, u, r);
            or_resid(stop_type, n, r, z, use_pc, &absres);
            relres = absres / (stop_type == 3 ? normu : normr0);
            if (relres < tol) break;
            if (more_step >= 20) { iter = -44; break; }
            memset(p, 0, sizeof(double) * n);
            ++more_step;
        }
        absres0 = absres;
        if (stop_type != 2) PC_APPLY();
        temp2 = or_dot(n, z, r);
        beta = temp2 / temp1;
        temp1 = temp2;
        for (int i = 0; i < n; ++i) p[i] = 1.0 * z[i] + beta * p[i];
    }
done:
    free(p);
    if (nhist) *nhist = nh;
#undef PC_APPLY
    if (iter > maxit) return -48;
    return iter;
}

int or_pcg(const double *b, double *x, double tol, int maxit, int stop_type,
           double *hist, int hist_cap, int *nhist)
{
    return or_pcg_core(&g_or.A[0], b, x, 1, tol, maxit, stop_type, hist,
                       hist_cap, nhist);
}

/* ---- kernel-level wrappers for the parity tests ------------------------ */
int or_hem_agg(int n, const int *ia, const int *ja, const double *a,
               double theta, int *agg)
{
    int nnz = ia[n];
    int *nia = (int *)malloc(sizeof(int) * (n + 1));
    int *nja = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    double *nv = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    or_strength(n, ia, ja, a, theta, nia, nja, nv);
    int nc = or_hem(n, nia, nja, nv, agg);
    free(nia); free(nja); free(nv);
    return nc;
}

/* aggregation_vmb amg_setup_ua.c:596-736 on the strength graph (the three
 * greedy steps in the reference's orders, with its count of unvisited rows).
 * Returns the number of aggregates, 0 where the reference returns
 * ERROR_AMG_COARSEING (none after step 1); rows without an aggregate -> -1. */
static int or_vmb(int n, const int *ia, const int *ja, int max_agg, int *v)
{
    int na = 0, left = n;
    for (int i = 0; i < n; ++i) v[i] = -2;
    for (int i = n - 1; i >= 0; --i) {                       /* step 1 */
        if (ia[i + 1] - ia[i] == 1) { v[i] = -1; --left; continue; }
        int subset = 1;
        for (int p = ia[i]; p < ia[i + 1]; ++p)
            if (v[ja[p]] >= -1) { subset = 0; break; }
        if (!subset) continue;
        int count = 1;
        v[i] = na; --left;
        for (int p = ia[i]; p < ia[i + 1]; ++p)
            if (ja[p] != i && count < max_agg) { v[ja[p]] = na; --left; ++count; }
        ++na;
    }
    if (na < 1) return 0;
    int *t = (int *)malloc(sizeof(int) * n);
    int *cnt = (int *)calloc(na, sizeof(int));
    for (int i = 0; i < n; ++i) { t[i] = v[i]; if (v[i] >= 0) cnt[v[i]]++; }
    for (int i = n - 1; i >= 0; --i) {                       /* step 2 */
        if (v[i] >= -1) continue;
        for (int p = ia[i]; p < ia[i + 1]; ++p) {
            int a = t[ja[p]];
            if (a > -1 && cnt[a] < max_agg) { v[i] = a; --left; cnt[a]++; break; }
        }
    }
    while (left > 0) {                                        /* step 3 */
        int before = left;
        for (int i = 0; i < n; ++i) {
            if (v[i] >= -1) continue;
            int count = 1;
            v[i] = na; --left;
            for (int p = ia[i]; p < ia[i + 1]; ++p)
                if (ja[p] != i && v[ja[p]] < -1 && count < max_agg) {
                    v[ja[p]] = na; --left; ++count;
                }
            ++na;
        }
        if (left == before) break;   /* the reference would loop forever */
    }
    for (int i = 0; i < n; ++i) if (v[i] < 0) v[i] = -1;
    free(t); free(cnt);
    return na;
}

int or_vmb_agg(int n, const int *ia, const int *ja, const double *a,
               double theta, int max_agg, int *agg)
{
    int nnz = ia[n];
    int *nia = (int *)malloc(sizeof(int) * (n + 1));
    int *nja = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    double *nv = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    or_strength(n, ia, ja, a, theta, nia, nja, nv);
    int nc = or_vmb(n, nia, nja, max_agg, agg);
    free(nia); free(nja); free(nv);
    return nc;
}

/* The C library's rand() as the reference's HEC draws it (iarray_shuffle,
 * array.c:302-315).  glibc's rand() is random() of the TYPE_3 additive
 * feedback generator (published in glibc's random_r.c; the same since the
 * BSD random(3)): srand(s) fills r[0..30] by r[i] = 16807 r[i-1] mod
 * (2^31 - 1) from r[0] = s (s = 0 counts as 1), copies r[31..33] = r[0..2],
 * discards 310 outputs of r[i] = r[i-31] + r[i-3] (mod 2^32), and returns
 * r[i] >> 1.  A test checks this against the system's rand(). */
static struct { uint32_t r[34]; int i; } g_rand;

void or_srand(unsigned seed)
{
    int32_t r[34];
    r[0] = (int32_t)(seed ? seed : 1);
    for (int i = 1; i < 31; ++i) {
        long long w = (16807LL * r[i - 1]) % 2147483647LL;
        if (w < 0) w += 2147483647LL;
        r[i] = (int32_t)w;
    }
    for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
    for (int i = 0; i < 34; ++i) g_rand.r[i] = (uint32_t)r[i];
    g_rand.i = 34;
    for (int k = 0; k < 310; ++k) {
        uint32_t v = g_rand.r[(g_rand.i - 31) % 34] + g_rand.r[(g_rand.i - 3) % 34];
        g_rand.r[g_rand.i % 34] = v;
        ++g_rand.i;
    }
}

int or_rand(void)
{
    uint32_t v = g_rand.r[(g_rand.i - 31) % 34] + g_rand.r[(g_rand.i - 3) % 34];
    g_rand.r[g_rand.i % 34] = v;
    ++g_rand.i;
    if (g_rand.i >= 34 * 1024) g_rand.i -= 34 * 1000;   /* keep the index small */
    return (int)(v >> 1);
}

/* aggregation_hec amg_setup_ua.c:752-845 on the strength graph: rows in the
 * order of iarray_shuffle's permutation (drawn from the stream above, which
 * continues across calls as the process-wide rand() does); each row pairs
 * with its most strongly coupled neighbour (first maximum of |a| off the
 * diagonal) when that one is unvisited, else joins its aggregate.  Returns
 * the number of aggregates, -1 where the reference exits (a row of length > 1
 * with no off-diagonal entry). */
static int or_hec(int n, const int *ia, const int *ja, const double *a, int *v)
{
    int *perm = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) { perm[i] = i; v[i] = -2; }
    for (int i = 0; i < n - 1; ++i) {
        int j = i + or_rand() / (2147483647 / (n - i) + 1);
        int t = perm[j]; perm[j] = perm[i]; perm[i] = t;
    }
    int na = 0;
    for (int q = 0; q < n; ++q) {
        int i = perm[q];
        if (ia[i + 1] - ia[i] == 1) { v[i] = -1; continue; }
        int k = -1;
        double mx = -1.0;
        for (int p = ia[i]; p < ia[i + 1]; ++p)
            if (ja[p] != i && fabs(a[p]) > mx) { k = p; mx = fabs(a[p]); }
        if (k < 0) { free(perm); return -1; }
        int j = ja[k];
        if (v[j] < -1) { v[j] = na; v[i] = na; ++na; }
        else v[i] = v[j];
    }
    for (int i = 0; i < n; ++i) if (v[i] < 0) v[i] = -1;
    free(perm);
    return na;
}

int or_hec_agg(int n, const int *ia, const int *ja, const double *a, double theta,
               int *agg)
{
    int nnz = ia[n];
    int *nia = (int *)malloc(sizeof(int) * (n + 1));
    int *nja = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    double *nv = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    or_strength(n, ia, ja, a, theta, nia, nja, nv);
    int nc = or_hec(n, nia, nja, nv, agg);
    free(nia); free(nja); free(nv);
    return nc;
}

/* ---- UA-AMG setup for block (BSR) matrices --------------------------------
 * amg_setup_unsmoothP_unsmoothR_bsr (amg_setup_ua.c:2183-2425) without the
 * smoother data: per level while the level has more than max(coarse_dof, 50)
 * block rows and fewer than max_levels levels exist, the condensed matrix
 * (condenseBSRLinf, sparse.c:6223: each block's max row sum of |a|, negated
 * off the diagonal, entries <= 1e-8 dropped as dcsr_compress_inplace does),
 * HEM or VMB on its strength graph (no threshold adaptation on this path; an
 * aggregation failure stops coarsening), and the block Galerkin product
 * dbsr_rap (sparse.c:5840-5980) with identity blocks in P and R: coarse row C
 * reserves its diagonal block (0.0, accumulated), then blocks in first-
 * encounter order over (fine rows of R row C ascending) x (A row order); a new
 * block takes ddense_mul's sums, which start from 0.0 (so -0.0 becomes +0.0),
 * a known block adds them.  Blocks are nb x nb, row-major. */
typedef struct {
    int nrow, nnzb; int *ia, *ja, *agg; double *val;
    /* the cycle's data: scalar expansion, diagonal-block inverses, scalar
     * aggregate map and its R pattern, level vectors */
    ocsr E; double *dinv; int *sagg, *sria, *srja, snc; double *b, *x, *w, *t1, *t2;
} obsr;
static struct { int nl, nb; obsr lv[32]; } g_bsr;

static void or_bsr_free(void)
{
    for (int l = 0; l < 32; ++l) {
        obsr *L = &g_bsr.lv[l];
        free(L->ia); free(L->ja); free(L->val); free(L->agg);
        ocsr_free(&L->E);
        free(L->dinv); free(L->sagg); free(L->sria); free(L->srja);
        free(L->b); free(L->x); free(L->w); free(L->t1); free(L->t2);
    }
    memset(&g_bsr, 0, sizeof(g_bsr));
}

static double ddense_linf(const double *b, int nb)
{
    double norm = 0.0;
    for (int r = 0; r < nb; ++r) {
        double v = 0.0;
        for (int c = 0; c < nb; ++c) v = v + fabs(b[r * nb + c]);
        norm = norm > v ? norm : v;
    }
    return norm;
}

int or_bsr_setup(int nrow, int nnzb, int nb, const int *ia, const int *ja, const double *val,
                 double theta, int coarse_dof, int max_levels, int agg_type, int max_agg)
{
    or_bsr_free();
    const int nb2 = nb * nb;
    const int min_cdof = coarse_dof > 50 ? coarse_dof : 50;
    if (max_levels > 32) max_levels = 32;
    g_bsr.nb = nb;
    obsr *L = &g_bsr.lv[0];
    L->nrow = nrow; L->nnzb = nnzb;
    L->ia = (int *)malloc(sizeof(int) * (nrow + 1));
    L->ja = (int *)malloc(sizeof(int) * (nnzb > 0 ? nnzb : 1));
    L->val = (double *)malloc(sizeof(double) * (size_t)(nnzb > 0 ? nnzb : 1) * nb2);
    memcpy(L->ia, ia, sizeof(int) * (nrow + 1));
    memcpy(L->ja, ja, sizeof(int) * nnzb);
    memcpy(L->val, val, sizeof(double) * (size_t)nnzb * nb2);
    int lvl = 0;
    while (g_bsr.lv[lvl].nrow > min_cdof && lvl < max_levels - 1) {
        L = &g_bsr.lv[lvl];
        const int m = L->nrow;
        /* condensed matrix, compressed */
        int *pia = (int *)malloc(sizeof(int) * (m + 1));
        int *pja = (int *)malloc(sizeof(int) * (L->nnzb > 0 ? L->nnzb : 1));
        double *pv = (double *)malloc(sizeof(double) * (L->nnzb > 0 ? L->nnzb : 1));
        int q = 0;
        pia[0] = 0;
        for (int i = 0; i < m; ++i) {
            for (int k = L->ia[i]; k < L->ia[i + 1]; ++k) {
                double v = ddense_linf(L->val + (size_t)k * nb2, nb);
                if (L->ja[k] != i) v = -v;
                if (fabs(v) > 1e-8) { pja[q] = L->ja[k]; pv[q] = v; ++q; }
            }
            pia[i + 1] = q;
        }
        int *nia = (int *)malloc(sizeof(int) * (m + 1));
        int *nja = (int *)malloc(sizeof(int) * (q > 0 ? q : 1));
        double *nv = (double *)malloc(sizeof(double) * (q > 0 ? q : 1));
        or_strength(m, pia, pja, pv, theta, nia, nja, nv);
        L->agg = (int *)malloc(sizeof(int) * m);
        int nc = agg_type == 1 ? or_vmb(m, nia, nja, max_agg, L->agg)
                               : or_hem(m, nia, nja, nv, L->agg);
        free(pia); free(pja); free(pv); free(nia); free(nja); free(nv);
        if (nc < 1) { free(L->agg); L->agg = NULL; break; }
        /* R pattern (fine rows ascending) and the block Galerkin product */
        int *ria = (int *)malloc(sizeof(int) * (nc + 1));
        int *rja = (int *)malloc(sizeof(int) * m);
        or_trans_agg(m, nc, L->agg, ria, rja);
        int *slot = (int *)malloc(sizeof(int) * nc);
        for (int c = 0; c < nc; ++c) slot[c] = -1;
        int cap = 16 * nc + 16, cnnz = 0;
        int *cia = (int *)malloc(sizeof(int) * (nc + 1));
        int *cja = (int *)malloc(sizeof(int) * cap);
        double *cv = (double *)malloc(sizeof(double) * (size_t)cap * nb2);
        for (int C = 0; C < nc; ++C) {
            cia[C] = cnnz;
            const int base = cnnz;
#define OR_BSR_GROW()                                                              \
            if (cnnz >= cap) {                                                     \
                cap *= 2;                                                          \
                cja = (int *)realloc(cja, sizeof(int) * cap);                      \
                cv = (double *)realloc(cv, sizeof(double) * (size_t)cap * nb2);    \
            }
            OR_BSR_GROW();
            cja[cnnz] = C; slot[C] = cnnz;
            for (int t = 0; t < nb2; ++t) cv[(size_t)cnnz * nb2 + t] = 0.0;
            ++cnnz;
            for (int r1 = ria[C]; r1 < ria[C + 1]; ++r1) {
                const int I = rja[r1];
                for (int k = L->ia[I]; k < L->ia[I + 1]; ++k) {
                    const int D = L->agg[L->ja[k]];
                    if (D < 0) continue;
                    const double *src = L->val + (size_t)k * nb2;
                    if (slot[D] < base) {
                        OR_BSR_GROW();
                        slot[D] = cnnz; cja[cnnz] = D;
                        for (int t = 0; t < nb2; ++t)
                            cv[(size_t)cnnz * nb2 + t] = src[t] + 0.0;
                        ++cnnz;
                    } else {
                        for (int t = 0; t < nb2; ++t)
                            cv[(size_t)slot[D] * nb2 + t] += src[t] + 0.0;
                    }
                }
            }
#undef OR_BSR_GROW
        }
        cia[nc] = cnnz;
        free(ria); free(rja); free(slot);
        obsr *Cl = &g_bsr.lv[lvl + 1];
        Cl->nrow = nc; Cl->nnzb = cnnz; Cl->ia = cia; Cl->ja = cja; Cl->val = cv;
        ++lvl;
    }
    g_bsr.nl = lvl + 1;
    /* the cycle's data (dbsr_getdiaginv sparse.c:6122 on the smoothed levels:
     * the row's last diagonal block inverted by ddense_inv_inplace's
     * Gauss-Jordan, dense.c:1266; 1/a for nb = 1) */
    for (int l = 0; l < g_bsr.nl; ++l) {
        obsr *L = &g_bsr.lv[l];
        const int n = L->nrow * nb;
        ocsr *E = &L->E;
        E->n = E->m = n; E->nnz = L->nnzb * nb2;
        E->ia = (int *)malloc(sizeof(int) * (n + 1));
        E->ja = (int *)malloc(sizeof(int) * (E->nnz > 0 ? E->nnz : 1));
        E->val = (double *)malloc(sizeof(double) * (E->nnz > 0 ? E->nnz : 1));
        int q = 0;
        for (int I = 0; I < L->nrow; ++I)
            for (int r = 0; r < nb; ++r) {
                E->ia[I * nb + r] = q;
                for (int k = L->ia[I]; k < L->ia[I + 1]; ++k)
                    for (int c = 0; c < nb; ++c, ++q) {
                        E->ja[q] = L->ja[k] * nb + c;
                        E->val[q] = L->val[(size_t)k * nb2 + r * nb + c];
                    }
            }
        E->ia[n] = q;
        L->b = (double *)calloc(n, sizeof(double));
        L->x = (double *)calloc(n, sizeof(double));
        L->w = (double *)calloc(n, sizeof(double));
        L->t1 = (double *)calloc(n, sizeof(double));
        L->t2 = (double *)calloc(n, sizeof(double));
        if (l == g_bsr.nl - 1) continue;
        L->dinv = (double *)calloc((size_t)L->nrow * nb2, sizeof(double));
        for (int i = 0; i < L->nrow; ++i) {
            double *a = L->dinv + (size_t)i * nb2;
            for (int k = L->ia[i]; k < L->ia[i + 1]; ++k)
                if (L->ja[k] == i) memcpy(a, L->val + (size_t)k * nb2, sizeof(double) * nb2);
            if (nb == 1) { a[0] = 1.0 / a[0]; continue; }
            for (int k = 0; k < nb; ++k) {
                const int kn = k * nb, ll = kn + k;
                const double alinv = 1.0 / a[ll];
                a[ll] = alinv;
                for (int j = 0; j < k; ++j) a[kn + j] *= alinv;
                for (int j = k + 1; j < nb; ++j) a[kn + j] *= alinv;
                for (int r = 0; r < k; ++r)
                    for (int j = 0; j < nb; ++j) if (j != k) a[r * nb + j] -= a[r * nb + k] * a[kn + j];
                for (int r = k + 1; r < nb; ++r)
                    for (int j = 0; j < nb; ++j) if (j != k) a[r * nb + j] -= a[r * nb + k] * a[kn + j];
                for (int r = 0; r < k; ++r) a[r * nb + k] *= -alinv;
                for (int r = k + 1; r < nb; ++r) a[r * nb + k] *= -alinv;
            }
        }
        const int nc = g_bsr.lv[l + 1].nrow;
        L->snc = nc * nb;
        L->sagg = (int *)malloc(sizeof(int) * n);
        for (int i = 0; i < n; ++i) {
            const int a = L->agg[i / nb];
            L->sagg[i] = a < 0 ? -1 : a * nb + i % nb;
        }
        L->sria = (int *)malloc(sizeof(int) * (L->snc + 1));
        L->srja = (int *)malloc(sizeof(int) * n);
        or_trans_agg(n, L->snc, L->sagg, L->sria, L->srja);
    }
    return g_bsr.nl;
}

/* block relaxation of row i: x_i = D_i^{-1} (b_i - sum_{j != i} A_ij x_j)
 * (smoother_dbsr_gs_ascend / _descend, smoother.c:904-1040: ddense_ymAx per
 * block, ddense_mxv from 0.0; nb = 1: (b - sum) * diaginv) */
static void or_bsr_relax(const obsr *L, int nb, int i, const double *b, const double *xin,
                         double *xout, double *bt)
{
    const int nb2 = nb * nb;
    for (int r = 0; r < nb; ++r) bt[r] = b[i * nb + r];
    for (int k = L->ia[i]; k < L->ia[i + 1]; ++k) {
        const int j = L->ja[k];
        if (j == i) continue;
        const double *a = L->val + (size_t)k * nb2;
        for (int r = 0; r < nb; ++r)
            for (int c = 0; c < nb; ++c) bt[r] -= a[r * nb + c] * xin[j * nb + c];
    }
    const double *d = L->dinv + (size_t)i * nb2;
    if (nb == 1) { xout[i] = bt[0] * d[0]; return; }
    for (int r = 0; r < nb; ++r) {
        double t = 0.0;
        for (int c = 0; c < nb; ++c) t += d[r * nb + c] * bt[c];
        xout[i * nb + r] = t;
    }
}

/* smoother_dbsr_jacobi (all rows from the old iterate) and the Gauss-Seidel
 * sweeps (kind 1 ascending, 2 descending) */
static void or_bsr_sweep(obsr *L, int nb, int kind)
{
    double bt[64];
    if (kind == 0) {
        for (int i = 0; i < L->nrow; ++i) or_bsr_relax(L, nb, i, L->b, L->x, L->t1, bt);
        memcpy(L->x, L->t1, sizeof(double) * L->E.n);
    } else if (kind == 1) {
        for (int i = 0; i < L->nrow; ++i) or_bsr_relax(L, nb, i, L->b, L->x, L->x, bt);
    } else {
        for (int i = L->nrow - 1; i >= 0; --i) or_bsr_relax(L, nb, i, L->b, L->x, L->x, bt);
    }
}

static void or_bsr_smoothing(obsr *L, int nb, int smoother, int steps, int pre)
{
    for (int k = 0; k < steps; ++k) {
        if (smoother == 1) or_bsr_sweep(L, nb, 0);
        else if (smoother == 2) or_bsr_sweep(L, nb, pre ? 1 : 2);
        else { or_bsr_sweep(L, nb, 1); or_bsr_sweep(L, nb, 2); }
    }
}

/* mgcycle_bsr mgcycle.c:952-1160 as precond_dbsr_amg runs it
 * (precond.c:1311-1339): presmooth_iter sweeps before and after the coarse
 * correction, the coarsest level by GMRES(25) without preconditioner to
 * 1e-6 with at most min(n^2, 200) steps, the coarse scaling of its PeH / Aeh
 * form (alpha <= 1); maxit cycles from x = 0 */
int or_bsr_precond(int cycle_type, int smoother, int steps, int coarse_scaling, int maxit,
                   const double *r, double *z)
{
    const int nl = g_bsr.nl, nb = g_bsr.nb;
    if (nb > 8 || nl < 1) return -1;
    obsr *L0 = &g_bsr.lv[0];
    memcpy(L0->b, r, sizeof(double) * L0->E.n);
    memset(L0->x, 0, sizeof(double) * L0->E.n);
    for (int it = 0; it < maxit; ++it) {
        int nu[32] = {0};
        int l = 0;
forward:
        while (l < nl - 1) {
            obsr *L = &g_bsr.lv[l];
            nu[l]++;
            or_bsr_smoothing(L, nb, smoother, steps, 1);
            or_resid_of(&L->E, 1, L->b, L->x, L->w);
            or_restrict(L->snc, L->sria, L->srja, L->w, g_bsr.lv[l + 1].b);
            ++l;
            memset(g_bsr.lv[l].x, 0, sizeof(double) * g_bsr.lv[l].E.n);
        }
        {
            obsr *C = &g_bsr.lv[nl - 1];
            const long long cs = C->E.n;
            const int cmaxit = cs * cs < 200 ? (int)(cs * cs) : 200;
            or_gmres_on(0, &C->E, 1, NULL, NULL, C->b, C->x, 1e-6, cmaxit, 25, 1, NULL, 0,
                        NULL);
        }
        while (l > 0) {
            --l;
            obsr *L = &g_bsr.lv[l];
            obsr *Cn = &g_bsr.lv[l + 1];
            const int n = L->E.n;
            if (coarse_scaling == 1) {
                double *peh = L->t1, *aeh = L->t2;
                memset(peh, 0, sizeof(double) * n);
                or_prolong(1.0, n, L->sagg, Cn->x, peh);
                or_mxv(n, L->E.ia, L->E.ja, L->E.val, peh, aeh);
                double alpha = or_dot(n, aeh, L->w) / or_dot(n, aeh, aeh);
                if (alpha > 1.0) alpha = 1.0;
                or_axpy(n, alpha, peh, L->x);
            } else {
                or_prolong(1.0, n, L->sagg, Cn->x, L->x);
            }
            or_bsr_smoothing(L, nb, smoother, steps, 0);
            if (nu[l] < cycle_type) break;
            nu[l] = 0;
        }
        if (l > 0) goto forward;
    }
    memcpy(z, L0->x, sizeof(double) * L0->E.n);
    return 0;
}

/* out: nrow, nnzb of level l */
void or_bsr_level_info(int l, int *out)
{
    out[0] = g_bsr.lv[l].nrow;
    out[1] = g_bsr.lv[l].nnzb;
}

void or_bsr_level_A(int l, int *ia, int *ja, double *val)
{
    const obsr *L = &g_bsr.lv[l];
    memcpy(ia, L->ia, sizeof(int) * (L->nrow + 1));
    memcpy(ja, L->ja, sizeof(int) * L->nnzb);
    memcpy(val, L->val, sizeof(double) * (size_t)L->nnzb * g_bsr.nb * g_bsr.nb);
}

void or_bsr_level_agg(int l, int *agg)
{
    memcpy(agg, g_bsr.lv[l].agg, sizeof(int) * g_bsr.lv[l].nrow);
}

/* ---- smoothed aggregation: amg_setup_smoothP_smoothR ---------------------
 * (amg_setup_ua.c:1461-1700) -- the aggregates of the UA setup (same adaptive
 * threshold), P = S P_tent with S = I - omega D^{-1} N (smooth_aggregation_p,
 * :472-560: N the strength graph with its diagonal corrected by the dropped
 * row sum when smooth_filter is on, else A; D its first diagonal entries,
 * |d| < 1e-6 -> 1; S's diagonal 1 - omega n_ii / d_i, off-diagonal
 * (-omega) n_ij / d_i), dcsr_mxm (sparse.c:1832-1917: columns in first-
 * encounter order, each value summed from 0.0 in (S entry, P entry) order),
 * R = P^T (dcsr_trans, rows ascending), A_c = dcsr_rap (sparse.c:2401-2520:
 * diagonal slot first from 0.0, new columns in first-encounter order, values
 * (r a) p added in traversal order; a fine column seen before in the coarse
 * row only adds).  With the direct coarse solver the coarsest matrix is
 * replaced by its transpose (:1631-1640). */
static struct { int nl; ocsr A[32], P[32]; } g_sa;

static void or_sa_free(void)
{
    for (int l = 0; l < 32; ++l) { ocsr_free(&g_sa.A[l]); ocsr_free(&g_sa.P[l]); }
    g_sa.nl = 0;
}

/* dcsr_trans of an n x m CSR with values: rows of T list rows of A ascending */
static void or_trans_full(int n, int m, const int *ia, const int *ja, const double *v,
                          ocsr *T)
{
    const int nnz = ia[n];
    T->n = m; T->m = n; T->nnz = nnz;
    T->ia = (int *)calloc(m + 1, sizeof(int));
    T->ja = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    T->val = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    for (int k = 0; k < nnz; ++k) T->ia[ja[k] + 1]++;
    for (int c = 0; c < m; ++c) T->ia[c + 1] += T->ia[c];
    int *pos = (int *)malloc(sizeof(int) * (m > 0 ? m : 1));
    memcpy(pos, T->ia, sizeof(int) * m);
    for (int i = 0; i < n; ++i)
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            int q = pos[ja[k]]++;
            T->ja[q] = i; T->val[q] = v[k];
        }
    free(pos);
}

int or_sa_setup(int n, int nnz, const int *ia, const int *ja, const double *val,
                double theta, int coarse_dof, int max_levels, int agg_type, int max_agg,
                int filter, double omega, int csolver, double *theta_out)
{
    or_sa_free();
    if (max_levels > 32) max_levels = 32;
    const int min_cdof = coarse_dof > 1 ? coarse_dof : 1;
    ocsr *A0 = &g_sa.A[0];
    A0->n = A0->m = n; A0->nnz = nnz;
    A0->ia = (int *)malloc(sizeof(int) * (n + 1));
    A0->ja = (int *)malloc(sizeof(int) * nnz);
    A0->val = (double *)malloc(sizeof(double) * nnz);
    memcpy(A0->ia, ia, sizeof(int) * (n + 1));
    memcpy(A0->ja, ja, sizeof(int) * nnz);
    memcpy(A0->val, val, sizeof(double) * nnz);
    int lvl = 0;
    while (g_sa.A[lvl].n > min_cdof && lvl < max_levels - 1) {
        ocsr *A = &g_sa.A[lvl];
        const int m = A->n;
        int *nia = (int *)malloc(sizeof(int) * (m + 1));
        int *nja = (int *)malloc(sizeof(int) * (A->nnz > 0 ? A->nnz : 1));
        double *nv = (double *)malloc(sizeof(double) * (A->nnz > 0 ? A->nnz : 1));
        or_strength(m, A->ia, A->ja, A->val, theta, nia, nja, nv);
        int *agg = (int *)malloc(sizeof(int) * m);
        int nc = agg_type == 1 ? or_vmb(m, nia, nja, max_agg, agg)
                               : or_hem(m, nia, nja, nv, agg);
        if (nc * 4 > m) theta /= 2;
        else if (nc * 1.25 < m) theta *= 2;
        if (nc < 1) { free(nia); free(nja); free(nv); free(agg); break; }
        /* the smoother's matrix: the filtered strength graph, or A */
        const int *sia = A->ia, *sja = A->ja;
        const double *sv = A->val;
        if (filter) {
            for (int i = 0; i < m; ++i) {
                double rsa = 0.0, rsn = 0.0;
                for (int k = A->ia[i]; k < A->ia[i + 1]; ++k)
                    if (A->ja[k] != i) rsa += A->val[k];
                for (int k = nia[i]; k < nia[i + 1]; ++k)
                    if (nja[k] != i) rsn += nv[k];
                for (int k = nia[i]; k < nia[i + 1]; ++k)
                    if (nja[k] == i) nv[k] += rsa - rsn;
            }
            sia = nia; sja = nja; sv = nv;
        }
        double *d = (double *)malloc(sizeof(double) * m);
        or_getdiag(m, sia, sja, sv, d);
        for (int i = 0; i < m; ++i) if (fabs(d[i]) < 1e-6) d[i] = 1.0;
        const int snnz = sia[m];
        double *S = (double *)malloc(sizeof(double) * (snnz > 0 ? snnz : 1));
        for (int i = 0; i < m; ++i)
            for (int k = sia[i]; k < sia[i + 1]; ++k)
                S[k] = sja[k] == i ? 1 - omega * sv[k] / d[i] : -omega * sv[k] / d[i];
        /* P = S P_tent: a column per aggregate met, first encounter first */
        ocsr *P = &g_sa.P[lvl];
        P->n = m; P->m = nc;
        P->ia = (int *)malloc(sizeof(int) * (m + 1));
        int pcap = snnz > 0 ? snnz : 1, q = 0;
        P->ja = (int *)malloc(sizeof(int) * pcap);
        P->val = (double *)malloc(sizeof(double) * pcap);
        /* each column's sum gets its products in S-row order, as dcsr_mxm's
         * per-entry loop over the row gives them */
        int *cslot = (int *)malloc(sizeof(int) * nc);
        for (int c = 0; c < nc; ++c) cslot[c] = -1;
        for (int i = 0; i < m; ++i) {
            P->ia[i] = q;
            for (int k = sia[i]; k < sia[i + 1]; ++k) {
                const int c = agg[sja[k]];
                if (c < 0) continue;
                if (cslot[c] < P->ia[i]) { cslot[c] = q; P->ja[q] = c; P->val[q] = 0.0; ++q; }
                P->val[cslot[c]] += S[k] * 1.0;
            }
        }
        free(cslot);
        P->ia[m] = q; P->nnz = q;
        free(S); free(d); free(nia); free(nja); free(nv); free(agg);
        /* R = P^T, A_c = R A P */
        ocsr R;
        or_trans_full(m, nc, P->ia, P->ja, P->val, &R);
        ocsr *Ac = &g_sa.A[lvl + 1];
        int *ps = (int *)malloc(sizeof(int) * nc);
        int *as = (int *)malloc(sizeof(int) * m);
        for (int c = 0; c < nc; ++c) ps[c] = -1;
        for (int i = 0; i < m; ++i) as[i] = -1;
        int ccap = 64 + 8 * nc, cc = 0;
        Ac->n = Ac->m = nc;
        Ac->ia = (int *)malloc(sizeof(int) * (nc + 1));
        Ac->ja = (int *)malloc(sizeof(int) * ccap);
        Ac->val = (double *)malloc(sizeof(double) * ccap);
        for (int ic = 0; ic < nc; ++ic) {
            const int row0 = cc;
            Ac->ia[ic] = cc;
            if (cc >= ccap) {
                ccap *= 2;
                Ac->ja = (int *)realloc(Ac->ja, sizeof(int) * ccap);
                Ac->val = (double *)realloc(Ac->val, sizeof(double) * ccap);
            }
            ps[ic] = cc; Ac->ja[cc] = ic; Ac->val[cc] = 0.0; ++cc;
            for (int j1 = R.ia[ic]; j1 < R.ia[ic + 1]; ++j1) {
                const double re = R.val[j1];
                const int i1 = R.ja[j1];
                for (int j2 = A->ia[i1]; j2 < A->ia[i1 + 1]; ++j2) {
                    const double ra = re * A->val[j2];
                    const int i2 = A->ja[j2];
                    const int first = as[i2] != ic;
                    as[i2] = ic;
                    for (int j3 = P->ia[i2]; j3 < P->ia[i2 + 1]; ++j3) {
                        const double rap = ra * P->val[j3];
                        const int i3 = P->ja[j3];
                        if (first && ps[i3] < row0) {
                            if (cc >= ccap) {
                                ccap *= 2;
                                Ac->ja = (int *)realloc(Ac->ja, sizeof(int) * ccap);
                                Ac->val = (double *)realloc(Ac->val, sizeof(double) * ccap);
                            }
                            ps[i3] = cc; Ac->ja[cc] = i3; Ac->val[cc] = rap; ++cc;
                        } else {
                            Ac->val[ps[i3]] += rap;
                        }
                    }
                }
            }
        }
        Ac->ia[nc] = cc; Ac->nnz = cc;
        free(ps); free(as); ocsr_free(&R);
        ++lvl;
    }
    g_sa.nl = lvl + 1;
    if (csolver == 32) {
        ocsr *C = &g_sa.A[lvl], T;
        or_trans_full(C->n, C->n, C->ia, C->ja, C->val, &T);
        ocsr_free(C);
        *C = T;
    }
    if (theta_out) *theta_out = theta;
    return g_sa.nl;
}

/* out: rows, stored entries of A, and of P (0 on the coarsest level) */
void or_sa_level_info(int l, int *out)
{
    out[0] = g_sa.A[l].n; out[1] = g_sa.A[l].nnz;
    out[2] = l < g_sa.nl - 1 ? g_sa.P[l].nnz : 0;
}

void or_sa_level_A(int l, int *ia, int *ja, double *val)
{
    const ocsr *A = &g_sa.A[l];
    memcpy(ia, A->ia, sizeof(int) * (A->n + 1));
    memcpy(ja, A->ja, sizeof(int) * A->nnz);
    memcpy(val, A->val, sizeof(double) * A->nnz);
}

void or_sa_level_P(int l, int *ia, int *ja, double *val)
{
    const ocsr *P = &g_sa.P[l];
    memcpy(ia, P->ia, sizeof(int) * (P->n + 1));
    memcpy(ja, P->ja, sizeof(int) * P->nnz);
    memcpy(val, P->val, sizeof(double) * P->nnz);
}

static ocsr g_rap;
int or_rap(int n, const int *ia, const int *ja, const double *a, int nc,
           const int *agg, int *rap_ia, int *rap_ja, double *rap_val)
{
    if (!rap_ja) {
        int *ria = (int *)malloc(sizeof(int) * (nc + 1));
        int *rja = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
        or_trans_agg(n, nc, agg, ria, rja);
        ocsr_free(&g_rap);
        or_rap_agg(n, ia, ja, a, nc, agg, ria, rja, &g_rap);
        free(ria); free(rja);
        memcpy(rap_ia, g_rap.ia, sizeof(int) * (nc + 1));
        return g_rap.nnz;
    }
    memcpy(rap_ja, g_rap.ja, sizeof(int) * g_rap.nnz);
    memcpy(rap_val, g_rap.val, sizeof(double) * g_rap.nnz);
    return g_rap.nnz;
}
