/*
 * hazmath_b200.h -- C ABI of the B200-native UA-AMG preconditioned Krylov solve.
 *
 * The library (hazmath_b200/libhazb200.so) drops in for HAZmath's
 * unsmoothed-aggregation AMG + CG path.  The data structures below are
 * layout-compatible with HAZmath's own (include/sparse.h, include/vec.h,
 * include/param.h, include/solver.h of the reference), the constants keep
 * HAZmath's values (include/macro.h), and every entry point in section 3 keeps
 * the signature and the meaning of the reference function it replaces (cited
 * file:line within the HAZmath project).  All numeric work runs in CUDA
 * kernels on an sm_100a GPU; host pointers are accepted wherever the
 * reference takes them and are copied to and from device memory internally.
 *
 * Section 4 adds what the reference has no counterpart for: options for the
 * mixed-precision and learned-smoother forms, a persistent solver handle that
 * works on device-resident arrays, the batched solver and the kernel-level
 * entry points used by the parity tests.
 */
#ifndef HAZMATH_B200_H
#define HAZMATH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------
 * 1. Scalar types and constants (values as in the reference's include/macro.h)
 * ------------------------------------------------------------------------- */
#ifndef INT
#define INT   int
#endif
#ifndef SHORT
#define SHORT short
#endif
#ifndef REAL
#define REAL  double
#endif

#define SMALLREAL  1e-20
#define BIGREAL    1e+20
#define MAX_AMG_LVL 20
#define MIN_CDOF   1
#define STAG_RATIO 1e-4
#define MAX_STAG   20
#define MAX_RESTART 20

#define SUCCESS                 0
#define ERROR_INPUT_PAR       -13
#define ERROR_MAT_SIZE        -15
#define ERROR_MISC            -19
#define ERROR_ALLOC_MEM       -20
#define ERROR_DATA_STRUCTURE  -21
#define ERROR_DATA_ZERODIAG   -22
#define ERROR_AMG_SMOOTH_TYPE -31
#define ERROR_AMG_AGG_TYPE    -32
#define ERROR_AMG_COARSEING   -33
#define ERROR_SOLVER_TYPE     -40
#define ERROR_SOLVER_PRECTYPE -41
#define ERROR_SOLVER_STAG     -42
#define ERROR_SOLVER_SOLSTAG  -43
#define ERROR_SOLVER_TOLSMALL -44
#define ERROR_SOLVER_MISC     -47
#define ERROR_SOLVER_MAXIT    -48
#define ERROR_SOLVER_EXIT     -49
#define ERROR_UNKNOWN         -99

#define PRINT_NONE 0
#define PRINT_MIN  1
#define PRINT_SOME 2
#define PRINT_MORE 4

#define SOLVER_DEFAULT  0
#define SOLVER_CG       1
#define SOLVER_MinRes   2
#define SOLVER_VGMRES   3
#define SOLVER_VFGMRES  4
#define SOLVER_GCG      5
#define SOLVER_AMG     21
#define SOLVER_UMFPACK 32

#define STOP_REL_RES     1
#define STOP_REL_PRECRES 2
#define STOP_MOD_REL_RES 3

#define PREC_NULL 0
#define PREC_DIAG 1
#define PREC_AMG  2

#define UA_AMG 1
#define SA_AMG 2

#define VMB 1
#define HEC 4
#define HEM 5

#define V_CYCLE 1
#define W_CYCLE 2
#define AMLI_CYCLE 3
#define NL_AMLI_CYCLE 4
#define ADD_CYCLE 5

#define SMOOTHER_JACOBI  1
#define SMOOTHER_GS      2
#define SMOOTHER_SGS     3
#define SMOOTHER_SOR     5
#define SMOOTHER_SSOR    6
#define SMOOTHER_GSOR    7
#define SMOOTHER_SGSOR   8
#define SMOOTHER_L1DIAG 10

#define UNPT -1
#ifndef ON
#define ON  1
#define OFF 0
#endif

/* ---------------------------------------------------------------------------
 * 2. Data structures, layout-identical to the reference's
 * ------------------------------------------------------------------------- */

/* include/sparse.h:25-45 */
typedef struct dCSRmat {
    INT row;    /* rows m */
    INT col;    /* columns n */
    INT nnz;    /* stored entries */
    INT *IA;    /* row pointers, m+1, 0-based */
    INT *JA;    /* column indices, nnz */
    REAL *val;  /* values, nnz */
} dCSRmat;

/* include/sparse.h:185-213: block sparse row matrix; ROW x COL blocks of
 * nb x nb values, block k at val[k nb^2 ..], row-major inside the block
 * (storage_manner 0, the only manner this library takes) */
typedef struct dBSRmat {
    INT ROW;            /* block rows */
    INT COL;            /* block columns */
    INT NNZ;            /* stored blocks */
    INT nb;             /* block size */
    INT storage_manner; /* 0: row-wise inside each block */
    REAL *val;          /* NNZ nb^2 values */
    INT *IA;            /* block row pointers, ROW+1 */
    INT *JA;            /* block column indices, NNZ */
} dBSRmat;

/* include/vec.h:20-28 */
typedef struct dvector {
    INT row;
    REAL *val;
} dvector;

/* include/vec.h:34-42 */
typedef struct ivector {
    INT row;
    INT *val;
} ivector;

/* include/param.h:138-156 */
typedef struct {
    SHORT linear_itsolver_type;
    SHORT linear_precond_type;
    SHORT linear_stop_type;
    INT   linear_maxit;
    REAL  linear_tol;
    INT   linear_restart;
    SHORT linear_print_level;
    SHORT HX_smooth_iter;
    REAL  AL_scaling_param;
} linear_itsolver_param;

/* include/param.h:164-266 */
typedef struct {
    SHORT AMG_type;
    SHORT print_level;
    INT   maxit;
    REAL  tol;
    SHORT max_levels;
    INT   coarse_dof;
    SHORT cycle_type;
    SHORT smoother;
    SHORT presmooth_iter;
    SHORT postsmooth_iter;
    REAL  relaxation;
    SHORT polynomial_degree;
    SHORT coarse_solver;
    SHORT coarse_scaling;
    SHORT amli_degree;
    REAL *amli_coef;
    SHORT nl_amli_krylov_type;
    SHORT aggregation_type;
    REAL  strong_coupled;
    INT   max_aggregation;
    SHORT smooth_filter;
    REAL  tentative_smooth;
    INT   Schwarz_levels;
    INT   Schwarz_mmsize;
    INT   Schwarz_maxlvl;
    INT   Schwarz_type;
    INT   Schwarz_blksolver;
    char *HAZDIR;
    INT  *Schwarz_on_blk;
    INT  *Schwarz_patch_type;
    REAL  damping_param;
    REAL  BSR_alpha;
    REAL  BSR_omega;
    REAL  fpwr;
    void *smoother_function;
} AMG_param;

/* include/solver.h:25-36 */
typedef struct {
    void *data;
    void (*fct)(REAL *, REAL *, void *);
    REAL setup_time;
} precond;

/* include/solver.h:46-104; only carried inside AMG_data (Schwarz smoothing
 * is not part of this path, the fields keep the layout).                    */
typedef struct {
    dCSRmat A;
    INT nblk;
    INT *iblock;
    INT *jblock;
    dvector rhsloc1;
    dvector xloc1;
    SHORT Schwarz_type;
    INT blk_solver;
    INT memt;
    INT *mask;
    INT maxbs;
    INT maxbnnz;
    dCSRmat *blk_data;
    void **numeric;
    void *swzparam;
} Schwarz_data;

/* include/solver.h:110-164.  The B200 hierarchy hangs off mgl[0].wdata. */
typedef struct {
    SHORT max_levels;
    SHORT num_levels;
    dCSRmat A;
    dCSRmat R;
    dCSRmat P;
    dvector b;
    dvector x;
    dCSRmat M;
    void *Numeric;
    INT near_kernel_dim;
    REAL **near_kernel_basis;
    INT Schwarz_levels;
    Schwarz_data Schwarz;
    dvector w;
    INT cycle_type;
    void *wdata;
} AMG_data;

/* include/solver.h:472-559 */
typedef struct {
    SHORT AMG_type;
    SHORT print_level;
    INT   maxit;
    SHORT max_levels;
    REAL  tol;
    SHORT cycle_type;
    SHORT smoother;
    SHORT presmooth_iter;
    SHORT postsmooth_iter;
    REAL  relaxation;
    SHORT polynomial_degree;
    SHORT coarse_solver;
    SHORT coarse_scaling;
    SHORT amli_degree;
    SHORT nl_amli_krylov_type;
    REAL *amli_coef;
    AMG_data *mgl_data;
    REAL  fpwr;
    dCSRmat *A;
    dCSRmat *A_nk;
    dCSRmat *P_nk;
    dCSRmat *R_nk;
    dvector *r;
    REAL *w;
} precond_data;

/* ---------------------------------------------------------------------------
 * 3. Drop-in entry points (same names, arguments and return conventions as
 *    the reference).  Return >= 0: iteration count; < 0: an ERROR_* code.
 *    The library never calls exit(); a device failure returns
 *    ERROR_ALLOC_MEM (allocation) or ERROR_SOLVER_MISC (CUDA error).
 * ------------------------------------------------------------------------- */

/* src/solver/itsolver.c:846-931.  Copies A to the GPU, runs the UA setup,
 * builds the AMG preconditioner and calls the Krylov method selected by
 * itparam->linear_itsolver_type (1 = CG).  x: initial guess in, solution
 * out. */
INT linear_solver_dcsr_krylov_amg(dCSRmat *A, dvector *b, dvector *x,
                                  linear_itsolver_param *itparam,
                                  AMG_param *amgparam);

/* src/solver/itsolver.c:524-630: AMG as a stand-alone iterative solver
 * (amg_solve, src/solver/amg_solve.c:109). */
INT linear_solver_amg(dCSRmat *A, dvector *b, dvector *x, AMG_param *param);

/* src/solver/itsolver.c:2104-2200: UA-AMG preconditioned Krylov method for
 * a block (BSR) matrix.  Setup as amg_setup_ua_bsr (amg_setup_ua.c:145):
 * diagonal-block inverses, the L-infinity condensed matrix aggregated by
 * heavy edge matching (threshold fixed), boolean block P, A_c = R A P by
 * dbsr_rap; levels while more than max(coarse_dof, 50) block rows.
 * Preconditioner precond_dbsr_amg (precond.c:1311): maxit cycles of
 * mgcycle_bsr (block Jacobi / Gauss-Seidel / symmetric Gauss-Seidel,
 * presmooth_iter sweeps on both sides, coarsest level by GMRES(25) to
 * 1e-6).  Krylov types 1 (CG, prints the condition estimate), 3 (GMRES) and
 * 4 (flexible GMRES); any other type returns ERROR_SOLVER_TYPE.  Block
 * sizes 1 to 8.  x: initial guess in, solution out. */
INT linear_solver_dbsr_krylov_amg(dBSRmat *A, dvector *b, dvector *x,
                                  linear_itsolver_param *itparam,
                                  AMG_param *amgparam);

/* src/solver/itsolver.c:135-229: Krylov switch on a host preconditioner:
 * type 1 CG (prints the condition estimate), 2 MINRES (prints the
 * reference's " NOTHING IMPLEMENTED FOR MINRES" line), 3 variable-restart
 * GMRES, 4 flexible GMRES; any other type returns ERROR_SOLVER_TYPE. */
INT solver_dcsr_linear_itsolver(dCSRmat *A, dvector *b, dvector *x,
                                precond *pc, linear_itsolver_param *itparam);

/* src/solver/amg_setup_ua.c:53 (amg_setup_unsmoothP_unsmoothR :1228-1452).
 * mgl[0].A must hold the fine matrix.  Fills mgl[l].A/P/R (host copies) and
 * num_levels, mutates param->strong_coupled as the reference does, and keeps
 * the device hierarchy in mgl[0].wdata (released by amg_data_free). */
SHORT amg_setup_ua(AMG_data *mgl, AMG_param *param);

/* src/solver/amg_setup_ua.c:76 (-> amg_setup_smoothP_smoothR, :1461-1700):
 * smoothed aggregation: the aggregates of amg_setup_ua, P = S P_tent with the
 * damped-Jacobi smoother S of the filtered strength graph (tentative_smooth,
 * smooth_filter), R = P^T, A_c = R A P by the general Galerkin product; the
 * device hierarchy as for amg_setup_ua.  linear_solver_dcsr_krylov_amg and
 * linear_solver_amg take this path for AMG_type SA_AMG. */
SHORT amg_setup_sa(AMG_data *mgl, AMG_param *param);

/* src/solver/mgcycle.c:245-415: one V/W cycle on mgl[0].b, mgl[0].x. */
void mgcycle(AMG_data *mgl, AMG_param *param);

/* src/solver/precond.c:164-184: z = B r with host arrays r, z. */
void precond_amg(REAL *r, REAL *z, void *data);

/* src/solver/precond.c:232-250, 301-320, 336-355: z = B r with maxit AMLI,
 * nonlinear AMLI or additive cycles of the device hierarchy.  The
 * preconditioners linear_solver_dcsr_krylov_amg uses for cycle_type 3, 4
 * and 5; handed to dcsr_pcg / dcsr_pgcg / dcsr_pvgmres / dcsr_pvfgmres
 * with the setup's mgl_data, the whole Krylov loop runs on the device. */
void precond_amli(REAL *r, REAL *z, void *data);
void precond_nl_amli(REAL *r, REAL *z, void *data);
void precond_amg_add(REAL *r, REAL *z, void *data);

/* src/solver/mgcycle.c:430-555, 561-690, 700-820: one AMLI, nonlinear
 * AMLI or additive cycle on mgl[0].b, mgl[0].x.  The device hierarchy in
 * mgl[0] runs from its finest level: level must be 0 and num_levels the
 * hierarchy's level count. */
void amli(AMG_data *mgl, AMG_param *param, INT level);
void nl_amli(AMG_data *mgl, AMG_param *param, INT level, INT num_levels);
void mgcycle_add(AMG_data *mgl, AMG_param *param);

/* src/utilities/parameters.c:714-775: coefficients of the polynomial of
 * best uniform approximation of 1/x on [lambda_min, lambda_max] (degree + 1
 * values); amg_setup_ua stores them in param->amli_coef for AMLI_CYCLE with
 * lambda in [0.5, 2]. */
void amg_amli_coef(const REAL lambda_max, const REAL lambda_min, const INT degree,
                   REAL *coef);

/* src/solver/krylov.c:122-398.  pc == NULL: plain CG; pc->fct ==
 * precond_amg with a B200 hierarchy: the whole loop runs on the device;
 * any other pc->fct is called on host arrays every iteration. */
INT dcsr_pcg(dCSRmat *A, dvector *b, dvector *u, precond *pc,
             const REAL tol, const INT MaxIt, const SHORT stop_type,
             const SHORT prtlvl);

/* src/solver/krylov.c:4612-4930: right-preconditioned GMRES whose restart
 * length adapts to the convergence rate of each cycle (Baker, Jessup and
 * Kolev).  Preconditioner handling as dcsr_pcg; MaxIt reached (iter >=
 * MaxIt) returns ERROR_SOLVER_MAXIT. */
INT dcsr_pvgmres(dCSRmat *A, dvector *b, dvector *x, precond *pc,
                 const REAL tol, const INT MaxIt, const SHORT restart,
                 const SHORT stop_type, const SHORT prtlvl);

/* src/solver/krylov.c:5974-6250: the flexible form (every preconditioned
 * vector kept, stopping on ||r|| <= tol ||b||); Krylov type 4, the
 * reference's default with restart 100. */
INT dcsr_pvfgmres(dCSRmat *A, dvector *b, dvector *x, precond *pc,
                  const REAL tol, const INT MaxIt, const SHORT restart,
                  const SHORT stop_type, const SHORT prtlvl);

/* src/solver/krylov.c:2449-2840: preconditioned MINRES (three-term
 * recurrence, B-normalised directions, the CG's three safety checks);
 * Krylov type 2. */
INT dcsr_pminres(dCSRmat *A, dvector *b, dvector *u, precond *pc, const REAL tol,
                 const INT MaxIt, const SHORT stop_type, const SHORT prtlvl);

/* src/solver/krylov.c:2309-2420: generalized conjugate gradient (every
 * direction kept and A-orthogonalised, no restart), stopping on
 * ||r|| < tol ||b||; the coarse-level solver of the nonlinear AMLI cycle
 * when nl_amli_krylov_type is SOLVER_GCG. */
INT dcsr_pgcg(dCSRmat *A, dvector *b, dvector *u, precond *pc, const REAL tol,
              const INT MaxIt, const SHORT stop_type, const SHORT prtlvl);

/* src/utilities/wrapper.c:36-99.  The reference reads ./input.dat; this one
 * uses the UA-AMG defaults of the HAZmath examples (V-cycle, GS 1/1, HEM,
 * coarse direct solve) unless ./input.dat exists, in which case the AMG and
 * solver keys of that file are honoured. */
void python_wrapper_krylov_amg(INT *n, INT *nnz, INT *ia, INT *ja, REAL *a,
                               REAL *b, REAL *u, REAL *tol, INT *maxit,
                               INT *print_lvl);

/* src/utilities/data.c:66-91, :96-140, :22-55 */
AMG_data *amg_data_create(SHORT max_levels);
void amg_data_free(AMG_data *mgl, AMG_param *param);
void precond_data_null(precond_data *pcdata);

/* src/utilities/parameters.c:158-205, :238-250, :604-640, :649-680 */
void param_amg_init(AMG_param *amgparam);
void param_linear_solver_init(linear_itsolver_param *itsparam);
void param_amg_to_prec(precond_data *pcdata, AMG_param *amgparam);
void param_prec_to_amg(AMG_param *amgparam, precond_data *pcdata);

/* ---------------------------------------------------------------------------
 * 4. B200 extensions (no counterpart in the reference)
 * ------------------------------------------------------------------------- */

/* precision of the V-cycle */
#define HZB_PREC_FP64  0   /* the drop-in: everything in FP64, reference order */
#define HZB_PREC_MIXED 1   /* FP32 V-cycle, FP64 flexible CG outer loop       */

/* Gauss-Seidel schedule */
#define HZB_GS_EXACT      0 /* lexicographic, level-scheduled: bit-exact      */
#define HZB_GS_MULTICOLOR 1 /* multicolour ordering: parallel, not bit-exact  */

/* heavy edge matching */
#define HZB_MATCH_EXACT    0 /* the reference's sequential visiting order     */
#define HZB_MATCH_PARALLEL 1 /* deterministic parallel rounds: not bit-exact  */

typedef struct {
    SHORT precision;      /* HZB_PREC_*                                        */
    SHORT gs_schedule;    /* HZB_GS_*                                          */
    SHORT matching;       /* HZB_MATCH_*                                       */
    SHORT export_hierarchy;/* amg_setup_ua: copy levels back into mgl[l]      */
    SHORT use_omega;      /* 1: fine-level l1-Jacobi uses per-row weights      */
    const float *omega;   /* host array (n) of weights in (0,2), or NULL       */
    INT   device;         /* CUDA device ordinal                               */
    SHORT fallback_check; /* 1: measure the learned cycle's contraction and    */
                          /*    drop omega if it is worse than plain weights   */
    SHORT use_graph;      /* 1: replay the V-cycle from a captured CUDA graph  */
    SHORT reserved[6];
} hzb_param;

void hzb_param_init(hzb_param *p);

/* The drop-in with explicit B200 options (linear_solver_dcsr_krylov_amg is
 * this call with hzb_param_init defaults). */
INT hzb_solver_dcsr_krylov_amg(dCSRmat *A, dvector *b, dvector *x,
                               linear_itsolver_param *itparam,
                               AMG_param *amgparam, const hzb_param *bp);

/* Persistent handle on device-resident data. */
typedef struct hzb_solver hzb_solver;

typedef struct {
    INT   num_levels;
    INT   rows[MAX_AMG_LVL];
    INT   nnz[MAX_AMG_LVL];
    INT   iterations;
    REAL  final_relres;
    REAL  setup_seconds;   /* device time of the last setup                  */
    REAL  solve_seconds;   /* device time of the last solve                  */
    REAL  strong_coupled;  /* threshold after the adaptive updates          */
    REAL  condest;         /* CG condition estimate (0 if not computed)      */
    REAL  omega_contraction[2]; /* measured contraction: plain, learned     */
    INT   omega_used;      /* 1 if learned weights were kept                 */
    INT   launches;        /* kernels launched by the last solve             */
} hzb_stats;

INT  hzb_create(hzb_solver **s, const AMG_param *amg,
                const linear_itsolver_param *it, const hzb_param *bp);
/* setup from device arrays (int32 CSR, FP64 values) */
INT  hzb_setup_device(hzb_solver *s, INT n, INT nnz, const INT *d_ia,
                      const INT *d_ja, const REAL *d_val);
/* setup from a host matrix (copied in) */
INT  hzb_setup_host(hzb_solver *s, const dCSRmat *A);
/* solve with device vectors; x holds the initial guess */
INT  hzb_solve_device(hzb_solver *s, const REAL *d_b, REAL *d_x);
/* solve with host vectors (H2D/D2H copies included) */
INT  hzb_solve_host(hzb_solver *s, const REAL *b, REAL *x);
/* one preconditioner application z = B r on device vectors */
INT  hzb_precond_device(hzb_solver *s, const REAL *d_r, REAL *d_z);
/* Batched independent systems (no counterpart in the reference, whose
 * solvers take one system per call).  The device CSR (n rows, nnz entries)
 * holds nsys SPD systems on its diagonal blocks: rows and columns of system
 * k are [off[k], off[k+1]) (host array, off[0] = 0, off[nsys] = n); an entry
 * outside its row's block is rejected (ERROR_INPUT_PAR).  One hierarchy is
 * built on the union -- aggregates never cross systems, so each system's
 * block of every level is a hierarchy of that system -- and one V-cycle
 * pass serves all systems.  The handle's hzb_param.precision picks the
 * cycle (HZB_PREC_MIXED: FP32).                                            */
INT  hzb_batch_setup_device(hzb_solver *s, INT nsys, const INT *off, INT n, INT nnz,
                            const INT *d_ia, const INT *d_ja, const REAL *d_val);
/* Flexible CG per system to the handle's linear_tol (relative residual,
 * the true FP64 residual checked before a system is retired) and
 * linear_maxit.  Per system (host arrays of nsys, any may be NULL): the
 * iterations (ERROR_SOLVER_MAXIT if not converged), the final relative
 * residual, and the device time in seconds from the solve's start until the
 * system converged.  Returns the largest iteration count, or
 * ERROR_SOLVER_MAXIT if a system did not converge.                        */
INT  hzb_batch_solve_device(hzb_solver *s, const REAL *d_b, REAL *d_x, INT *iters,
                            REAL *relres, REAL *seconds);
/* per-row l1-Jacobi weights for the fine level (device array, n) */
INT  hzb_set_omega_device(hzb_solver *s, const float *d_omega);
INT  hzb_get_stats(const hzb_solver *s, hzb_stats *st);
/* level l of the device hierarchy copied to host arrays sized from stats;
 * agg (rows of level l) is the aggregate map, -1 for an empty row of P.   */
/* the smoothed prolongation P of level l (n_l x n_{l+1}, CSR with values)
 * into host arrays; *nnz receives its entry count (0 for an unsmoothed level,
 * whose P is the aggregate map of hzb_level_copy) */
INT  hzb_level_prolongation(const hzb_solver *s, INT l, INT *ia, INT *ja, REAL *val,
                            INT *nnz);
INT  hzb_level_copy(const hzb_solver *s, INT l, INT *ia, INT *ja, REAL *val,
                    INT *agg);
/* Block (BSR) hierarchy on the handle (the pieces of
 * linear_solver_dbsr_krylov_amg): amg_setup_ua_bsr of a host matrix with the
 * handle's AMG_param; level l's block matrix (ROW, NNZ and nb always; the
 * arrays copied where out->IA / JA / val are given) and its block aggregates
 * (agg, ROW entries, levels below the coarsest); precond_dbsr_amg on device
 * or host vectors; the handle's Krylov type (1, 3, 4) preconditioned by it,
 * x holding the initial guess. */
INT  hzb_bsr_setup_host(hzb_solver *s, const dBSRmat *A);
/* the same from device arrays (row pointers, block columns, blocks) */
INT  hzb_bsr_setup_device(hzb_solver *s, INT nrow, INT nnzb, INT nb, const INT *d_ia,
                          const INT *d_ja, const REAL *d_val);
INT  hzb_bsr_level(const hzb_solver *s, INT l, dBSRmat *out, INT *agg);
INT  hzb_bsr_precond_device(hzb_solver *s, const REAL *d_r, REAL *d_z);
INT  hzb_bsr_precond_host(hzb_solver *s, const REAL *r, REAL *z);
INT  hzb_bsr_solve_device(hzb_solver *s, const REAL *d_b, REAL *d_x);
INT  hzb_bsr_solve_host(hzb_solver *s, const REAL *b, REAL *x);
void hzb_destroy(hzb_solver *s);
/* last CUDA error message of this thread ("" if none) */
const char *hzb_last_error(void);

/* Learned l1-Jacobi weights (no counterpart in the reference).
 * A 3-layer message-passing network over the fine-level matrix graph (width
 * 32, BF16 weights, FP32 accumulation; tensor-core dense layers) maps
 * scale-invariant node/edge features of A to omega_i in (0,2).  An untrained
 * network returns omega = 1 (the reference's l1-Jacobi).  Training uses the
 * method's own error vectors and the two-cycle A-norm contraction as loss. */
typedef struct hzb_gnn hzb_gnn;
INT  hzb_gnn_num_params(void);
INT  hzb_gnn_create(hzb_gnn **g, unsigned long long seed, INT device);
void hzb_gnn_destroy(hzb_gnn *g);
INT  hzb_gnn_get_params(const hzb_gnn *g, float *host);   /* FP32 master copy */
INT  hzb_gnn_set_params(hzb_gnn *g, const float *host);
INT  hzb_gnn_get_grads(const hzb_gnn *g, float *host);
INT  hzb_gnn_zero_grad(hzb_gnn *g);
INT  hzb_gnn_adam_step(hzb_gnn *g, REAL lr);
/* omega (device array, n) for level 0 of the solver's hierarchy; keeps the
 * activations for hzb_gnn_backward */
INT  hzb_gnn_infer(hzb_gnn *g, hzb_solver *s, float *d_omega);
/* accumulate parameter gradients for dL/domega (device array, n) */
INT  hzb_gnn_backward(hzb_gnn *g, hzb_solver *s, const float *d_domega);
/* ns training error vectors (device, n x ns, FP64): seeded random vectors
 * after three plain l1 sweeps and ncycles (0..16) V-cycles, unit A-norm; the
 * cycles use the fine-level weights d_omega (device, n) or plain weights if
 * NULL.  ncycles = 0 gives vectors that do not depend on omega.            */
INT  hzb_learn_errors(hzb_solver *s, INT ns, unsigned long long seed, REAL *d_E,
                      const float *d_omega, INT ncycles);
/* mean over the ns vectors of ||E(omega)^k e||_A^2 / ||e||_A^2, k = ncycles
 * (1..16), for the V(2,2) l1-Jacobi cycle with fine-level weights omega, and
 * its gradient (adjoint cycles; d_domega NULL: the loss alone).  Training minimises the two-cycle
 * contraction of the errors the current cycle leaves, (||E^4 z||/||E^2 z||)^2
 * for omega-independent z, through the k = 4 and k = 2 gradients.          */
INT  hzb_learn_loss_grad(hzb_solver *s, const float *d_omega, INT ns,
                         const REAL *d_E, INT ncycles, REAL *loss, float *d_domega);
/* Set up the learned weights on a solver with fallback: infer omega, measure
 * the per-cycle contraction of the solve's own cycle (the FP32 cycle in
 * mixed precision) with and without it on ns method-generated error vectors
 * (the errors two cycles leave), keep omega only if it contracts better.
 * Both contractions are returned and recorded in hzb_stats
 * (omega_contraction, omega_used).                                          */
INT  hzb_learn_select_omega(hzb_solver *s, hzb_gnn *g, INT ns,
                            unsigned long long seed, REAL *rho_plain,
                            REAL *rho_learned);

/* Time `reps` back-to-back launches of one cycle kernel on level `level` of
 * the handle's hierarchy, on the handle's stream with CUDA events, after a
 * warm-up launch.  Returns the mean device time per launch and the
 * algorithmic bytes one launch must move (FP64 value 8 B or FP32 4 B + int32
 * index per entry, row pointers, and each vector once).  which:
 *   HZB_K_SPMV64  y = A x, FP64        HZB_K_SPMV32  y = A x, FP32
 *   HZB_K_RES64   w = b - A x, FP64    HZB_K_L1_32   l1-Jacobi sweep, FP32
 *   HZB_K_L1_64   l1-Jacobi sweep, FP64  HZB_K_GS64    forward Gauss-Seidel sweep
 *                                        on the level's schedule; needs a
 *                                        setup with a Gauss-Seidel smoother
 *                                        (ERROR_INPUT_PAR otherwise)
 * HZB_K_L1_32 on level 0 runs with the learned weights (and counts their
 * 4 bytes per row) when the handle's solve uses them.
 * The byte counts are single-pass lower bounds: the exact Gauss-Seidel
 * schedule's level sets and the multicolour schedule's colours re-read x,
 * which the count leaves out.
 * and on a block (BSR) hierarchy of the handle:
 *   HZB_K_BSR_RES  w = b - A x         HZB_K_BSR_JAC  block Jacobi sweep
 *   HZB_K_BSR_GS   ascending block Gauss-Seidel sweep (all level sets)     */
#define HZB_K_SPMV64 0
#define HZB_K_SPMV32 1
#define HZB_K_RES64  2
#define HZB_K_L1_32  3
#define HZB_K_L1_64  4
#define HZB_K_BSR_RES 5
#define HZB_K_BSR_JAC 6
#define HZB_K_BSR_GS  7
#define HZB_K_GS64    8
INT hzb_time_kernel(hzb_solver *s, INT which, INT level, INT reps,
                    REAL *ms_per_launch, REAL *bytes_per_launch);

/* Kernel-level entry points on device arrays, one stream-ordered launch
 * sequence each, used by the parity tests.  Each returns SUCCESS or
 * ERROR_SOLVER_MISC and synchronises before returning. */
INT hzb_dcsr_mxv_device(INT n, INT nnz, const INT *ia, const INT *ja,
                        const REAL *val, const REAL *x, REAL *y);
INT hzb_dcsr_aAxpy_device(REAL alpha, INT n, INT nnz, const INT *ia,
                          const INT *ja, const REAL *val, const REAL *x,
                          REAL *y);
/* smoother as called by mgcycle's pre (forward=1) or post (forward=0)
 * smoothing, SMOOTHER_* types JACOBI, GS, SGS, SOR, L1DIAG */
INT hzb_smoother_device(SHORT smoother, SHORT forward, INT sweeps, REAL relax,
                        INT n, INT nnz, const INT *ia, const INT *ja,
                        const REAL *val, const REAL *b, REAL *x);
/* strength graph + heavy edge matching: agg (n) and the aggregate count */
INT hzb_aggregation_hem_device(INT n, INT nnz, const INT *ia, const INT *ja,
                               const REAL *val, REAL strong_coupled,
                               INT *agg, INT *num_aggregates);
/* Galerkin product for an aggregate map; the device pattern (int32) and the
 * values are written to freshly allocated device arrays returned through
 * rap_*; free them with hzb_free_device.  The inputs are checked on the
 * device first (agg in [-1, nc), ia rising from 0 to nnz, ja in [0, n)); a
 * violation returns ERROR_INPUT_PAR before any kernel indexes by them. */
INT hzb_rap_agg_device(INT n, INT nnz, const INT *ia, const INT *ja,
                       const REAL *val, INT nc, const INT *agg,
                       INT *rap_nnz, INT **rap_ia, INT **rap_ja,
                       REAL **rap_val);
void hzb_free_device(void *p);

/* P1 stiffness matrix of -div(k K grad u) on the Kuhn (Freudenthal) mesh of
 * N^3 cubes of the unit cube (each cube split into the 6 simplices
 * 0 -> e_a -> e_a + e_b -> (1,1,1)), with the Dirichlet vertices eliminated,
 * assembled on the device.  Replaces the cube mesh of mesh_cube_init
 * (src/amr/mesh_cube_anydim.c:30-128), the element loop of call_assembly
 * (examples/elliptic_p1/supporting_elliptic_p1.h:537-647) and
 * set_essential_bc for this mesh.
 *  - rows: the (N-1)^3 interior vertices, x fastest; columns ascending; the
 *    15-point pattern (0, +-e_a, +-(e_a + e_b), +-(1,1,1)) cut at the
 *    boundary, couplings that are exactly zero stay stored.
 *  - d_kcell: per-cube coefficient [z][y][x] (N^3, device), NULL = 1;
 *    K: constant 3x3 tensor, row-major (host), NULL = identity.
 *  - d_ia ((N-1)^3 + 1 ints, device) is always filled and *nnz (host)
 *    receives the entry count; d_ja / d_val (device, nnz each) are filled
 *    when both are given (call once without them to size them).
 *  - ERROR_MAT_SIZE when N < 2 or 15 (N-1)^3 does not fit an INT. */
INT hzb_assemble_p1_kuhn_device(INT N, const REAL *d_kcell, const REAL *K, INT *d_ia,
                                INT *d_ja, REAL *d_val, INT *nnz);
/* copy bytes from device memory returned above into host memory */
INT hzb_copy_to_host(void *dst, const void *src_device, size_t bytes);

/* Galerkin product that allocates nothing.  No counterpart in the
 * reference.  It serves callers that cannot call cudaMalloc: processes whose
 * device memory is reserved up front by their own allocator (a caching pool
 * that owns the whole budget, an embedded solver with a fixed footprint),
 * and library code that must not trigger the implicit device
 * synchronisation of cudaMalloc or cudaFree.  The result equals
 * hzb_rap_agg_device's bit for bit.
 *  - Inputs and outputs are the caller's device arrays: rap_ia (nc+1 ints),
 *    rap_ja (cap_nnz ints) and rap_val (cap_nnz doubles); *rap_nnz receives
 *    the product's entry count, also when it exceeds cap_nnz (then the call
 *    returns ERROR_INPUT_PAR and fills only rap_ia).
 *  - The inputs are checked on the device before any kernel indexes by them:
 *    agg in [-1, nc), ia rising from 0 to nnz, ja in [0, n); a violation
 *    returns ERROR_INPUT_PAR and writes nothing.
 *  - Scratch is one file-scope device array of about 15 MB, held by every
 *    device that loads the library until the process exits.  It limits the
 *    fine matrix to n <= HZB_NOALLOC_MAX_ROWS rows and nnz <=
 *    HZB_NOALLOC_MAX_NNZ entries; larger sizes return ERROR_MAT_SIZE.
 *  - The first call on a device looks up the array's device address (with
 *    that device current); make that first call before any stream capture.
 *  - Every call shares the array, which keeps the last call's contents (the
 *    call clears what must start at zero): calls that overlap on the GPU
 *    (several host threads or streams at once) race.  Runs on the legacy
 *    default stream; it waits for the device three times (after the input
 *    check, to read the slot-list total, to read the entry count) and once
 *    more before returning. */
#define HZB_NOALLOC_MAX_ROWS 65536
#define HZB_NOALLOC_MAX_NNZ  1048576
INT hzb_rap_agg_device_noalloc(INT n, INT nnz, const INT *ia, const INT *ja,
                               const REAL *val, INT nc, const INT *agg,
                               INT cap_nnz, INT *rap_ia, INT *rap_ja,
                               REAL *rap_val, INT *rap_nnz);

#ifdef __cplusplus
}
#endif
#endif /* HAZMATH_B200_H */
