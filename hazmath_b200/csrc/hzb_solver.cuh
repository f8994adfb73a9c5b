// hzb_solver.cuh -- the device-resident UA-AMG hierarchy and its solvers.
#pragma once
#include <vector>
#include "hzb_setup.cuh"

struct hzb_solver;

namespace hzb {

struct Level {
    int n = 0, nnz = 0;
    int *ia = nullptr, *ja = nullptr;
    double *val = nullptr;
    bool own_A = true;
    int bundle_cap = 0;
    int bundle_rows = 128;            // picked by autotune_bundle
    // FP32 copy for the mixed cycle without the stored exact zeros (a zero
    // entry adds nothing to a row sum); aliases ia/ja when there are none
    int nnz32 = 0, bundle_cap32 = 0;
    int vec32 = 0;                    // FP32 schedule: lanes per row, 0 = bundles,
                                      // SELL_LANES = the sliced-ELL copy
    // activity of 256-row blocks while a batched solve runs (else null):
    // the level kernels skip blocks of converged systems
    const unsigned char *act = nullptr;
    int *ia32 = nullptr, *ja32 = nullptr;
    float *val32 = nullptr;
    bool own32 = false;
    SellArrays sell32;                // sliced-ELL copy, when vec32 = SELL_LANES
    // level 0 of the mixed solve with stored exact zeros: the FP64 values of
    // the FP32 copy's pattern, for the outer Krylov loop's SpMV (a zero adds
    // nothing to a row sum, so its result is the full matrix's)
    double *val64nz = nullptr;
    // transfer to level + 1 (P = agg map, R = P^T with ascending rows);
    // smoothed aggregation keeps P as a CSR with values and R's values too
    int nc = 0;
    int *agg = nullptr, *ria = nullptr, *rja = nullptr;
    bool sa = false;
    int *pia = nullptr, *pja = nullptr, pnnz = 0, pcap = 0, rcap = 0;
    double *pval = nullptr, *rval = nullptr;
    DCsr<double> P64() const {
        DCsr<double> m;
        m.n = n; m.nnz = pnnz; m.ia = pia; m.ja = pja; m.val = pval; m.bundle_cap = pcap;
        return m;
    }
    DCsr<double> R64() const {
        DCsr<double> m;
        m.n = nc; m.nnz = pnnz; m.ia = ria; m.ja = rja; m.val = rval; m.bundle_cap = rcap;
        return m;
    }
    // cycle vectors; r1 keeps the restricted residual of the AMLI cycle
    // (allocated on levels >= 1 when that cycle first runs)
    double *b = nullptr, *x = nullptr, *w = nullptr, *t = nullptr, *r1 = nullptr;
    float *b32 = nullptr, *x32 = nullptr, *w32 = nullptr, *t32 = nullptr;
    // smoother data
    double *d_jac = nullptr, *d_gs_f = nullptr, *d_gs_b = nullptr;
    double *d_sor_f = nullptr, *d_sor_b = nullptr;
    float *d_gs32 = nullptr;
    float *l1_32 = nullptr;           // l1 row norms for the FP32 first sweep
    Schedule fwd, bwd, col;
    // coarsest level with the direct solver: the transposed matrix the
    // reference factors (and leaves in mgl[nl-1].A)
    int *tia = nullptr, *tja = nullptr;
    double *tval = nullptr;
    DCsr<double> AT64() const {
        DCsr<double> m;
        m.n = n; m.nnz = nnz; m.ia = tia; m.ja = tja; m.val = tval;
        return m;
    }
    DCsr<double> A64() const {
        DCsr<double> m;
        m.n = n; m.nnz = nnz; m.ia = ia; m.ja = ja; m.val = val; m.bundle_cap = bundle_cap;
        m.bundle_rows = bundle_rows;
        m.act = act;
        return m;
    }
    // the outer loop's FP64 operator: the zero-free copy when there is one
    DCsr<double> A64outer() const {
        if (!val64nz) return A64();
        DCsr<double> m;
        m.n = n; m.nnz = nnz32; m.ia = ia32; m.ja = ja32; m.val = val64nz;
        m.bundle_cap = bundle_cap32;
        m.bundle_rows = bundle_rows;
        m.act = act;
        return m;
    }
    DCsr<float> A32() const {
        DCsr<float> m;
        m.n = n; m.nnz = nnz32; m.ia = ia32; m.ja = ja32; m.val = val32;
        m.bundle_cap = bundle_cap32;
        m.bundle_rows = bundle_rows;
        m.vec_lanes = vec32;
        m.sell = sell32.view();
        m.act = act;
        return m;
    }
    void release();
};

// Scratch of one Krylov loop on an n-vector system.
struct KrylovWork {
    int n = 0;
    double *p = nullptr, *z = nullptr, *r = nullptr, *t = nullptr;
    double *part = nullptr;   // 4 * reduce_blocks(n) + spmv_blocks(n)
    double *sc = nullptr;     // device scalars
    double *h_sc = nullptr;   // pinned host mirror
    int alloc(int n, cudaStream_t s = nullptr);   // scalars zeroed on s (or the current stream)
    void release_device();   // the device arrays (the pinned host mirror stays)
    void release();
};

// A captured preconditioner application, replayed while its key matches.
struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    const void *k0 = nullptr, *k1 = nullptr;
    long long tag = -1, tag2 = 0;
    long long kernels = 0;
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        tag = -1;
    }
};

struct GmresWork;   // Krylov basis of gmres (hzb_gmres.cu)
struct GcgWork;     // search directions of gcg (hzb_cycles.cu)

struct Batch;   // packed independent systems (hzb_batch.cu)
struct BsrHier; // hierarchy of a block (BSR) matrix (hzb_bsr.cu)

// Host-side preconditioner callback used when a foreign pc->fct is given.
struct HostPrecond {
    void (*fct)(double *, double *, void *) = nullptr;
    void *data = nullptr;
    double *h_r = nullptr, *h_z = nullptr;
};

}  // namespace hzb

struct hzb_solver {
    AMG_param amg;
    linear_itsolver_param it;
    hzb_param bp;
    AMG_param *caller_amg = nullptr;   // receives the strong_coupled update
    AMG_param pc_cyc;                  // cycle parameters of precond_amg
    double *pr = nullptr, *pz = nullptr;   // host-pointer precond staging
    cudaStream_t s = nullptr;
    std::vector<hzb::Level> lv;
    int nl = 0;
    double *Ainv = nullptr;           // coarsest-level inverse (coarse_solver 32)
    hzb::KrylovWork kw;               // outer Krylov loop
    hzb::KrylovWork kwc;              // coarse-level CG (coarse_solver != 32)
    hzb::GraphCache g64, g32;         // captured FP64 / FP32 preconditioners
    hzb::GraphCache g32c;             // the FP32 cycles alone (level-0 b32 given)
    hzb::GraphCache gcyc;             // captured AMLI / additive preconditioner
    std::vector<double> amli_coef;    // polynomial of the AMLI cycle (degree + 1)
    // Krylov work kept per level for the coarse-level solves of the
    // nonlinear AMLI cycle and the coarse GMRES fallback
    std::vector<hzb::GmresWork *> gm_ws;
    std::vector<hzb::GcgWork *> gcg_ws;
    unsigned *hec_state = nullptr;    // rand() stream of HEC aggregation (35 words)
    float *omega = nullptr;           // learned fine-level weights (device)
    bool omega_active = false;
    hzb_stats st{};
    const int *host_ia = nullptr;     // host matrix given to setup, if any
    const int *host_ja = nullptr;
    const double *host_val = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    hzb::Batch *batch = nullptr;      // set by batch_setup
    hzb::BsrHier *bsr = nullptr;      // set by bsr_setup
    AMG_param bsr_cyc;                // cycle parameters of precond_dbsr_amg
};

namespace hzb {
int setup(hzb_solver *S, int n, int nnz, const int *d_ia, const int *d_ja,
          const double *d_val, bool copy_in);
// z = B r with B = maxit V/W cycles of the FP64 hierarchy (precond_amg)
int precond64(hzb_solver *S, const double *r, double *z, const AMG_param &cyc);
// one cycle on level-0 b/x already in place (mgcycle)
int cycle64(hzb_solver *S, const AMG_param &cyc, int l0 = 0);
int cycle32(hzb_solver *S, const AMG_param &cyc, bool level0_zero);
// reference PCG on level-0 operator
int pcg(hzb_solver *S, const DCsr<double> &A, const double *b, double *u,
        int pc_kind, HostPrecond *hp, double tol, int maxit, int stop_type,
        int prtlvl, KrylovWork &w, double *relres_out, double *condest);
// preconditioner kinds of pcg / gmres / gcg: none, precond_amg (V/W
// cycles), a host callback, precond_amli, precond_amg_add, and
// precond_nl_amli rooted at level l (PC_NLAMLI + l)
enum { PC_NONE = 0, PC_AMG = 1, PC_HOST = 2, PC_AMLI = 3, PC_ADD = 4, PC_BSR = 5,
       PC_NLAMLI = 16 };
// the preconditioner linear_solver_dcsr_krylov_amg picks for a cycle type
// (itsolver.c:899-917)
int pc_kind_of_cycle(int cycle_type);
// z = M r for a preconditioner kind of pcg / gmres
int apply_precond(hzb_solver *S, int kind, HostPrecond *hp, int n, const double *r,
                  double *z);
// variable-restart GMRES (flexible = false, dcsr_pvgmres) or flexible GMRES
// (dcsr_pvfgmres), right-preconditioned (hzb_gmres.cu)
// (hzb_gmres.cu); ws_slot >= 0 keeps the basis in S->gm_ws[ws_slot] for the
// next call
int gmres(hzb_solver *S, const DCsr<double> &A, const double *b, double *x, int kind,
          HostPrecond *hp, double tol, int MaxIt, int restart, int stop_type, int prtlvl,
          bool flexible, double *relres_out, int ws_slot = -1);
void gmres_release(hzb_solver *S);
// preconditioned MINRES, dcsr_pminres (hzb_minres.cu)
int minres(hzb_solver *S, const DCsr<double> &A, const double *b, double *u, int kind,
           HostPrecond *hp, double tol, int MaxIt, int stop_type, int prtlvl,
           double *relres_out);
// generalized conjugate gradient, dcsr_pgcg (hzb_cycles.cu)
int gcg(hzb_solver *S, const DCsr<double> &A, const double *b, double *u, int kind,
        HostPrecond *hp, double tol, int MaxIt, int stop_type, int prtlvl, double *relres_out,
        int ws_slot = -1);
void gcg_release(hzb_solver *S);
// coefficients of the AMLI polynomial, amg_amli_coef (parameters.c:714-775)
int amli_coefficients(double lambda_max, double lambda_min, int degree, double *coef);
// what the cycles of a kind need before they run (and before a graph
// capture): S->amli_coef for the AMLI cycle (cyc.amli_coef when given, else
// the setup's choice lambda in [0.5, 2], amg_setup_ua.c:1276-1281) and the
// per-level r1 vectors
int cycles_prepare(hzb_solver *S, int kind, const AMG_param &cyc);
// AMLI / nonlinear AMLI / additive cycles from level l with level l's b and
// x in place (hzb_cycles.cu)
int amli64(hzb_solver *S, const AMG_param &cyc, const double *coef, int l);
int nl_amli64(hzb_solver *S, const AMG_param &cyc, int l);
int add_cycle64(hzb_solver *S, const AMG_param &cyc);
// z = B r with maxit cycles of the kind (precond_amli / precond_nl_amli
// rooted at level l / precond_amg_add, precond.c:232-355)
int precond_cycles(hzb_solver *S, int kind, int l, int maxit, const double *r, double *z,
                   const AMG_param &cyc);
// coarsest-level solve of the cycles: the direct inverse, else
// coarse_itsolver (mgcycle.c:34-52) to the tolerance ctol
int coarse_solve64(hzb_solver *S, const AMG_param &cyc, double ctol);
// alpha = min((e_c, r_c) / (e_c, A_c e_c), 2) on level c (uses the level's t)
int coarse_alpha(hzb_solver *S, int c, const double *rc, double *alpha);
// FP32-cycle flexible CG (mixed precision)
int fcg_mixed(hzb_solver *S, const double *b, double *x, double tol, int maxit,
              int prtlvl, double *relres_out);
int ensure_fp32(hzb_solver *S);
// z = B r with the preconditioner the handle's solve uses (the FP32 cycle in
// mixed precision, precond_amg's FP64 cycle otherwise)
int solver_precond(hzb_solver *S, const double *r, double *z);
// Mean over ns seeded vectors of ||E^2 e||_A^2 / ||e||_A^2 for the solve's
// own cycle E = I - B A, e the errors two cycles leave (random vectors after
// three plain l1 sweeps); uses the Krylov scratch vectors r, z.
int cycle_contraction(hzb_solver *S, int ns, unsigned long long seed, double *loss);
// learned-weight loss (hzb_learn.cu)
int learn_errors(hzb_solver *S, int ns, unsigned long long seed, double *E,
                 const float *omega, int ncyc);
int learn_loss_grad(hzb_solver *S, const float *omega, int ns, const double *E, int ncyc,
                    double *loss, float *domega);
// transfers of mgcycle: b_{l+1} = R w (dcsr_mxv_agg, or dcsr_mxv for
// smoothed aggregation) and x_l += alpha P x_{l+1} (dcsr_aAxpy_agg /
// dcsr_aAxpy)
int restrict_level(hzb_solver *S, int l, const double *w, double *bc);
int prolong_level(hzb_solver *S, int l, const double *xc, double *x, double alpha);
// one forward Gauss-Seidel sweep of level l on its schedule (level b, x)
int time_gs_sweep(hzb_solver *S, int l);
// smoothing of level l as mgcycle's pre (pre = true) / post smoothing calls
int smooth64(hzb_solver *S, int l, bool pre, const AMG_param &cyc);
// diagonals and sweep schedules the configured smoother needs on level L
int level_smoother_data(hzb_solver *S, Level &L);
void destroy(hzb_solver *S);
// batched independent systems (hzb_batch.cu): off[nsys + 1] host row offsets
int batch_setup(hzb_solver *S, int nsys, const int *off, int n, int nnz, const int *d_ia,
                const int *d_ja, const double *d_val);
int batch_solve(hzb_solver *S, const double *b, double *x, double tol, int maxit,
                int *h_iters, double *h_relres, double *h_seconds);
void batch_release(hzb_solver *S);
// ERROR_SOLVER_MISC if a device wait of the cycle (a grid barrier) ran out
int check_waits(hzb_solver *S);
// that word as an int for the kernels' bounded waits (null before the
// handle's Krylov scratch exists: the caller then avoids the waits)
int *wait_err(hzb_solver *S);
// terminal levels of the batched systems, called by setup's level loop in
// batch mode: which systems end on level lvl (their dense inverses; *live =
// rows of the others), then after the aggregation the removal of their rows
// from the coarser levels; and the solves of a level's terminal blocks
int batch_level_begin(hzb_solver *S, int lvl, bool force, int *live);
int batch_level_end(hzb_solver *S, int lvl, int *agg, int *nagg);
int batch_terminal_solve(hzb_solver *S, int lvl, bool fp32);
bool batch_has_terminal(const hzb_solver *S, int lvl);
// UA-AMG of a block matrix (hzb_bsr.cu): amg_setup_ua_bsr on nrow block rows
// of nb x nb blocks (row-major); z = B r of precond_dbsr_amg with the cycle
// parameters S->bsr_cyc; the scalar expansion of the level-0 matrix (the
// operator of the Krylov loop); a level's block matrix (sizes always, the
// arrays where given) and its block aggregates
int bsr_setup(hzb_solver *S, int nrow, int nnzb, int nb, const int *d_ia, const int *d_ja,
              const double *d_val);
int bsr_precond(hzb_solver *S, const double *r, double *z);
int bsr_cycle(hzb_solver *S, const AMG_param &cyc);
DCsr<double> bsr_scalar_A(hzb_solver *S);
int bsr_block_size(const hzb_solver *S);
int bsr_level_copy(const hzb_solver *S, int l, int *nrow, int *nnzb, int *ia, int *ja,
                   double *val, int *agg);
void bsr_release(hzb_solver *S);
// hzb_time_kernel's block kernels (HZB_K_BSR_*)
int bsr_time_kernel(hzb_solver *S, int which, int l, int reps, double *ms_per_launch,
                    double *bytes_per_launch);
}  // namespace hzb
