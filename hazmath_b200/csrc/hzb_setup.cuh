// hzb_setup.cuh -- setup-phase kernels: strength graph, heavy edge matching,
// restriction pattern, Galerkin product, smoother diagonals, level schedules,
// colouring, dense coarse factorisation.
#pragma once
#include <vector>
#include "hzb_kernels.cuh"

namespace hzb {

// out[0..n] = exclusive scan of in[0..n), out[n] = total.  tmp: >= scan_tmp(n)
int scan_tmp_size(int n);
int scan_exclusive(const int *in, int *out, int n, int *tmp, cudaStream_t s);

// strength graph Neigh (construct_strongly_coupled, amg_setup_ua.c:375-455);
// nia sized n+1, nja/nval sized nnz; returns its nnz through *nnnz.
int strength_graph(const DCsr<double> &A, double theta, int *nia, int *nja,
                   double *nval, int *nnnz, int *tmp, cudaStream_t s);

// heavy edge matching (aggregation_hem, amg_setup_ua.c:913-1050), exact
// reference visiting order, on the strength graph.  agg: n outputs.
// Returns SUCCESS, or ERROR_AMG_COARSEING where the reference exits (an
// isolated point on the second pass).
int hem_exact(int n, const int *nia, const int *nja, const double *nval,
              int *agg, int *nagg, int *work_n, cudaStream_t s);
// deterministic parallel matching (mutual heaviest neighbour rounds + the
// same leftover rule against pre-pass-2 sizes); not bit-exact.
int hem_parallel(int n, const int *nia, const int *nja, const double *nval,
                 int *agg, int *nagg, int *work, cudaStream_t s);

// VMB aggregation (aggregation_vmb, amg_setup_ua.c:596-736) on the strength
// graph in the reference's three sequential steps and visiting orders;
// *nagg = 0 where the reference fails (no aggregate after step 1).
// work: 2n ints.
int vmb_aggregate(int n, const int *nia, const int *nja, int max_agg, int *agg, int *nagg,
                  int *work, cudaStream_t s);

// HEC aggregation (aggregation_hec, amg_setup_ua.c:752-845) in the
// reference's order: rows visited in the permutation iarray_shuffle draws
// from glibc's rand() (state: 35 device words, seeded by hec_seed and carried
// across levels), each pairing with its strongest neighbour when that one is
// unvisited, else joining its aggregate.  work: hec_work_ints(n) ints.
// ERROR_AMG_COARSEING where the reference exits (a row of several entries
// without an off-diagonal one).
int hec_seed(unsigned *state, unsigned seed, cudaStream_t s);
int hec_aggregate(int n, const int *nia, const int *nja, const double *nval, int *agg,
                  int *nagg, unsigned *state, int *work, cudaStream_t s);
size_t hec_work_ints(int n);

// A caller's Galerkin inputs checked on the device before any kernel indexes
// by them (aggregate ids in [-1, nc), row pointers rising from 0 to nnz,
// columns in [0, n)); d_bad is one device int of scratch.  Synchronises s;
// ERROR_INPUT_PAR with a message on bad input.
int check_rap_inputs(int n, int nnz, const int *ia, const int *ja, int nc, const int *agg,
                     int *d_bad, cudaStream_t s);

// R = P^T: rows of R list fine indices ascending (dcsr_trans, sparse.c:770).
int restriction_pattern(int n, int nc, const int *agg, int *ria, int *rja,
                        int *tmp, cudaStream_t s);

// A_c = R A P (dcsr_rap_agg, sparse.c:2557-2690), reference slot order and
// summation order.  Allocates *cia (nc+1), *cja, *cval.
int rap_agg(const DCsr<double> &A, int nc, const int *agg, const int *ria,
            const int *rja, int **cia, int **cja, double **cval, int *cnnz,
            cudaStream_t s);

// A^T with ascending column indices in every row (dcsr_transz with p = NULL,
// sparse.c); allocates the three arrays.
int transpose_csr(const DCsr<double> &A, int **tia, int **tja, double **tval,
                  cudaStream_t s);

// Per-row diagonals used by the smoothers (d_jac: last diagonal entry or 0;
// d_gs_f/_b: 1/a_ii of the last usable diagonal entry with the reference's
// carry-over from the previous row in sweep order; d_sor_f/_b: last diagonal
// entry with carry-over).
int smoother_diagonals(const DCsr<double> &A, double *d_jac, double *d_gs_f,
                       double *d_gs_b, double *d_sor_f, double *d_sor_b,
                       cudaStream_t s);

// Level schedule of lexicographic Gauss-Seidel: rows grouped into sets that
// depend only on earlier sets (forward: on lower-numbered neighbours in A or
// A^T; backward: higher).  perm (n) and host set pointers.
struct Schedule {
    int *rows = nullptr;           // device, n
    int *set_ptr = nullptr;        // device, nsets+1
    std::vector<int> h_ptr;        // host copy of set_ptr
    std::vector<int> run_first;    // runs of small sets for one CTA: [first,last)
    std::vector<int> run_last;     // (-1: one large set)
    std::vector<int> run_max;      // the run's largest set
    unsigned *bar = nullptr;       // device, 2 words: grid barrier of gs_sets_grid
    void release();
};
int gs_schedule(int n, const int *ia, const int *ja, int nnz, int backward,
                Schedule *sch, cudaStream_t s);
// Colour classes (Jones-Plassmann with hashed priorities, smallest free
// colour): rows sorted by colour, host colour pointers.
int multicolor(int n, const int *ia, const int *ja, Schedule *sch,
               cudaStream_t s);

// Coarsest level: dense inverse (row-major, n x n) of the SPD coarse matrix
// through a Cholesky factorisation.  Returns ERROR_DATA_ZERODIAG if a pivot
// is not positive.
int dense_inverse(const DCsr<double> &A, double **Ainv, cudaStream_t s);

// Smoothed aggregation (hzb_sa.cu).  sa_prolongation turns N (nval, in
// place: the strength graph, filtered, or a copy of A without the filter)
// into S = I - omega D^{-1} N and forms P = S P_tent for the aggregate map;
// transpose_rect is dcsr_trans of an n x ncols CSR; rap_general is dcsr_rap
// in the reference's traversal order.
int sa_prolongation(const DCsr<double> &A, const int *nia, const int *nja, double *nval,
                    int nc, const int *agg, double omega, bool filter, int **pia, int **pja,
                    double **pval, int *pnnz, cudaStream_t s);
int transpose_rect(int n, int ncols, int nnz, const int *ia, const int *ja, const double *val,
                   int **tia, int **tja, double **tval, cudaStream_t s);
int rap_general(int nc, const int *ria, const int *rja, const double *rval,
                const DCsr<double> &A, const int *pia, const int *pja, const double *pval,
                int **cia, int **cja, double **cval, int *cnnz, cudaStream_t s);

// P1 stiffness on the Kuhn mesh of N^3 cubes, interior dofs (hzb_assemble.cu):
// ia ((N-1)^3 + 1) always; ja, val (nnz each) when both are given.
int assemble_kuhn_p1(int N, const double *kcell, const double *K, int *ia, int *ja,
                     double *val, int *nnz_out, cudaStream_t s);

}  // namespace hzb
