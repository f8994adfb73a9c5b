// hzb_hec.cu -- HEC aggregation (aggregation_hec, amg_setup_ua.c:752-845) in
// the reference's order.
//
// The reference visits the rows in the order of a random permutation drawn
// by iarray_shuffle (array.c:302-315) from the C library's rand(): for
// i = 0 .. n-2, j = i + rand() / (RAND_MAX / (n - i) + 1), swap perm[i] and
// perm[j].  Each visited row i pairs with its most strongly coupled
// neighbour j (the first maximum of |a_ij| off the diagonal of the strength
// graph) when j is still unvisited, else takes j's aggregate -- also when i
// was already placed by an earlier row; a row whose strength-graph row holds
// only itself is UNPT.
//
// rand() here is glibc's: random() of the TYPE_3 additive feedback generator
// (the published algorithm of glibc's random_r.c and BSD random(3)).  srand(s)
// fills r[0..30] with r[0] = s (0 counts as 1), r[k] = 16807 r[k-1] mod
// (2^31 - 1); r[31..33] = r[0..2]; then 310 outputs of
// r[k] = r[k-31] + r[k-3] (mod 2^32) are discarded; each rand() returns the
// next r[k] >> 1.  The reference never seeds it, so a fresh process starts
// from srand(1), and the stream continues across levels and setups.  Every
// setup here starts from srand(1): the first UA-AMG setup of a fresh
// process, whose aggregates this reproduces bit for bit.
//
// The best neighbour of every row depends on the matrix alone and is found in
// parallel; the shuffle and the walk are sequential by definition and run in
// one thread, with the permutation and the map in shared memory when they
// fit (about 40 ns per row) and in global memory otherwise (about 1 us per
// row).  A parity path, like exact HEM.
#include "hzb_setup.cuh"

namespace hzb {

namespace {
constexpr int UNVISITED = -2;
constexpr int ISOLATED = -3;      // best[i] of a row with only its diagonal
constexpr int HEC_SMEM_ROWS = 26 * 1024;   // perm + map in 208 KB

// glibc TYPE_3 state: 34-word ring and the index of the next output
struct Rand3 {
    unsigned r[34];
    int k;
    __device__ void seed(unsigned s) {
        int x = (int)(s ? s : 1u);
        r[0] = (unsigned)x;
        for (int i = 1; i < 31; ++i) {
            // 16807 x mod (2^31 - 1) without overflow (Schrage's method)
            const int hi = x / 127773, lo = x % 127773;
            x = 16807 * lo - 2836 * hi;
            if (x < 0) x += 2147483647;
            r[i] = (unsigned)x;
        }
        for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
        k = 34;
        for (int i = 0; i < 310; ++i) next();
    }
    __device__ unsigned next() {
        const unsigned v = r[(k - 31) % 34] + r[(k - 3) % 34];
        r[k % 34] = v;
        k = k + 1 >= 34 * 64 ? k + 1 - 34 * 32 : k + 1;   // same residue mod 34
        return v;
    }
    __device__ int rand() { return (int)(next() >> 1); }
};

// first maximum of |a| off the diagonal; ISOLATED for a row of one entry;
// -1 (an error) for a longer row without an off-diagonal entry
__global__ void k_hec_best(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                           const double *__restrict__ a, int *best, int *bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b0 = ia[i], b1 = ia[i + 1];
        if (b1 - b0 == 1) { best[i] = ISOLATED; continue; }
        int k = -1;
        double mx = -1.0;
        for (int p = b0; p < b1; ++p)
            if (ja[p] != i && fabs(a[p]) > mx) { k = p; mx = fabs(a[p]); }
        best[i] = k < 0 ? -1 : ja[k];
        if (k < 0) atomicOr(bad, 1);
    }
}

// One thread: the shuffle, then the walk.  state: 35 words (ring + index)
// carried across levels; out[0] = aggregates.  SMEM: perm and map staged in
// shared memory (n <= HEC_SMEM_ROWS).
template <bool SMEM>
__global__ void __launch_bounds__(32)
k_hec_walk(int n, const int *__restrict__ best, int *perm_g, int *agg, unsigned *state,
           int *out) {
    extern __shared__ int sh[];
    if (threadIdx.x != 0) return;
    Rand3 g;
    for (int i = 0; i < 34; ++i) g.r[i] = state[i];
    g.k = (int)state[34];
    int *perm = SMEM ? sh : perm_g;
    int *v = SMEM ? sh + n : agg;
    for (int i = 0; i < n; ++i) { perm[i] = i; v[i] = UNVISITED; }
    for (int i = 0; i < n - 1; ++i) {
        const int j = i + g.rand() / (2147483647 / (n - i) + 1);
        const int t = perm[j];
        perm[j] = perm[i];
        perm[i] = t;
    }
    int na = 0;
    for (int q = 0; q < n; ++q) {
        const int i = perm[q];
        const int j = best[i];
        if (j == ISOLATED) { v[i] = UNPT; continue; }
        if (v[j] < UNPT) { v[j] = na; v[i] = na; ++na; }
        else v[i] = v[j];
    }
    for (int i = 0; i < n; ++i) agg[i] = v[i] < 0 ? UNPT : v[i];
    for (int i = 0; i < 34; ++i) state[i] = g.r[i];
    state[34] = (unsigned)g.k;
    out[0] = na;
}

__global__ void k_hec_seed(unsigned *state, unsigned s) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Rand3 g;
    g.seed(s);
    for (int i = 0; i < 34; ++i) state[i] = g.r[i];
    state[34] = (unsigned)g.k;
}
}  // namespace

int hec_seed(unsigned *state, unsigned seed, cudaStream_t s) {
    k_hec_seed<<<1, 32, 0, s>>>(state, seed);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

int hec_aggregate(int n, const int *nia, const int *nja, const double *nval, int *agg,
                  int *nagg, unsigned *state, int *work, cudaStream_t s) {
    // work: n (best) + 2 (flag, count) ints, + n (permutation) when the walk
    // does not fit shared memory
    int *best = work, *flag = work + n, *cnt = work + n + 1, *perm = work + n + 2;
    HZB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    k_hec_best<<<grid_for(n), 256, 0, s>>>(n, nia, nja, nval, best, flag);
    count_launch();
    const bool smem = n <= HEC_SMEM_ROWS;
    if (smem) {
        const size_t bytes = sizeof(int) * 2 * (size_t)n;
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_hec_walk<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(int) * 2 * HEC_SMEM_ROWS));
            attr = true;
        }
        k_hec_walk<true><<<1, 32, bytes, s>>>(n, best, perm, agg, state, cnt);
    } else {
        k_hec_walk<false><<<1, 32, 0, s>>>(n, best, perm, agg, state, cnt);
    }
    count_launch();
    HZB_LAUNCH_CHECK();
    int h[2] = {0, 0};
    HZB_CUDA(cudaMemcpyAsync(h, flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    HZB_CUDA(cudaStreamSynchronize(s));
    if (h[0]) {
        // the reference exits here (amg_setup_ua.c:830-834)
        set_error_msg("HEC aggregation: a strength-graph row of several entries has no "
                      "off-diagonal entry");
        return ERROR_AMG_COARSEING;
    }
    *nagg = h[1];
    return SUCCESS;
}

size_t hec_work_ints(int n) { return (size_t)2 * n + 2; }

}  // namespace hzb
