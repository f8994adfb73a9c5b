// hzb_assemble.cu -- P1 stiffness matrix of -div(k K grad u) on the Kuhn
// (Freudenthal) tetrahedral mesh of N^3 cubes of the unit cube, assembled on
// the device straight into the interior-dof CSR the solver reads.
//
// The reference assembles element by element: call_assembly
// (examples/elliptic_p1/supporting_elliptic_p1.h:537-647) computes each
// simplex's local stiffness |T| grad(l_i) . grad(l_j) (grad_compute,
// local_sm), adds it into the pattern of symb_assembly (assemble_matrix), and
// set_essential_bc then removes the Dirichlet vertices; the mesh is the cube
// triangulation of mesh_cube_init (src/amr/mesh_cube_anydim.c:30-128).
//
// Here the mesh is implicit.  Every cube is split into the 6 path simplices
// 0 -> e_p0 -> e_p0 + e_p1 -> (1,1,1) (p a permutation of the axes), whose
// barycentric gradients are constant multiples of the axes, so a simplex's
// local matrix is (G K G^T) / 6 * h times the cube's coefficient, with G the
// 4 x 3 gradient table of the path (entries -1, 0, 1).  Every interior
// vertex gathers its 15 couplings (0, +-e_a, +-(e_a + e_b), +-(1,1,1)) from
// the simplices of its 8 surrounding cubes: no scatter, no atomics, each row
// written once.
//
// Which coupling and which surrounding cube each of the 96 local entries
// (6 simplices x 4 x 4) feeds is fixed by the geometry, so the kernel is
// generated at compile time from that table: the 15 sums and the 8 cube
// coefficients live in registers and each entry is one multiply and one add
// whose coefficient (the only thing K changes) is a constant-bank operand.
// A coupling sums its entries in the order (permutation, local row, local
// column) starting from +0.0, the order of the host generator
// (hazmath_b200/problems.py kuhn3d_p1), so both give the same bits.
//
// Layout: interior vertices (x, y, z) in [0, N-1)^3, row r = x + m (y + m z)
// with m = N - 1, columns ascending; the coefficient array is [z][y][x] over
// the N^3 cubes.  One kernel writes everything: a CTA takes 256 consecutive
// rows, gets its first row pointer in closed form and the others by a block
// scan of the row lengths (no count pass, no host round trip), stages its
// entries in shared memory and writes its contiguous slice of ja / val with
// coalesced stores; it is bound by those writes (12 bytes per entry).
#include "hzb_setup.cuh"
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

namespace hzb {

namespace {
constexpr int KU_ROWS = 256;     // rows per CTA pass
constexpr int KU_OFFS = 15;      // couplings per row
constexpr int KU_TERMS = 96;     // 6 simplices x 4 x 4 local entries
// staging slots: a CTA's entries plus room for the alignment offset of its
// first entry (the value slots keep the column slots 16-byte aligned)
constexpr int KU_SV = KU_ROWS * KU_OFFS + 2, KU_SJ = KU_ROWS * KU_OFFS + 4;
static_assert((KU_SV * 8) % 16 == 0, "column staging alignment");

// The couplings in ascending column order: the column offset
// ox + m oy + m^2 oz orders them by (oz, oy, ox) for every m >= 2 (their
// components are all >= 0 or all <= 0); for m = 1 only (0, 0, 0) exists.
constexpr int KU_OFF[KU_OFFS][3] = {
    {-1, -1, -1}, {0, -1, -1}, {-1, 0, -1}, {0, 0, -1}, {-1, -1, 0}, {0, -1, 0}, {-1, 0, 0},
    {0, 0, 0},    {1, 0, 0},   {0, 1, 0},   {1, 1, 0},  {0, 0, 1},   {1, 0, 1},  {0, 1, 1},
    {1, 1, 1}};

// the permutations of (0, 1, 2) in lexicographic order
constexpr int KU_PERM[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

struct KuTerms {
    int o[KU_TERMS];        // coupling fed by local entry t
    int corner[KU_TERMS];   // surrounding cube: the row vertex's corner dx | dy<<1 | dz<<2
};

constexpr int ku_find(int ox, int oy, int oz) {
    for (int o = 0; o < KU_OFFS; ++o)
        if (KU_OFF[o][0] == ox && KU_OFF[o][1] == oy && KU_OFF[o][2] == oz) return o;
    return -1;
}

// local entry t = 16 p + 4 a + b: row vertex v_a, column vertex v_b of the
// path simplex of permutation p
constexpr KuTerms ku_terms_table() {
    KuTerms T{};
    for (int p = 0; p < 6; ++p) {
        int v[4][3] = {};
        for (int i = 0; i < 3; ++i) {
            for (int d = 0; d < 3; ++d) v[i + 1][d] = v[i][d];
            v[i + 1][KU_PERM[p][i]] += 1;
        }
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const int t = 16 * p + 4 * a + b;
                T.o[t] = ku_find(v[b][0] - v[a][0], v[b][1] - v[a][1], v[b][2] - v[a][2]);
                T.corner[t] = v[a][0] | (v[a][1] << 1) | (v[a][2] << 2);
            }
    }
    return T;
}
constexpr KuTerms KU_T = ku_terms_table();
static_assert(ku_find(1, 1, 1) == 14 && ku_find(0, 0, 0) == 7, "coupling order");

__constant__ double c_ku_e[KU_TERMS];   // local entries (G K G^T) / 6 * h, t order

// The local entries for N cubes per axis and the tensor K.
void ku_entries(int N, const double *K, double *e) {
    const double h = 1.0 / N;
    double Kt[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Kt[i][j] = K ? K[3 * i + j] : (i == j ? 1.0 : 0.0);
    // barycentric gradients in permuted coordinates (h = 1):
    // l0 = 1 - x'0, l1 = x'0 - x'1, l2 = x'1 - x'2, l3 = x'2
    const int Gp[4][3] = {{-1, 0, 0}, {1, -1, 0}, {0, 1, -1}, {0, 0, 1}};
    for (int p = 0; p < 6; ++p) {
        double G[4][3];
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c) G[a][KU_PERM[p][c]] = Gp[a][c];
        // every row of G has at most two nonzeros, equal to +-1, so these
        // sums are exact whatever their order
        double GK[4][3];
        for (int a = 0; a < 4; ++a)
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += G[a][k] * Kt[k][j];
                GK[a][j] = s;
            }
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += GK[a][k] * G[b][k];
                e[16 * p + 4 * a + b] = s / 6.0 * h;
            }
    }
}

// The coupling and cube of local entry T as compile-time constants, and
// whether the entry vanishes for every diagonal K: path vertices a, b whose
// gradients share no axis ((0,2), (0,3), (1,3) and their transposes).
template <int T> struct KuTerm {
    static constexpr int o = KU_T.o[T], corner = KU_T.corner[T];
    static constexpr int a = (T >> 2) & 3, b = T & 3;
    static constexpr bool zero_if_diagonal =
        (a == 0 && b >= 2) || (b == 0 && a >= 2) || (a == 1 && b == 3) || (a == 3 && b == 1);
};

// acc[o] += e_t k_corner for entry T.  With DIAG the entries that vanish
// for a diagonal K are left out: their products are signed zeros, and adding
// one to a sum that starts at +0.0 never changes it.
template <bool DIAG, int T>
__device__ __forceinline__ void ku_term(double (&acc)[KU_OFFS], const double (&kc)[8]) {
    if constexpr (!(DIAG && KuTerm<T>::zero_if_diagonal))
        acc[KuTerm<T>::o] =
            __dadd_rn(acc[KuTerm<T>::o], __dmul_rn(c_ku_e[T], kc[KuTerm<T>::corner]));
}

// every entry in t order (a comma fold runs left to right)
template <bool DIAG, int... T>
__device__ __forceinline__ void ku_sum(double (&acc)[KU_OFFS], const double (&kc)[8],
                                       std::integer_sequence<int, T...>) {
    (ku_term<DIAG, T>(acc, kc), ...);
}

// Entries of the rows before t along one axis whose neighbour at offset od
// is inside [0, m): t' in [0, t) with 0 <= t' + od < m.
__device__ __forceinline__ int ku_prefix(int od, int t, int m) {
    return od == 0 ? t : (od > 0 ? min(t, m - 1) : max(t - 1, 0));
}

// the components of coupling O as compile-time constants
template <int O> struct KuOff {
    static constexpr int x = KU_OFF[O][0], y = KU_OFF[O][1], z = KU_OFF[O][2];
};
using KuSeq = std::make_integer_sequence<int, KU_OFFS>;

// Row pointer of interior vertex (x, y, z) in closed form: the entries of the
// slabs before z, of the lines before y in slab z and of the vertices before
// x in line (y, z), coupling by coupling (a box of rows keeps the couplings
// whose neighbour stays inside, a product of per-axis counts).  (0, 0, m)
// gives the total.  Every partial sum is below 15 m^3 < 2^31.
template <int O>
__device__ __forceinline__ int ku_rowptr_term(int m, int x, int y, int z) {
    constexpr int ox = KuOff<O>::x, oy = KuOff<O>::y, oz = KuOff<O>::z;
    const int fx = m - (ox < 0 ? -ox : ox), fy = m - (oy < 0 ? -oy : oy);
    const int iny = (unsigned)(y + oy) < (unsigned)m, inz = (unsigned)(z + oz) < (unsigned)m;
    return fx * fy * ku_prefix(oz, z, m) + fx * ku_prefix(oy, y, m) * inz +
           ku_prefix(ox, x, m) * iny * inz;
}

template <int... O>
__device__ __forceinline__ int ku_rowptr(int m, int x, int y, int z,
                                         std::integer_sequence<int, O...>) {
    return (ku_rowptr_term<O>(m, x, y, z) + ...);
}

__device__ __forceinline__ int ku_rowptr_of(int m, int r) {
    const int q = r / m;
    return ku_rowptr(m, r - q * m, q % m, q / m, KuSeq{});
}

// bit o set when coupling o of vertex (x, y, z) stays inside the grid
template <int... O>
__device__ __forceinline__ unsigned ku_inside(int m, int x, int y, int z,
                                              std::integer_sequence<int, O...>) {
    return ((((unsigned)(x + KuOff<O>::x) < (unsigned)m &&
              (unsigned)(y + KuOff<O>::y) < (unsigned)m &&
              (unsigned)(z + KuOff<O>::z) < (unsigned)m) ? 1u << O : 0u) | ...);
}

// the row's inside couplings, in column order, into the CTA's staging slice
template <int... O>
__device__ __forceinline__ void ku_put(unsigned mask, const double (&acc)[KU_OFFS], int r, int m,
                                       double *sv, int *sj, int p,
                                       std::integer_sequence<int, O...>) {
    (((mask >> O) & 1u
          ? (sv[p] = acc[O], sj[p] = r + KuOff<O>::x + m * (KuOff<O>::y + m * KuOff<O>::z), ++p)
          : 0),
     ...);
}

// q = n / m for 0 <= n < 2^31 and m < 2^10 through a double product (exact
// to within one) and one correction
__device__ __forceinline__ int ku_div(int n, int m, double inv_m) {
    int q = (int)((double)n * inv_m);
    if (q * m > n) --q;
    else if ((q + 1) * m <= n) ++q;
    return q;
}

// Row pointers (and, when ja and val are given, the entries) of all rows.
// The staging slices start at the CTA's first entry's offset within a
// 16-byte group, so with VEC the copy-out moves aligned pairs of values and
// quadruples of columns (ja and val 16-byte aligned).
template <bool VEC, bool DIAG>
__global__ void __launch_bounds__(KU_ROWS)
k_kuhn_fill(int N, int rows, const double *__restrict__ kcell, int *__restrict__ ia,
            int *__restrict__ ja, double *__restrict__ val) {
    extern __shared__ __align__(16) double ku_sm[];
    __shared__ int s_warp[KU_ROWS / 32];
    __shared__ int s_base;
    double *sv = ku_sm;                                   // KU_SV values
    int *sj = reinterpret_cast<int *>(sv + KU_SV);        // KU_SJ columns
    const int m = N - 1;
    const double inv_m = 1.0 / m;
    const bool fill = ja && val;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r0 = blockIdx.x * KU_ROWS; r0 < rows; r0 += gridDim.x * KU_ROWS) {
        const int r = r0 + threadIdx.x;
        int x = 0, y = 0, z = 0;
        unsigned mask = 0;
        if (r < rows) {
            const int q = ku_div(r, m, inv_m);
            z = ku_div(q, m, inv_m);
            y = q - z * m;
            x = r - q * m;
            mask = ku_inside(m, x, y, z, KuSeq{});
        }
        // exclusive scan of the row lengths over the CTA
        const int len = __popc(mask);
        int inc = len;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += v;
        }
        if (lane == 31) s_warp[warp] = inc;
        if (threadIdx.x == 0) s_base = ku_rowptr_of(m, r0);
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < KU_ROWS / 32; ++w) {
            const int t = s_warp[w];
            before += w < warp ? t : 0;
            total += t;
        }
        const int pos = before + inc - len;   // within the CTA's slice
        const int base = s_base;
        const int vo = VEC ? (base & 1) : 0, jo = VEC ? (base & 3) : 0;
        if (r < rows) {
            ia[r] = base + pos;
            if (r == rows - 1) ia[rows] = base + total;
        }
        if (fill && r < rows) {
            // the 8 cubes around vertex (x+1, y+1, z+1)
            double kc[8];
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                const int cx = x + 1 - (d & 1), cy = y + 1 - ((d >> 1) & 1),
                          cz = z + 1 - (d >> 2);
                kc[d] = kcell ? kcell[((long long)cz * N + cy) * N + cx] : 1.0;
            }
            double acc[KU_OFFS];
#pragma unroll
            for (int o = 0; o < KU_OFFS; ++o) acc[o] = 0.0;
            ku_sum<DIAG>(acc, kc, std::make_integer_sequence<int, KU_TERMS>{});
            ku_put(mask, acc, r, m, sv + vo, sj + jo, pos, KuSeq{});
        }
        __syncthreads();
        if (fill) {
            const int stop = base + total;
            if (VEC) {
                // values: aligned pairs from the even entry at or before base
                const int vb = base - vo;
                for (int k = threadIdx.x; vb + 2 * k < stop; k += KU_ROWS) {
                    const int g = vb + 2 * k;
                    const double2 v2 = reinterpret_cast<const double2 *>(sv)[k];
                    if (g >= base && g + 1 < stop) {
                        reinterpret_cast<double2 *>(val + g)[0] = v2;
                    } else {
                        if (g >= base) val[g] = v2.x;
                        if (g + 1 >= base && g + 1 < stop) val[g + 1] = v2.y;
                    }
                }
                // columns: aligned quadruples
                const int jb = base - jo;
                for (int k = threadIdx.x; jb + 4 * k < stop; k += KU_ROWS) {
                    const int g = jb + 4 * k;
                    const int4 j4 = reinterpret_cast<const int4 *>(sj)[k];
                    if (g >= base && g + 3 < stop) {
                        reinterpret_cast<int4 *>(ja + g)[0] = j4;
                    } else {
                        const int e[4] = {j4.x, j4.y, j4.z, j4.w};
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            if (g + u >= base && g + u < stop) ja[g + u] = e[u];
                    }
                }
            } else {
                for (int i = threadIdx.x; i < total; i += KU_ROWS) {
                    val[base + i] = sv[i];
                    ja[base + i] = sj[i];
                }
            }
        }
        __syncthreads();
    }
}
}  // namespace

int assemble_kuhn_p1(int N, const double *kcell, const double *K, int *ia, int *ja,
                     double *val, int *nnz_out, cudaStream_t s) {
    if (N < 2) return ERROR_MAT_SIZE;
    const long long m = N - 1, rows = m * m * m;
    if (rows * KU_OFFS >= (1LL << 31)) return ERROR_MAT_SIZE;
    // entries: per coupling, the vertices whose neighbour stays inside
    long long nnz = 0;
    for (int o = 0; o < KU_OFFS; ++o) {
        long long c = 1;
        for (int d = 0; d < 3; ++d) c *= m - (KU_OFF[o][d] < 0 ? -KU_OFF[o][d] : KU_OFF[o][d]);
        nnz += c;
    }
    if (nnz_out) *nnz_out = (int)nnz;
    double e[KU_TERMS];
    ku_entries(N, K, e);
    HZB_CUDA(cudaMemcpyToSymbolAsync(c_ku_e, e, sizeof(e), 0, cudaMemcpyHostToDevice, s));
    const bool fill = ja && val;
    // staging: the values (two spare slots for the alignment offset), then
    // the columns (four spare)
    const size_t smem = fill ? (size_t)KU_SV * sizeof(double) + (size_t)KU_SJ * sizeof(int) : 0;
    const bool vec = ((uintptr_t)ja % 16 == 0) && ((uintptr_t)val % 16 == 0);
    const bool diag = !K || (K[1] == 0.0 && K[2] == 0.0 && K[3] == 0.0 && K[5] == 0.0 &&
                             K[6] == 0.0 && K[7] == 0.0);
    auto kern = vec ? (diag ? k_kuhn_fill<true, true> : k_kuhn_fill<true, false>)
                    : (diag ? k_kuhn_fill<false, true> : k_kuhn_fill<false, false>);
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, KU_ROWS, smem);
    const long long tiles = (rows + KU_ROWS - 1) / KU_ROWS;
    const int grid = (int)std::min<long long>(tiles, (long long)sms * std::max(per_sm, 1));
    kern<<<grid, KU_ROWS, smem, s>>>(N, (int)rows, kcell, ia, fill ? ja : nullptr,
                                     fill ? val : nullptr);
    count_launch();
    HZB_LAUNCH_CHECK();
    return SUCCESS;
}

}  // namespace hzb
