/*
 * hzgnn_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU oracle of the learned
 * l1-Jacobi weights (no counterpart in the reference).
 *
 *  - or_gnn_forward / or_gnn_backward: the message-passing network of the
 *    CUDA library, restated sequentially in FP32 with BF16 rounding at the
 *    same points (stored activations, dense-layer inputs and weights);
 *  - or_learn_errors / or_learn_loss_grad: the method-generated training
 *    errors and the ncyc-cycle A-norm contraction loss with its adjoint
 *    gradient, in FP64 on the oracle hierarchy built by or_setup (l1-Jacobi
 *    smoother), so the GPU gradients can be checked here and by finite
 *    differences.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* hierarchy access from hzoracle.c */
int or_num_levels(void);
void or_level_info(int l, int *out);
void or_precond(const double *r, double *z);
int or_hier_level(int l, int *n, const int **ia, const int **ja, const double **a,
                  const int **agg, const int **ria, const int **rja, int *nc);
void or_cycle_from(int l0, const double *b, double *x);

#define H 32
#define OFF_WIN 0
#define OFF_BIN 128
#define LAYER 3200
#define L_U 0
#define L_V 1024
#define L_C 1088
#define L_W 1120
#define L_B 3168
#define OFF_L0 160
#define OFF_WO (OFF_L0 + 3 * LAYER)
#define OFF_BO (OFF_WO + 32)
#define NPARAM (OFF_BO + 1)

int or_gnn_version(void) { return 1; }
int or_gnn_num_params(void) { return NPARAM; }

/* rounding to BF16 at the CUDA kernels' points (on by default); off gives
 * the plain FP32 network, for checking the backward against autograd */
static int g_round = 1;
void or_gnn_set_rounding(int on) { g_round = on; }

static float bf16r(float f)
{
    uint32_t u;
    if (!g_round) return f;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return f;
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&f, &u, 4);
    return f;
}

static void edge_feat(double aij, double aii, double ajj, float *e0, float *e1)
{
    *e0 = (float)(aij / sqrt(fabs(aii * ajj)));
    float l = (float)(0.5 * log(fabs(ajj / aii)));
    *e1 = l > 4.f ? 4.f : (l < -4.f ? -4.f : l);
}

/* activations of the last forward pass */
static int g_n = 0;
static float *g_feats, *g_h[4], *g_P[3], *g_M[3], *g_y[3], *g_om;
static double *g_diag;
static const int *g_ia, *g_ja;
static const double *g_a;

static void gnn_alloc(int n)
{
    if (g_n == n) return;
    free(g_feats); free(g_om); free(g_diag);
    for (int l = 0; l < 4; ++l) free(g_h[l]);
    for (int l = 0; l < 3; ++l) { free(g_P[l]); free(g_M[l]); free(g_y[l]); }
    g_feats = (float *)malloc(sizeof(float) * 4 * n);
    g_om = (float *)malloc(sizeof(float) * n);
    g_diag = (double *)malloc(sizeof(double) * n);
    for (int l = 0; l < 4; ++l) g_h[l] = (float *)malloc(sizeof(float) * H * n);
    for (int l = 0; l < 3; ++l) {
        g_P[l] = (float *)malloc(sizeof(float) * H * n);
        g_M[l] = (float *)malloc(sizeof(float) * H * n);
        g_y[l] = (float *)malloc(sizeof(float) * H * n);
    }
    g_n = n;
}

void or_gnn_forward(int n, const int *ia, const int *ja, const double *a,
                    const float *prm, float *omega)
{
    gnn_alloc(n);
    g_ia = ia; g_ja = ja; g_a = a;
    for (int i = 0; i < n; ++i) {
        double d = 0.0, l1 = 0.0, off = 0.0, mx = 0.0;
        int got = 0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) {
            double v = a[k];
            l1 += fabs(v);
            if (ja[k] == i) { if (!got) { d = v; got = 1; } }
            else { off += v; if (fabs(v) > mx) mx = fabs(v); }
        }
        g_diag[i] = d;
        double il = l1 > 0 ? 1.0 / l1 : 0.0;
        g_feats[4 * i + 0] = (float)(d * il);
        g_feats[4 * i + 1] = (float)(off * il);
        g_feats[4 * i + 2] = (float)(mx * il);
        g_feats[4 * i + 3] = 1.0f;
    }
    for (int i = 0; i < n; ++i)
        for (int f = 0; f < H; ++f) {
            float v = prm[OFF_BIN + f];
            for (int k = 0; k < 4; ++k) v += prm[OFF_WIN + f * 4 + k] * g_feats[4 * i + k];
            g_h[0][i * H + f] = bf16r(v > 0.f ? v : 0.f);
        }
    for (int l = 0; l < 3; ++l) {
        const float *lay = prm + OFF_L0 + l * LAYER;
        const float *h = g_h[l];
        for (int i = 0; i < n; ++i)                         /* P = h U^T */
            for (int o = 0; o < H; ++o) {
                float s = 0.f;
                for (int k = 0; k < H; ++k) s += h[i * H + k] * bf16r(lay[L_U + o * H + k]);
                g_P[l][i * H + o] = bf16r(s);
            }
        for (int i = 0; i < n; ++i) {                       /* messages */
            int deg = 0;
            float acc[H];
            for (int f = 0; f < H; ++f) acc[f] = 0.f;
            for (int k = ia[i]; k < ia[i + 1]; ++k) {
                int j = ja[k];
                if (j == i) continue;
                float e0, e1;
                edge_feat(a[k], g_diag[i], g_diag[j], &e0, &e1);
                for (int f = 0; f < H; ++f) {
                    float q = g_P[l][j * H + f] + lay[L_V + 2 * f] * e0 +
                              lay[L_V + 2 * f + 1] * e1 + lay[L_C + f];
                    acc[f] += q > 0.f ? q : 0.f;
                }
                ++deg;
            }
            for (int f = 0; f < H; ++f) g_M[l][i * H + f] = bf16r(deg ? acc[f] / deg : 0.f);
        }
        for (int i = 0; i < n; ++i)                         /* y, h_next */
            for (int o = 0; o < H; ++o) {
                float s = 0.f;
                for (int k = 0; k < H; ++k) s += h[i * H + k] * bf16r(lay[L_W + o * 64 + k]);
                for (int k = 0; k < H; ++k)
                    s += g_M[l][i * H + k] * bf16r(lay[L_W + o * 64 + 32 + k]);
                float yv = s + lay[L_B + o];
                g_y[l][i * H + o] = bf16r(yv);
                g_h[l + 1][i * H + o] = bf16r((yv > 0.f ? yv : 0.f) + h[i * H + o]);
            }
    }
    for (int i = 0; i < n; ++i) {
        float z = prm[OFF_BO];
        for (int f = 0; f < H; ++f) z += prm[OFF_WO + f] * g_h[3][i * H + f];
        z = z > 12.f ? 12.f : (z < -12.f ? -12.f : z);
        g_om[i] = 2.0f / (1.0f + expf(-z));
        omega[i] = g_om[i];
    }
}

/* parameter gradients for dL/domega of the last forward pass */
void or_gnn_backward(const float *prm, const float *domega, float *grad)
{
    const int n = g_n;
    float *dH = (float *)calloc((size_t)H * n, sizeof(float));
    float *dY = (float *)calloc((size_t)H * n, sizeof(float));
    float *dM = (float *)calloc((size_t)H * n, sizeof(float));
    float *dP = (float *)calloc((size_t)H * n, sizeof(float));
    memset(grad, 0, sizeof(float) * NPARAM);
    for (int i = 0; i < n; ++i) {
        float om = g_om[i];
        float dz = domega[i] * om * (1.f - 0.5f * om);
        grad[OFF_BO] += dz;
        for (int f = 0; f < H; ++f) {
            dH[i * H + f] = dz * prm[OFF_WO + f];
            grad[OFF_WO + f] += dz * g_h[3][i * H + f];
        }
    }
    for (int l = 2; l >= 0; --l) {
        const float *lay = prm + OFF_L0 + l * LAYER;
        float *glay = grad + OFF_L0 + l * LAYER;
        for (int i = 0; i < n * H; ++i) {
            dY[i] = g_y[l][i] > 0.f ? dH[i] : 0.f;
            glay[L_B + i % H] += dY[i];
        }
        for (int i = 0; i < n; ++i)                         /* dW, dX */
            for (int o = 0; o < H; ++o) {
                float d = dY[i * H + o], db = bf16r(d);
                for (int k = 0; k < H; ++k) {
                    glay[L_W + o * 64 + k] += d * g_h[l][i * H + k];
                    glay[L_W + o * 64 + 32 + k] += d * g_M[l][i * H + k];
                    dH[i * H + k] += db * bf16r(lay[L_W + o * 64 + k]);
                }
                for (int k = 0; k < H; ++k)
                    dM[i * H + k] = (o == 0 ? 0.f : dM[i * H + k]) +
                                    db * bf16r(lay[L_W + o * 64 + 32 + k]);
            }
        memset(dP, 0, sizeof(float) * H * n);
        for (int i = 0; i < n; ++i) {                       /* messages */
            int deg = 0;
            for (int k = g_ia[i]; k < g_ia[i + 1]; ++k) deg += g_ja[k] != i;
            if (!deg) continue;
            for (int k = g_ia[i]; k < g_ia[i + 1]; ++k) {
                int j = g_ja[k];
                if (j == i) continue;
                float e0, e1;
                edge_feat(g_a[k], g_diag[i], g_diag[j], &e0, &e1);
                for (int f = 0; f < H; ++f) {
                    float q = g_P[l][j * H + f] + lay[L_V + 2 * f] * e0 +
                              lay[L_V + 2 * f + 1] * e1 + lay[L_C + f];
                    if (q > 0.f) {
                        float gm = dM[i * H + f] / deg;
                        dP[j * H + f] += gm;
                        glay[L_V + 2 * f] += gm * e0;
                        glay[L_V + 2 * f + 1] += gm * e1;
                        glay[L_C + f] += gm;
                    }
                }
            }
        }
        for (int i = 0; i < n; ++i)                         /* dU, dh */
            for (int o = 0; o < H; ++o) {
                float d = dP[i * H + o], db = bf16r(d);
                for (int k = 0; k < H; ++k) {
                    glay[L_U + o * H + k] += d * g_h[l][i * H + k];
                    dH[i * H + k] += db * bf16r(lay[L_U + o * H + k]);
                }
            }
    }
    for (int i = 0; i < n; ++i)
        for (int f = 0; f < H; ++f) {
            float d = g_h[0][i * H + f] > 0.f ? dH[i * H + f] : 0.f;
            grad[OFF_BIN + f] += d;
            for (int k = 0; k < 4; ++k) grad[OFF_WIN + f * 4 + k] += d * g_feats[4 * i + k];
        }
    free(dH); free(dY); free(dM); free(dP);
}

/* ------------------------------------------------------------------------ */
/* method-generated loss on the oracle hierarchy                             */
/* ------------------------------------------------------------------------ */
static double hash_unit(unsigned long long seed, unsigned long long i)
{
    unsigned long long x = seed * 0x9E3779B97F4A7C15ull + i * 0xBF58476D1CE4E5B9ull + 1;
    x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27; x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

static void mxv(int n, const int *ia, const int *ja, const double *a, const double *x,
                double *y)
{
    for (int i = 0; i < n; ++i) {
        double t = 0.0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) t += a[k] * x[ja[k]];
        y[i] = t;
    }
}
static double dotp(int n, const double *x, const double *y)
{
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}

/* x_1 = B_c b_1 where b_1 = R r; then out -= alpha P x_1 (alpha = 1) or
 * out += P x_1 (alpha = -1) */
static void coarse(const double *r, double *out, int add)
{
    int n0, n1, nc;
    const int *ia, *ja, *agg, *ria, *rja;
    const double *a;
    or_hier_level(0, &n0, &ia, &ja, &a, &agg, &ria, &rja, &nc);
    n1 = nc;
    double *b1 = (double *)calloc(n1 > 0 ? n1 : 1, sizeof(double));
    double *x1 = (double *)calloc(n1 > 0 ? n1 : 1, sizeof(double));
    for (int c = 0; c < n1; ++c) {
        double t = 0.0;
        for (int k = ria[c]; k < ria[c + 1]; ++k) t += r[rja[k]];
        b1[c] = t;
    }
    or_cycle_from(1, b1, x1);
    for (int i = 0; i < n0; ++i) {
        double t = 0.0;
        if (agg[i] >= 0) t += x1[agg[i]];
        if (add) out[i] += t; else out[i] -= t;
    }
    free(b1); free(x1);
}

static void l1n(int n, const int *ia, const double *a, double *l1)
{
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = ia[i]; k < ia[i + 1]; ++k) s += fabs(a[k]);
        l1[i] = s;
    }
}

void or_set_omega(const float *omega);

/* seeded random vectors after three plain l1 sweeps and ncyc V-cycles, unit
 * A-norm; the cycles use omega on the fine level (NULL: plain weights).
 * ncyc = 0 gives vectors that do not depend on omega. */
void or_learn_errors(int ns, unsigned long long seed, double *E, const float *omega,
                     int ncyc)
{
    or_set_omega(omega);
    int n, nc;
    const int *ia, *ja, *agg, *ria, *rja;
    const double *a;
    or_hier_level(0, &n, &ia, &ja, &a, &agg, &ria, &rja, &nc);
    double *l1 = (double *)malloc(sizeof(double) * n);
    double *r = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    l1n(n, ia, a, l1);
    for (int s = 0; s < ns; ++s) {
        double *e = E + (size_t)s * n;
        for (int i = 0; i < n; ++i) e[i] = hash_unit(seed + 7919ull * (unsigned long long)s, i);
        for (int it = 0; it < 3; ++it) {
            mxv(n, ia, ja, a, e, r);
            for (int i = 0; i < n; ++i) e[i] -= (1.0 / l1[i]) * r[i];
        }
        for (int it = 0; it < ncyc; ++it) {
            mxv(n, ia, ja, a, e, r);
            or_precond(r, t);
            for (int i = 0; i < n; ++i) e[i] -= t[i];
        }
        mxv(n, ia, ja, a, e, r);
        double s2 = 1.0 / sqrt(dotp(n, e, r));
        for (int i = 0; i < n; ++i) e[i] *= s2;
    }
    or_set_omega(NULL);
    free(l1); free(r); free(t);
}

double or_learn_loss_grad(const float *omega, int ns, const double *E, int ncyc,
                          double *domega)
{
    int n, nc;
    const int *ia, *ja, *agg, *ria, *rja;
    const double *a;
    or_hier_level(0, &n, &ia, &ja, &a, &agg, &ria, &rja, &nc);
    double *l1 = (double *)malloc(sizeof(double) * n);
    double *e = (double *)malloc(sizeof(double) * n);
    double *r = (double *)malloc(sizeof(double) * n);
    double *g = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    double *Ae = (double *)malloc(sizeof(double) * 4 * (size_t)ncyc * (size_t)n);
    l1n(n, ia, a, l1);
    memset(domega, 0, sizeof(double) * n);
    double total = 0.0;
    for (int s = 0; s < ns; ++s) {
        memcpy(e, E + (size_t)s * n, sizeof(double) * n);
        mxv(n, ia, ja, a, e, r);
        double n0 = dotp(n, e, r);
        int q = 0;
        for (int c = 0; c < ncyc; ++c) {
            for (int j = 0; j < 2; ++j, ++q) {
                mxv(n, ia, ja, a, e, Ae + (size_t)q * n);
                for (int i = 0; i < n; ++i) e[i] -= ((double)omega[i] / l1[i]) * Ae[(size_t)q * n + i];
            }
            mxv(n, ia, ja, a, e, r);
            coarse(r, e, 0);
            for (int j = 0; j < 2; ++j, ++q) {
                mxv(n, ia, ja, a, e, Ae + (size_t)q * n);
                for (int i = 0; i < n; ++i) e[i] -= ((double)omega[i] / l1[i]) * Ae[(size_t)q * n + i];
            }
        }
        mxv(n, ia, ja, a, e, r);
        double n1 = dotp(n, e, r);
        total += n1 / n0;
        for (int i = 0; i < n; ++i) g[i] = r[i] * (2.0 / n0);
        for (int c = ncyc - 1; c >= 0; --c) {
            for (int j = 0; j < 2; ++j) {
                --q;
                for (int i = 0; i < n; ++i) {
                    double inv = 1.0 / l1[i];
                    domega[i] -= g[i] * Ae[(size_t)q * n + i] * inv;
                    t[i] = (double)omega[i] * inv * g[i];
                }
                mxv(n, ia, ja, a, t, r);
                for (int i = 0; i < n; ++i) g[i] -= r[i];
            }
            memset(t, 0, sizeof(double) * n);
            coarse(g, t, 1);                 /* t = P B_c R g */
            mxv(n, ia, ja, a, t, r);
            for (int i = 0; i < n; ++i) g[i] -= r[i];
            for (int j = 0; j < 2; ++j) {
                --q;
                for (int i = 0; i < n; ++i) {
                    double inv = 1.0 / l1[i];
                    domega[i] -= g[i] * Ae[(size_t)q * n + i] * inv;
                    t[i] = (double)omega[i] * inv * g[i];
                }
                mxv(n, ia, ja, a, t, r);
                for (int i = 0; i < n; ++i) g[i] -= r[i];
            }
        }
    }
    for (int i = 0; i < n; ++i) domega[i] /= ns;
    free(l1); free(e); free(r); free(g); free(t); free(Ae);
    return total / ns;
}
