/*
 * ref_assembly.c -- test infrastructure only.
 *
 * The reference's own P1 stiffness assembly on its own cube mesh, for
 * pinning the project's Kuhn-mesh generator (hazmath_b200/problems.py
 * kuhn3d_p1) and the device assembly built on it: mesh_cube_init
 * (src/amr/mesh_cube_anydim.c:30-128) with uniform refinement, scfinalize,
 * sc_vols, then call_assembly (examples/elliptic_p1/
 * supporting_elliptic_p1.h:537-647, read in place from the reference tree by
 * the include below) with alpha = 1, gamma = 0, which ends with
 * set_essential_bc: Dirichlet rows become identity rows and the other rows
 * keep only their non-Dirichlet columns.  Linked into libhazref.so by
 * build_ref.sh; nothing in the product loads it.
 */
#include "hazmath.h"
#include "functions_elliptic_p1.h"
#include "supporting_elliptic_p1.h"

static dCSRmat g_cube = {0, 0, 0, NULL, NULL, NULL};
static REAL *g_xv = NULL;
static INT *g_dir = NULL;

static void cube_free(void)
{
    free(g_cube.IA); free(g_cube.JA); free(g_cube.val);
    g_cube.IA = NULL; g_cube.JA = NULL; g_cube.val = NULL;
    g_cube.row = g_cube.col = g_cube.nnz = 0;
    free(g_xv); g_xv = NULL;
    free(g_dir); g_dir = NULL;
}

/* Build and assemble on the unit cube with ndiv divisions per edge; out:
 * [0] vertices, [1] stored entries, [2] simplices. */
void ref_cube_p1(int ndiv, int *out)
{
    cube_free();
    scomplex **sc_all = mesh_cube_init(3, ndiv, 11);
    scomplex *sc = sc_all[0];
    scfinalize(sc, NULL, (INT)1);
    sc_vols(sc);
    dCSRmat A = dcsr_create(0, 0, 0);
    dvector rhs;
    rhs.row = 0;
    rhs.val = NULL;
    call_assembly(sc, &A, &rhs, 1e0, 0e0);
    g_cube = A;
    g_xv = (REAL *)malloc(sizeof(REAL) * 3 * sc->nv);
    memcpy(g_xv, sc->x, sizeof(REAL) * 3 * sc->nv);
    g_dir = (INT *)malloc(sizeof(INT) * sc->nv);
    for (INT i = 0; i < sc->nv; ++i)
        g_dir[i] = (sc->bndry[i] >= MARKER_DIRICHLET) && (sc->bndry[i] < MARKER_NEUMANN);
    out[0] = sc->nv;
    out[1] = A.IA[A.row];
    out[2] = sc->ns;
    free(rhs.val);
    haz_scomplex_free(sc);
    free(sc_all);
}

/* the matrix, vertex coordinates (nv x 3) and Dirichlet flags of the last
 * ref_cube_p1 */
void ref_cube_p1_get(int *ia, int *ja, double *val, double *xv, int *dirichlet)
{
    memcpy(ia, g_cube.IA, sizeof(int) * (g_cube.row + 1));
    memcpy(ja, g_cube.JA, sizeof(int) * g_cube.IA[g_cube.row]);
    memcpy(val, g_cube.val, sizeof(double) * g_cube.IA[g_cube.row]);
    memcpy(xv, g_xv, sizeof(double) * 3 * g_cube.row);
    for (INT i = 0; i < g_cube.row; ++i) dirichlet[i] = g_dir[i];
}
