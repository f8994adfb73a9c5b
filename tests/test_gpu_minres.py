"""Preconditioned MINRES (Krylov type 2, dcsr_pminres) against the reference's
own runs (tests/golden/minres.npz, on the matrices of gmres.npz): the same
iteration counts and solutions with the V-cycle preconditioner for the three
stopping types, through the device handle and through dcsr_pminres with the
setup's preconditioner, and without a preconditioner."""
import ctypes as C

import numpy as np
import pytest

import hazmath_b200 as hz
from conftest import small_case

pytestmark = pytest.mark.gpu

XTOL = 1e-10
BASES = {"fix": {}, "kuhn": dict(smoother=hz.SMOOTHER_L1DIAG, presmooth_iter=2,
                                 postsmooth_iter=2, coarse_dof=100)}


def amg(case):
    return hz.bench_amg(**BASES[case])


def check(it, x, g):
    assert it == int(g["iters"]), (it, int(g["iters"]), hz.last_error())
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=XTOL * np.abs(g["x"]).max())


@pytest.mark.parametrize("case", ["fix", "kuhn"])
@pytest.mark.parametrize("stop", [1, 2, 3])
def test_minres_matches_reference(golden, case, stop):
    c = small_case(golden("gmres.npz"), case)
    g = small_case(golden("minres.npz"), f"{case}/s{stop}")
    S = hz.Solver(amg(case), hz.itsolver_param(
        linear_itsolver_type=hz.SOLVER_MinRes, linear_precond_type=hz.PREC_AMG,
        linear_tol=1e-8, linear_maxit=500, linear_stop_type=stop))
    assert S.setup_host(c["A_ia"], c["A_ja"], c["A_val"]) == 0
    x = np.zeros(len(c["b"]))
    it = S.solve_host(c["b"], x)
    S.close()
    check(it, x, g)


def test_minres_drop_in_with_amg_setup_ua(golden):
    c = small_case(golden("gmres.npz"), "kuhn")
    g = small_case(golden("minres.npz"), "kuhn/s1")
    H = hz.AMGHierarchy(c["A_ia"], c["A_ja"], c["A_val"], amg("kuhn"))
    assert H.status == 0
    x = np.zeros(len(c["b"]))
    it = H.minres(c["b"], x, tol=1e-8, maxit=500)
    H.free()
    check(it, x, g)


def test_minres_without_preconditioner(golden):
    c = small_case(golden("gmres.npz"), "kuhn")
    g = small_case(golden("minres.npz"), "kuhn/nopc")
    A = hz._HostCSR(c["A_ia"], c["A_ja"], c["A_val"])
    b = np.ascontiguousarray(c["b"])
    x = np.zeros(len(b))
    it = hz.lib().dcsr_pminres(C.byref(A.mat), C.byref(hz._dvec(b)), C.byref(hz._dvec(x)),
                               None, 1e-6, 2000, 1, 0)
    # 139 unpreconditioned steps: inner products summed in another order move
    # the step at which ||r|| crosses 1e-6 ||b|| by at most one
    assert abs(it - int(g["iters"])) <= 1, (it, int(g["iters"]))
    import scipy.sparse as sp
    M = sp.csr_matrix((c["A_val"], c["A_ja"], c["A_ia"]))
    assert np.linalg.norm(b - M @ x) <= 1e-6 * np.linalg.norm(b)


def test_solver_dispatch_runs_minres(golden):
    """solver_dcsr_linear_itsolver type 2 (the reference prints a notice and
    runs dcsr_pminres)."""
    c = small_case(golden("gmres.npz"), "fix")
    g = small_case(golden("minres.npz"), "fix/s1")
    it = hz.itsolver_param(linear_itsolver_type=hz.SOLVER_MinRes, linear_precond_type=hz.PREC_AMG,
                           linear_tol=1e-8, linear_maxit=500, linear_stop_type=1)
    x = np.zeros(len(c["b"]))
    n_it = hz.linear_solver_dcsr_krylov_amg(c["A_ia"], c["A_ja"], c["A_val"], c["b"], x, it,
                                            amg("fix"))
    check(n_it, x, g)
