"""The AMLI (cycle_type 3), nonlinear AMLI (4) and additive (5) cycles and the
generalized CG method against the reference's own runs (tests/golden/
cycles.npz, on the matrices of gmres.npz): the same level count, one
preconditioner application z = B b, and for PCG, flexible GMRES(100) and GCG
with the cycle's preconditioner the same iteration counts (error codes
included) and the same solutions.  Variants: AMLI degrees 1-3, coarse
scaling, the iterative coarse solver, deep hierarchies (coarse_dof 50),
nonlinear AMLI with FGMRES or GCG on the coarse levels, GCG with the
V-cycle."""
import numpy as np
import pytest

import hazmath_b200 as hz
from conftest import small_case

pytestmark = pytest.mark.gpu

XTOL = 1e-10        # solutions: max-norm error relative to max |x|
ZTOL = 1e-12        # one preconditioner application, relative to max |z|
# with the iterative coarse solver (CG to 1e-4 tol = 1e-10) a cycle agrees to
# the accuracy of that solve: its inner products are summed in another order
ZTOL_CG = 1e-8
VARIANTS = ["a2", "a1", "a3", "a2s", "a2i", "a2d", "n", "ng", "nd", "ngd", "ni", "d", "ds",
            "di"]


def amg_of(v):
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    return hz.bench_amg(max_levels=ip[0], coarse_dof=ip[1], cycle_type=ip[2], smoother=ip[3],
                         presmooth_iter=ip[4], postsmooth_iter=ip[5], coarse_solver=ip[6],
                         aggregation_type=ip[7], max_aggregation=ip[8], coarse_scaling=ip[9],
                         maxit=ip[11], amli_degree=ip[12], nl_amli_krylov_type=ip[13],
                         strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])


def load(golden, case, var):
    A = small_case(golden("gmres.npz"), case)
    v = small_case(golden("cycles.npz"), f"{case}/{var}")
    return A, v


def check_run(it, x, r):
    assert it == int(r["iters"]), (it, int(r["iters"]), hz.last_error())
    if "x" in r:
        np.testing.assert_allclose(x, r["x"], rtol=0, atol=XTOL * np.abs(r["x"]).max())


@pytest.mark.parametrize("case", ["fix", "kuhn"])
@pytest.mark.parametrize("var", VARIANTS)
@pytest.mark.parametrize("krylov", ["pcg", "fgmres"])
def test_cycle_solve_matches_reference(golden, case, var, krylov):
    """linear_solver_dcsr_krylov_amg's pairing of the cycle type with its
    preconditioner, through the device handle."""
    A, v = load(golden, case, var)
    r = small_case(golden("cycles.npz"), f"{case}/{var}/{krylov}")
    it = hz.itsolver_param(
        linear_itsolver_type=hz.SOLVER_CG if krylov == "pcg" else hz.SOLVER_VFGMRES,
        linear_precond_type=hz.PREC_AMG, linear_tol=1e-8, linear_maxit=300,
        linear_stop_type=hz.STOP_REL_RES, linear_restart=100)
    S = hz.Solver(amg_of(v), it)
    assert S.setup_host(A["A_ia"], A["A_ja"], A["A_val"]) == 0, hz.last_error()
    assert S.stats().num_levels == int(v["levels"])
    x = np.zeros(len(A["b"]))
    n_it = S.solve_host(A["b"], x)
    S.close()
    check_run(n_it, x, r)


@pytest.mark.parametrize("case", ["fix", "kuhn"])
@pytest.mark.parametrize("var", VARIANTS + ["v"])
def test_gcg_and_precond_match_reference(golden, case, var):
    """amg_setup_ua + the cycle type's precond_* function (one application,
    and inside dcsr_pgcg), the pieces a caller assembles itself."""
    A, v = load(golden, case, var)
    r = small_case(golden("cycles.npz"), f"{case}/{var}/gcg")
    H = hz.AMGHierarchy(A["A_ia"], A["A_ja"], A["A_val"], amg_of(v))
    assert H.status == 0
    assert H.num_levels == int(v["levels"])
    if "z" in v:
        z = H.precond(A["b"])
        tol = ZTOL_CG if int(v["params"][6]) != hz.SOLVER_UMFPACK else ZTOL
        np.testing.assert_allclose(z, v["z"], rtol=0, atol=tol * np.abs(v["z"]).max())
    x = np.zeros(len(A["b"]))
    n_it = H.gcg(A["b"], x, tol=1e-8, maxit=100)
    H.free()
    check_run(n_it, x, r)


@pytest.mark.parametrize("var", ["a2", "n", "d"])
def test_cycle_drop_in_krylov_entry_points(golden, var):
    """dcsr_pcg / dcsr_pvfgmres given precond_amli, precond_nl_amli or
    precond_amg_add run the whole loop on the device with that cycle."""
    A, v = load(golden, "kuhn", var)
    H = hz.AMGHierarchy(A["A_ia"], A["A_ja"], A["A_val"], amg_of(v))
    assert H.status == 0
    for kr in ("pcg", "fgmres"):
        r = small_case(golden("cycles.npz"), f"kuhn/{var}/{kr}")
        x = np.zeros(len(A["b"]))
        if kr == "pcg":
            n_it = H.pcg(A["b"], x, tol=1e-8, maxit=300)
        else:
            n_it = H.gmres(A["b"], x, tol=1e-8, maxit=300, restart=100, flexible=True)
        check_run(n_it, x, r)
    H.free()


@pytest.mark.parametrize("var", ["a2", "n", "d"])
def test_single_cycle_matches_precond(golden, var):
    """amli / nl_amli / mgcycle_add on mgl[0].b with x = 0 is one
    application of the matching precond_* function (maxit = 1)."""
    A, v = load(golden, "kuhn", var)
    H = hz.AMGHierarchy(A["A_ia"], A["A_ja"], A["A_val"], amg_of(v))
    assert H.status == 0
    x = H.cycle(A["b"], np.zeros(len(A["b"])))
    H.free()
    np.testing.assert_allclose(x, v["z"], rtol=0, atol=ZTOL * np.abs(v["z"]).max())


def test_cycles_refuse_mixed_precision(golden):
    A, v = load(golden, "kuhn", "a2")
    S = hz.Solver(amg_of(v), hz.itsolver_param(linear_itsolver_type=hz.SOLVER_CG,
                                               linear_tol=1e-8, linear_maxit=50),
                  hz.b200_param(precision=hz.HZB_PREC_MIXED))
    assert S.setup_host(A["A_ia"], A["A_ja"], A["A_val"]) == 0
    assert S.solve_host(A["b"], np.zeros(len(A["b"]))) == hz.ERROR_INPUT_PAR
    assert "V and W" in hz.last_error()
    S.close()
