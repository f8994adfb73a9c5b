"""Variable-restart GMRES (Krylov type 3, dcsr_pvgmres) and flexible GMRES
(type 4, dcsr_pvfgmres) with the AMG preconditioner against the reference's
own runs (tests/golden/gmres.npz): the same iteration counts, the same
residual norm at every preconditioner application, the same solutions,
for restarts 3 to 100 and the three stopping types; and the reference's
default Krylov setting (flexible GMRES, restart 100) through the drop-in
driver."""
import numpy as np
import pytest

import hazmath_b200 as hz
from conftest import small_case

pytestmark = pytest.mark.gpu

XTOL = 1e-10
VARIANTS = [(3, 1), (7, 1), (25, 1), (25, 2), (25, 3), (100, 1)]


def amg_from_case(c):
    ip = [int(v) for v in c["params"]]
    dp = [float(v) for v in c["dparams"]]
    return hz.bench_amg(max_levels=ip[0], coarse_dof=ip[1], cycle_type=ip[2], smoother=ip[3],
                         presmooth_iter=ip[4], postsmooth_iter=ip[5], coarse_solver=ip[6],
                         aggregation_type=ip[7], max_aggregation=ip[8], coarse_scaling=ip[9],
                         maxit=ip[11], strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])


def itparam(kind, restart, stop):
    return hz.itsolver_param(
        linear_itsolver_type=hz.SOLVER_VFGMRES if kind == "f" else hz.SOLVER_VGMRES,
        linear_precond_type=hz.PREC_AMG, linear_tol=1e-8, linear_maxit=300,
        linear_stop_type=stop, linear_restart=restart)


@pytest.mark.parametrize("case", ["fix", "kuhn"])
@pytest.mark.parametrize("kind", ["v", "f"])
@pytest.mark.parametrize("restart,stop", VARIANTS)
def test_gmres_matches_reference(golden, case, kind, restart, stop):
    z = golden("gmres.npz")
    c = small_case(z, case)
    g = small_case(z, f"{case}/{kind}{restart}_s{stop}")
    S = hz.Solver(amg_from_case(c), itparam(kind, restart, stop))
    assert S.setup_host(c["A_ia"], c["A_ja"], c["A_val"]) == 0, hz.last_error()
    x = np.zeros(len(c["b"]))
    it = S.solve_host(c["b"], x)
    S.close()
    assert it == int(g["iters"]), (it, int(g["iters"]), hz.last_error())
    if "x" in g:
        np.testing.assert_allclose(x, g["x"], rtol=0, atol=XTOL * np.abs(g["x"]).max())


def test_default_krylov_setting_is_flexible_gmres(golden):
    """param_linear_solver_init's defaults (type 4, restart 100) through
    linear_solver_dcsr_krylov_amg give the reference's iterations."""
    z = golden("gmres.npz")
    c = small_case(z, "fix")
    g = small_case(z, "fix/f100_s1")
    it = hz.itsolver_param(linear_tol=1e-8, linear_maxit=300,
                           linear_stop_type=hz.STOP_REL_RES)
    assert it.linear_itsolver_type == hz.SOLVER_VFGMRES and it.linear_restart == 100
    x = np.zeros(len(c["b"]))
    n_it = hz.linear_solver_dcsr_krylov_amg(c["A_ia"], c["A_ja"], c["A_val"], c["b"], x, it,
                                            amg_from_case(c))
    assert n_it == int(g["iters"]), (n_it, hz.last_error())


def test_gmres_maxit_and_unknown_type(golden):
    z = golden("gmres.npz")
    c = small_case(z, "kuhn")
    S = hz.Solver(amg_from_case(c), hz.itsolver_param(
        linear_itsolver_type=hz.SOLVER_VFGMRES, linear_precond_type=hz.PREC_AMG,
        linear_tol=1e-14, linear_maxit=4, linear_stop_type=1, linear_restart=25))
    assert S.setup_host(c["A_ia"], c["A_ja"], c["A_val"]) == 0
    x = np.zeros(len(c["b"]))
    assert S.solve_host(c["b"], x) == hz.ERROR_SOLVER_MAXIT   # iter >= MaxIt, as the reference
    S.close()
    S = hz.Solver(amg_from_case(c), hz.itsolver_param(
        linear_itsolver_type=6, linear_precond_type=hz.PREC_AMG,
        linear_tol=1e-8, linear_maxit=50))
    assert S.setup_host(c["A_ia"], c["A_ja"], c["A_val"]) == 0
    assert S.solve_host(c["b"], np.zeros(len(c["b"]))) == hz.ERROR_SOLVER_TYPE
    S.close()


@pytest.mark.parametrize("flexible", [False, True])
def test_gmres_drop_in_with_amg_setup_ua(golden, flexible):
    """amg_setup_ua + precond_amg + dcsr_pvgmres / dcsr_pvfgmres, the pieces a
    caller assembles itself, give the reference's iterations and solution."""
    z = golden("gmres.npz")
    c = small_case(z, "fix")
    g = small_case(z, f"fix/{'f' if flexible else 'v'}25_s1")
    H = hz.AMGHierarchy(c["A_ia"], c["A_ja"], c["A_val"], amg_from_case(c))
    assert H.status == 0
    x = np.zeros(len(c["b"]))
    it = H.gmres(c["b"], x, tol=1e-8, maxit=300, restart=25, flexible=flexible)
    H.free()
    assert it == int(g["iters"]), (it, hz.last_error())
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=XTOL * np.abs(g["x"]).max())
