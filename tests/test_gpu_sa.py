"""Smoothed aggregation (AMG_type SA_AMG, amg_setup_sa) against the
reference's own setup and solves (tests/golden/sa.npz, on the matrices of
gmres.npz): the same level sizes and adapted threshold, every coarse operator
and every smoothed prolongation bit for bit (SHA-256 of the arrays, the
coarsest as the reference leaves it, transposed), and the same PCG /
flexible GMRES iterations and solutions.  Variants: filtered and unfiltered
smoother, a threshold that adapts, the W-cycle with the iterative coarse
solver."""
import hashlib

import numpy as np
import pytest

import hazmath_b200 as hz
from conftest import small_case

pytestmark = pytest.mark.gpu

XTOL = 1e-10
VARIANTS = ["fix/sa", "fix/sa_nf", "kuhn/sa", "kuhn/sa_nf", "kuhn/sa_t", "kuhn/sa_w"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def amg_of(v):
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    return hz.bench_amg(max_levels=ip[0], coarse_dof=ip[1], cycle_type=ip[2], smoother=ip[3],
                         presmooth_iter=ip[4], postsmooth_iter=ip[5], coarse_solver=ip[6],
                         aggregation_type=ip[7], max_aggregation=ip[8], coarse_scaling=ip[9],
                         maxit=ip[11], amli_degree=ip[12], nl_amli_krylov_type=ip[13],
                         AMG_type=ip[14], smooth_filter=ip[15], strong_coupled=dp[0],
                         relaxation=dp[1], tol=dp[2], tentative_smooth=dp[3])


def setup(golden, key):
    case = key.split("/")[0]
    A = small_case(golden("gmres.npz"), case)
    v = small_case(golden("sa.npz"), key)
    return A, v


@pytest.mark.parametrize("key", VARIANTS)
def test_sa_hierarchy_bit_exact(golden, key):
    A, v = setup(golden, key)
    S = hz.Solver(amg_of(v), hz.itsolver_param(linear_itsolver_type=hz.SOLVER_CG,
                                               linear_tol=1e-8, linear_maxit=300))
    assert S.setup_host(A["A_ia"], A["A_ja"], A["A_val"]) == 0, hz.last_error()
    st = S.stats()
    info = v["info"]
    assert st.num_levels == len(info)
    assert [st.rows[l] for l in range(len(info))] == [int(r) for r in info[:, 0]]
    assert [st.nnz[l] for l in range(len(info))] == [int(r) for r in info[:, 1]]
    assert st.strong_coupled == float(v["theta_after"])
    for l in range(len(info)):
        ia, ja, val, _ = S.level(l)
        assert [sha(ia), sha(ja), sha(val)] == list(v[f"A{l}_sha"]), f"A{l}"
        if l < len(info) - 1:
            P = S.prolongation(l)
            assert P is not None and len(P[1]) == int(info[l, 3])
            assert [sha(P[0]), sha(P[1]), sha(P[2])] == list(v[f"P{l}_sha"]), f"P{l}"
    S.close()


@pytest.mark.parametrize("key", VARIANTS)
@pytest.mark.parametrize("krylov", ["pcg", "fgmres"])
def test_sa_solve_matches_reference(golden, key, krylov):
    A, v = setup(golden, key)
    it = hz.itsolver_param(
        linear_itsolver_type=hz.SOLVER_CG if krylov == "pcg" else hz.SOLVER_VFGMRES,
        linear_precond_type=hz.PREC_AMG, linear_tol=1e-8, linear_maxit=300,
        linear_stop_type=hz.STOP_REL_RES, linear_restart=100)
    S = hz.Solver(amg_of(v), it)
    assert S.setup_host(A["A_ia"], A["A_ja"], A["A_val"]) == 0
    x = np.zeros(len(A["b"]))
    n_it = S.solve_host(A["b"], x)
    S.close()
    r = small_case(golden("sa.npz"), f"{key}/{krylov}")
    assert n_it == int(r["iters"]), (n_it, int(r["iters"]), hz.last_error())
    if "x" in r:
        np.testing.assert_allclose(x, r["x"], rtol=0, atol=XTOL * np.abs(r["x"]).max())


def test_sa_drop_in_amg_setup_sa(golden):
    """amg_setup_sa + precond_amg + dcsr_pcg, assembled by the caller;
    amg_setup_sa smooths whatever AMG_type says, as the reference's."""
    A, v = setup(golden, "kuhn/sa")
    prm = amg_of(v)
    prm.AMG_type = hz.UA_AMG
    H = hz.AMGHierarchy(A["A_ia"], A["A_ja"], A["A_val"], prm, smoothed=True)
    assert H.status == 0
    assert H.num_levels == len(v["info"])
    x = np.zeros(len(A["b"]))
    n_it = H.pcg(A["b"], x, tol=1e-8, maxit=300)
    H.free()
    r = small_case(golden("sa.npz"), "kuhn/sa/pcg")
    assert n_it == int(r["iters"])
    np.testing.assert_allclose(x, r["x"], rtol=0, atol=XTOL * np.abs(r["x"]).max())


def test_sa_refuses_mixed_precision(golden):
    A, v = setup(golden, "kuhn/sa")
    S = hz.Solver(amg_of(v), None, hz.b200_param(precision=hz.HZB_PREC_MIXED))
    assert S.setup_host(A["A_ia"], A["A_ja"], A["A_val"]) == hz.ERROR_INPUT_PAR
    assert "unsmoothed" in hz.last_error()
    S.close()
