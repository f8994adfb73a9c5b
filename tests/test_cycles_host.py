"""Host-side pieces of the AMLI cycle, no GPU needed: amg_amli_coef of the
library against the reference's coefficients (tests/golden/cycles.npz), bit
for bit, and the preconditioner each cycle type selects."""
import numpy as np
import pytest

import hazmath_b200 as hz
from conftest import small_case


@pytest.fixture(scope="module", autouse=True)
def built():
    from hazmath_b200 import build
    build.build()


@pytest.mark.parametrize("degree", range(5))
def test_amli_coefficients_bit_exact(golden, degree):
    ref = golden("cycles.npz")[f"amli_coef/{degree}"]
    got = hz.amli_coef(2.0, 0.5, degree)
    assert got.tobytes() == ref.tobytes(), (got, ref)


def test_amli_coefficients_other_interval(golden):
    ref = golden("cycles.npz")["amli_coef/wide3"]
    assert hz.amli_coef(10.0, 0.1, 3).tobytes() == ref.tobytes()


def test_amli_polynomial_approximates_inverse():
    """x q(x) stays within the best-approximation error of 1 on [0.5, 2]."""
    x = np.linspace(0.5, 2.0, 2001)
    errs = []
    for d in range(5):
        c = hz.amli_coef(2.0, 0.5, d)
        q = sum(c[k] * x ** k for k in range(d + 1))
        errs.append(np.abs(1 - x * q).max())
    assert all(errs[k + 1] < errs[k] for k in range(4)), errs


def test_precond_of_cycle_type():
    assert hz._PRECOND_OF_CYCLE[hz.AMLI_CYCLE] == "precond_amli"
    assert hz._PRECOND_OF_CYCLE[hz.NL_AMLI_CYCLE] == "precond_nl_amli"
    assert hz._PRECOND_OF_CYCLE[hz.ADD_CYCLE] == "precond_amg_add"
    assert hz.V_CYCLE not in hz._PRECOND_OF_CYCLE


def test_cycle_fixture_covers_every_variant(golden):
    z = golden("cycles.npz")
    for case in ("fix", "kuhn"):
        for var in ("a2", "n", "d"):
            v = small_case(z, f"{case}/{var}")
            assert int(v["params"][2]) in (3, 4, 5)
            assert "pcg/iters" in v and "fgmres/iters" in v and "gcg/iters" in v


ORACLE_CYCLES = [("fix", "a2"), ("fix", "d"), ("kuhn", "a1"), ("kuhn", "a2"), ("kuhn", "a3"),
                 ("kuhn", "a2s"), ("kuhn", "a2i"), ("kuhn", "a2d"), ("kuhn", "d"),
                 ("kuhn", "ds"), ("kuhn", "di")]


@pytest.mark.parametrize("case,var", ORACLE_CYCLES)
def test_oracle_amli_and_additive_cycles_match_reference(golden, port, case, var):
    """The oracle's restatement of amli / mgcycle_add (oracle/hzoracle.c
    or_amli, or_add_cycle) against one application of the reference's
    precond_amli / precond_amg_add: bit for bit with the iterative coarse
    solver, to 1e-13 of max |z| with the direct one (dense Cholesky here,
    the reference's sparse LDL^T there)."""
    import oracle
    A = small_case(golden("gmres.npz"), case)
    z = golden("cycles.npz")
    v = small_case(z, f"{case}/{var}")
    names = ["max_levels", "coarse_dof", "cycle_type", "smoother", "presmooth_iter",
             "postsmooth_iter", "coarse_solver", "aggregation_type", "max_aggregation",
             "coarse_scaling", "print_level", "maxit", "amli_degree", "nl_amli_krylov_type"]
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    kw = dict(zip(names, ip[:14]))
    kw.update(strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])
    prm = oracle.AMGParams(**kw)
    assert port.setup(A["A_ia"], A["A_ja"], A["A_val"], prm) == 0
    assert port.num_levels() == int(v["levels"])
    kind = 3 if var.startswith("a") else 5
    coef = z[f"amli_coef/{prm.amli_degree}"] if kind == 3 else None
    got = port.precond_cycle(kind, A["b"], coef, prm.tol)
    if prm.coarse_solver != 32:
        assert got.tobytes() == v["z"].tobytes()
    else:
        np.testing.assert_allclose(got, v["z"], rtol=0, atol=1e-13 * np.abs(v["z"]).max())


GCG_CASES = [(c, v) for c in ("fix", "kuhn")
             for v in ("v", "a1", "a2", "a3", "a2s", "a2i", "a2d", "d", "ds", "di")]


@pytest.mark.parametrize("case,var", GCG_CASES)
def test_oracle_gcg_matches_reference(golden, port, case, var):
    """The oracle's dcsr_pgcg (or_gcg) with the cycle type's preconditioner
    against the reference's run: the same iteration count, the residual norm
    at every preconditioner call to 1e-13 of the largest (bit for bit with the
    iterative coarse solver), the solution to 1e-13 of max |x| where stored."""
    import oracle
    A = small_case(golden("gmres.npz"), case)
    z = golden("cycles.npz")
    v = small_case(z, f"{case}/{var}")
    names = ["max_levels", "coarse_dof", "cycle_type", "smoother", "presmooth_iter",
             "postsmooth_iter", "coarse_solver", "aggregation_type", "max_aggregation",
             "coarse_scaling", "print_level", "maxit", "amli_degree", "nl_amli_krylov_type"]
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    kw = dict(zip(names, ip[:14]))
    kw.update(strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])
    prm = oracle.AMGParams(**kw)
    assert port.setup(A["A_ia"], A["A_ja"], A["A_val"], prm) == 0
    kind = {1: 1, 2: 1, 3: 3, 5: 5}[prm.cycle_type]
    coef = z[f"amli_coef/{prm.amli_degree}"] if kind == 3 else None
    it, x, hist = port.gcg(A["b"], kind, coef, prm.tol, tol=1e-8, maxit=100)
    assert it == int(v["gcg/iters"])
    rh = v["gcg/hist"]
    assert len(hist) == len(rh)
    if prm.coarse_solver != 32:
        assert hist.tobytes() == rh.tobytes()
    else:
        np.testing.assert_allclose(hist, rh, rtol=0, atol=1e-13 * rh.max())
    if "gcg/x" in v:
        np.testing.assert_allclose(x, v["gcg/x"], rtol=0, atol=1e-13 * np.abs(v["gcg/x"]).max())


NL_CASES = [("fix", "n"), ("kuhn", "n"), ("kuhn", "ng"), ("kuhn", "nd"), ("kuhn", "ngd"),
            ("kuhn", "ni")]


@pytest.mark.parametrize("case,var", NL_CASES)
def test_oracle_nl_amli_matches_reference(golden, port, case, var):
    """The oracle's nonlinear AMLI cycle (or_nl_amli: flexible GMRES(30) or
    GCG on the coarse levels, preconditioned by the cycle one level down)
    against one application of the reference's precond_nl_amli: bit for bit
    with the iterative coarse solver, to 1e-13 of max |z| with the direct
    one."""
    import oracle
    A = small_case(golden("gmres.npz"), case)
    v = small_case(golden("cycles.npz"), f"{case}/{var}")
    names = ["max_levels", "coarse_dof", "cycle_type", "smoother", "presmooth_iter",
             "postsmooth_iter", "coarse_solver", "aggregation_type", "max_aggregation",
             "coarse_scaling", "print_level", "maxit", "amli_degree", "nl_amli_krylov_type"]
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    kw = dict(zip(names, ip[:14]))
    kw.update(strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])
    prm = oracle.AMGParams(**kw)
    assert port.setup(A["A_ia"], A["A_ja"], A["A_val"], prm) == 0
    assert port.num_levels() == int(v["levels"])
    got = port.precond_nl_amli(A["b"], prm.amli_degree, prm.nl_amli_krylov_type, prm.tol)
    if prm.coarse_solver != 32:
        assert got.tobytes() == v["z"].tobytes()
    else:
        np.testing.assert_allclose(got, v["z"], rtol=0, atol=1e-13 * np.abs(v["z"]).max())
