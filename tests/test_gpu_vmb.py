"""VMB aggregation (aggregation_type 1, aggregation_vmb) against the
reference's own setup and solve (tests/golden/vmb.npz, on the matrices of
gmres.npz): the same level sizes, every aggregate map and every coarse
operator bit for bit (SHA-256; the coarsest as the reference leaves it,
transposed), the same adapted threshold, PCG iterations and solutions.
Variants: the default cap of 20 per aggregate and caps of 4 and 9, a
threshold that adapts, the W-cycle; also the mixed-precision cycle on a VMB
hierarchy (the method of the drop-in, judged by the true residual)."""
import hashlib

import numpy as np
import pytest

import hazmath_b200 as hz
from conftest import small_case

pytestmark = pytest.mark.gpu

XTOL = 1e-10
VARIANTS = ["fix/vmb", "fix/vmb4", "kuhn/vmb", "kuhn/vmb_t", "kuhn/vmb_w"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def amg_of(v):
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    return hz.bench_amg(max_levels=ip[0], coarse_dof=ip[1], cycle_type=ip[2], smoother=ip[3],
                         presmooth_iter=ip[4], postsmooth_iter=ip[5], coarse_solver=ip[6],
                         aggregation_type=ip[7], max_aggregation=ip[8], coarse_scaling=ip[9],
                         maxit=ip[11], strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])


def setup(golden, key):
    A = small_case(golden("gmres.npz"), key.split("/")[0])
    v = small_case(golden("vmb.npz"), key)
    return A, v


@pytest.mark.parametrize("key", VARIANTS)
def test_vmb_hierarchy_and_pcg_match_reference(golden, key):
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
        ia, ja, val, agg = S.level(l)
        assert [sha(ia), sha(ja), sha(val)] == list(v[f"A{l}_sha"]), f"A{l}"
        if l < len(info) - 1:
            np.testing.assert_array_equal(agg, v[f"agg{l}"])
    x = np.zeros(len(A["b"]))
    n_it = S.solve_host(A["b"], x)
    S.close()
    assert n_it == int(v["pcg/iters"]), (n_it, int(v["pcg/iters"]), hz.last_error())
    np.testing.assert_allclose(x, v["pcg/x"], rtol=0, atol=XTOL * np.abs(v["pcg/x"]).max())


def test_vmb_mixed_precision_cycle(golden):
    A, v = setup(golden, "kuhn/vmb")
    S = hz.Solver(amg_of(v), hz.itsolver_param(linear_itsolver_type=hz.SOLVER_CG,
                                               linear_tol=1e-8, linear_maxit=300),
                  hz.b200_param(precision=hz.HZB_PREC_MIXED))
    assert S.setup_host(A["A_ia"], A["A_ja"], A["A_val"]) == 0
    assert S.stats().num_levels == len(v["info"])
    x = np.zeros(len(A["b"]))
    n_it = S.solve_host(A["b"], x)
    S.close()
    assert 0 < n_it < 300
    import scipy.sparse as sp
    M = sp.csr_matrix((A["A_val"], A["A_ja"], A["A_ia"]))
    assert np.linalg.norm(A["b"] - M @ x) <= 1e-8 * np.linalg.norm(A["b"])
