"""End-to-end parity of the B200 UA-AMG-PCG drop-in with the reference:
hierarchies (sizes, aggregate maps, coarse operators) bit-exact, PCG
iteration counts equal, solutions within 1e-10 of the reference's relative
to max|x| (the coarsest direct solve and the reduction order differ by
rounding), and the drop-in entry points behaving like HAZmath's."""
import hashlib

import numpy as np
import pytest

import hazmath_b200 as hz
from conftest import small_case, small_case_names
from hazmath_b200 import problems as P
from gpu_util import DevCSR, dev, host, ptr

pytestmark = pytest.mark.gpu
XTOL = 1e-10


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def amg_from_case(c):
    ip = [int(v) for v in c["params"]]
    dp = [float(v) for v in c["dparams"]]
    return hz.bench_amg(max_levels=ip[0], coarse_dof=ip[1], cycle_type=ip[2], smoother=ip[3],
                         presmooth_iter=ip[4], postsmooth_iter=ip[5], coarse_solver=ip[6],
                         aggregation_type=ip[7], max_aggregation=ip[8], coarse_scaling=ip[9],
                         maxit=ip[11], strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])


def check_levels(S, g, full):
    st = S.stats()
    info = g["info"]
    assert st.num_levels == len(info)
    for l in range(st.num_levels):
        ia, ja, val, agg = S.level(l)
        assert (st.rows[l], st.nnz[l]) == (info[l][0], info[l][1])
        if full:
            assert np.array_equal(ia, g[f"A{l}_ia"])
            assert np.array_equal(ja, g[f"A{l}_ja"])
            assert np.array_equal(val, g[f"A{l}_val"])
        else:
            assert [sha(ia), sha(ja), sha(val)] == list(g[f"A{l}_sha"])
        if l < st.num_levels - 1:
            assert np.array_equal(agg, g[f"agg{l}"])
    assert st.strong_coupled == float(g["theta_after"])


@pytest.mark.parametrize("name", ["p2d_40", "aniso2d_31", "kuhn_12", "p2d_40_l1",
                                  "p2d_40_sgs_w", "p2d_40_sor_cs", "p2d_40_jac_cg",
                                  "theta_p2d_40"])
def test_small_case_end_to_end(golden, name):
    z = golden("small_cases.npz")
    assert name in small_case_names(z)
    c = small_case(z, name)
    S = hz.Solver(amg_from_case(c))
    assert S.setup_host(c["A_ia"], c["A_ja"], c["A_val"]) == 0, hz.last_error()
    check_levels(S, c, full=True)
    r, zz = dev(c["r"]), dev(np.zeros(len(c["r"])))
    assert S.precond_device(ptr(r), ptr(zz)) == 0
    np.testing.assert_allclose(host(zz), c["z"], rtol=0, atol=1e-11 * np.abs(c["z"]).max())
    x = np.zeros(len(c["b"]))
    it = S.solve_host(c["b"], x)
    assert it == int(c["iters"]), hz.last_error()
    np.testing.assert_allclose(x, c["x"], rtol=0, atol=XTOL * np.abs(c["x"]).max())
    S.close()


def test_fixture128_drop_in(golden):
    """examples/solvers known answer through linear_solver_dcsr_krylov_amg."""
    g = golden("fixture128.npz")
    ia, ja, val = P.poisson2d_5pt(128)
    it = hz.itsolver_param(linear_itsolver_type=1, linear_precond_type=2, linear_tol=1e-8,
                           linear_maxit=500, linear_stop_type=1)
    amg = hz.bench_amg()
    x = np.zeros(len(ia) - 1)
    n_it = hz.linear_solver_dcsr_krylov_amg(ia, ja, val, g["b"], x, it, amg)
    assert n_it == int(g["iters"]) == 15
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=XTOL * np.abs(g["x"]).max())
    assert amg.strong_coupled == float(g["theta_after"])    # caller's param mutated


def test_fixture128_hierarchy_and_history(golden):
    g = golden("fixture128.npz")
    ia, ja, val = P.poisson2d_5pt(128)
    S = hz.Solver()
    assert S.setup_host(ia, ja, val) == 0
    check_levels(S, g, full=False)
    S.close()


@pytest.mark.parametrize("path", [2, 4])
def test_c1_hierarchy_other_hem_paths(golden, monkeypatch, path):
    monkeypatch.setenv("HZB_HEM_PATH", str(path))
    g = golden("c1_poisson255.npz")
    ia, ja, val = P.poisson2d_5pt(255)
    S = hz.Solver()
    assert S.setup_host(ia, ja, val) == 0, hz.last_error()
    check_levels(S, g, full=False)
    S.close()


def test_c1_poisson255(golden):
    g = golden("c1_poisson255.npz")
    ia, ja, val = P.poisson2d_5pt(255)
    b = P.rhs_uniform(len(ia) - 1, 1)
    S = hz.Solver()
    A = DevCSR(ia, ja, val)
    assert S.setup_device(*A.args()) == 0, hz.last_error()
    check_levels(S, g, full=False)
    bd, xd = dev(b), dev(np.zeros(len(b)))
    it = S.solve_device(ptr(bd), ptr(xd))
    assert it == int(g["iters"]) == 24
    x = host(xd)
    np.testing.assert_allclose(x[:64], g["x_head"], rtol=0, atol=XTOL * np.abs(x).max())
    st = S.stats()
    assert st.final_relres < 1e-8
    S.close()


def test_amg_setup_precond_pcg_pieces(golden):
    """amg_data_create + amg_setup_ua + precond_amg + dcsr_pcg, the way
    HAZNICS' create_precond_amg assembles the preconditioner."""
    g = golden("fixture128.npz")
    ia, ja, val = P.poisson2d_5pt(128)
    H = hz.AMGHierarchy(ia, ja, val, hz.bench_amg())
    assert H.status == 0
    assert H.num_levels == len(g["info"])
    for l in range(H.num_levels - 1):
        assert np.array_equal(H.agg(l), g[f"agg{l}"])
    x = np.zeros(len(ia) - 1)
    assert H.pcg(g["b"], x) == 15
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=XTOL * np.abs(g["x"]).max())
    H.free()


def test_python_wrapper(golden):
    g = golden("fixture128.npz")
    ia, ja, val = P.poisson2d_5pt(128)
    u = np.zeros(len(ia) - 1)
    hz.python_wrapper_krylov_amg(ia, ja, val, g["b"], u, tol=1e-8, maxit=500)
    np.testing.assert_allclose(u, g["x"], rtol=0, atol=XTOL * np.abs(g["x"]).max())


def test_linear_solver_amg_converges():
    ia, ja, val = P.poisson2d_5pt(64)
    b = P.rhs_uniform(len(ia) - 1, 5)
    x = np.zeros(len(b))
    it = hz.linear_solver_amg(ia, ja, val, b, x, hz.bench_amg(maxit=100, tol=1e-8))
    assert 0 < it <= 100
    r = b - _spmv(ia, ja, val, x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-8


def _spmv(ia, ja, val, x):
    import scipy.sparse as sp
    return sp.csr_matrix((val, ja, ia)) @ x


def test_error_codes():
    # GCR (6) is not one of solver_dcsr_linear_itsolver's types
    it = hz.itsolver_param(linear_itsolver_type=6, linear_tol=1e-8)
    ia, ja, val = P.poisson2d_5pt(20)
    x = np.zeros(400)
    b = np.ones(400)
    assert hz.linear_solver_dcsr_krylov_amg(ia, ja, val, b, x, it, hz.bench_amg()) \
        == hz.ERROR_SOLVER_TYPE
    it = hz.itsolver_param(linear_itsolver_type=1, linear_tol=1e-8, linear_maxit=2)
    assert hz.linear_solver_dcsr_krylov_amg(ia, ja, val, b, x, it, hz.bench_amg(
        coarse_dof=10)) == hz.ERROR_SOLVER_MAXIT


def test_fast_modes_converge():
    """multicolour GS + parallel matching: not bit-exact, judged by
    convergence against the exact mode's iteration count."""
    ia, ja, val = P.poisson2d_5pt(255)
    b = P.rhs_uniform(len(ia) - 1, 1)
    S = hz.Solver(b200=hz.b200_param(gs_schedule=hz.HZB_GS_MULTICOLOR,
                                     matching=hz.HZB_MATCH_PARALLEL))
    assert S.setup_host(ia, ja, val) == 0
    x = np.zeros(len(b))
    it = S.solve_host(b, x)
    assert 0 < it <= 40, it
    r = b - _spmv(ia, ja, val, x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-8
    S.close()


def test_mixed_precision_kuhn():
    """FP32 V-cycle (l1-Jacobi x2) inside FP64 flexible CG reaches 1e-8 in
    FP64 and agrees with the FP64 solve to the tolerance's order."""
    N = 24
    ia, ja, val = P.kuhn3d_p1(N, P.lognormal_field(N, 1.0, 8.0, 2))
    b = P.rhs_uniform(len(ia) - 1, 3)
    amg = hz.bench_amg(smoother=hz.SMOOTHER_L1DIAG, presmooth_iter=2, postsmooth_iter=2)
    S64 = hz.Solver(amg)
    assert S64.setup_host(ia, ja, val) == 0
    x64 = np.zeros(len(b))
    it64 = S64.solve_host(b, x64)
    S32 = hz.Solver(hz.bench_amg(smoother=hz.SMOOTHER_L1DIAG, presmooth_iter=2,
                                  postsmooth_iter=2),
                    b200=hz.b200_param(precision=hz.HZB_PREC_MIXED))
    assert S32.setup_host(ia, ja, val) == 0
    x32 = np.zeros(len(b))
    it32 = S32.solve_host(b, x32)
    assert it64 > 0 and it32 > 0
    r = b - _spmv(ia, ja, val, x32)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-8
    assert it32 <= it64 + 3
    assert np.linalg.norm(x32 - x64) / np.linalg.norm(x64) < 1e-6
    S64.close()
    S32.close()
