"""UA-AMG for block (BSR) matrices against the reference's own runs
(tests/golden/bsr.npz): amg_setup_ua_bsr's hierarchy bit for bit (level
sizes, block aggregates, SHA-256 of every level's block matrix), one
application of precond_dbsr_amg, and linear_solver_dbsr_krylov_amg's CG,
GMRES(25) and flexible GMRES(25) iteration counts and solutions.  Matrices:
problems.block_system of the Kuhn P1 matrix of gmres.npz with 3 x 3 blocks
and of the 5-point matrix with 2 x 2 blocks.  Variants: block Gauss-Seidel,
Jacobi (two sweeps), symmetric Gauss-Seidel, the W-cycle, coarse scaling, two
cycles per application, a threshold that drops couplings, VMB aggregation."""
import hashlib

import numpy as np
import pytest

import hazmath_b200 as hz
from hazmath_b200 import problems as P
from conftest import small_case

pytestmark = pytest.mark.gpu

# The coarsest level is solved by GMRES(25) to 1e-6 in both libraries; the
# residuals and inner products of that solve and of the Krylov loop are
# summed in another order here (the hierarchy and the smoothing are not), so
# z and x agree to rounding, not bit for bit.
ZTOL = 1e-10        # one preconditioner application, relative to max |z|
XTOL = 1e-9         # solutions, relative to max |x|
VARIANTS = ["kuhn/gs", "kuhn/jac", "kuhn/sgs", "kuhn/w", "kuhn/cs", "kuhn/m2", "kuhn/t",
            "kuhn/vmb", "fix/gs"]
NB = {"kuhn": 3, "fix": 2}
SEED = {"kuhn": 31, "fix": 32}
KRYLOV = {"pcg": hz.SOLVER_CG, "gmres": hz.SOLVER_VGMRES, "fgmres": hz.SOLVER_VFGMRES}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def amg_of(v):
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    return hz.bench_amg(max_levels=ip[0], coarse_dof=ip[1], cycle_type=ip[2], smoother=ip[3],
                         presmooth_iter=ip[4], postsmooth_iter=ip[5], coarse_solver=ip[6],
                         aggregation_type=ip[7], max_aggregation=ip[8], coarse_scaling=ip[9],
                         maxit=ip[11], strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])


_MATS = {}


def matrix(golden, case):
    if case not in _MATS:
        g = small_case(golden("gmres.npz"), case)
        _MATS[case] = P.block_system(g["A_ia"], g["A_ja"], g["A_val"], NB[case], SEED[case])
    return _MATS[case]


def load(golden, key):
    case = key.split("/")[0]
    ia, ja, val = matrix(golden, case)
    z = golden("bsr.npz")
    assert [sha(ia), sha(ja), sha(val)] == list(z[f"{case}/A_sha"])
    return case, (ia, ja, val), z[f"{case}/b"], small_case(z, key)


def itparam(kind, maxit=300):
    return hz.itsolver_param(linear_itsolver_type=KRYLOV[kind], linear_tol=1e-8,
                             linear_maxit=maxit, linear_stop_type=hz.STOP_REL_RES,
                             linear_restart=25)


@pytest.mark.parametrize("key", VARIANTS)
def test_bsr_hierarchy_and_precond_match_reference(golden, key):
    case, (ia, ja, val), b, v = load(golden, key)
    S = hz.Solver(amg_of(v), itparam("pcg"))
    assert S.setup_bsr_host(NB[case], ia, ja, val) == 0, hz.last_error()
    info = v["info"]
    assert S.stats().num_levels == len(info)
    for l in range(len(info)):
        lia, lja, lval, agg = S.bsr_level(l)
        assert (len(lia) - 1, len(lja)) == tuple(info[l]), l
        assert [sha(lia), sha(lja), sha(lval)] == list(v[f"A{l}_sha"]), l
        if l < len(info) - 1:
            np.testing.assert_array_equal(agg, v[f"agg{l}"])
    z = S.bsr_precond_host(b)
    S.close()
    np.testing.assert_allclose(z, v["z"], rtol=0, atol=ZTOL * np.abs(v["z"]).max())


@pytest.mark.parametrize("key", VARIANTS)
@pytest.mark.parametrize("kind", ["pcg", "gmres", "fgmres"])
def test_bsr_krylov_amg_matches_reference(golden, key, kind):
    """linear_solver_dbsr_krylov_amg from x = 0."""
    case, (ia, ja, val), b, v = load(golden, key)
    x = np.zeros(len(b))
    it = hz.linear_solver_dbsr_krylov_amg(NB[case], ia, ja, val, b, x, itparam(kind),
                                          amg_of(v))
    r = small_case(golden("bsr.npz"), f"{key}/{kind}")
    assert it == int(r["iters"]), (it, int(r["iters"]), hz.last_error())
    if "x" in r:
        np.testing.assert_allclose(x, r["x"], rtol=0, atol=XTOL * np.abs(r["x"]).max())
    sia, sja, sval = P.bsr_to_csr(ia, ja, val, NB[case])
    res = b - hz_mxv(sia, sja, sval, x)
    assert np.linalg.norm(res) <= 1e-7 * np.linalg.norm(b)


def hz_mxv(ia, ja, val, x):
    import scipy.sparse as sp
    return sp.csr_matrix((val, ja, ia), shape=(len(ia) - 1, len(x))) @ x


def test_bsr_handle_solve_and_device_vectors(golden):
    """The handle's pieces: setup once, solve twice (host and device
    vectors), the Krylov loop preconditioned by precond_dbsr_amg."""
    import torch
    case, (ia, ja, val), b, v = load(golden, "kuhn/gs")
    r = small_case(golden("bsr.npz"), "kuhn/gs/pcg")
    S = hz.Solver(amg_of(v), itparam("pcg"))
    assert S.setup_bsr_host(NB[case], ia, ja, val) == 0
    x = np.zeros(len(b))
    assert S.bsr_solve_host(b, x) == int(r["iters"])
    np.testing.assert_allclose(x, r["x"], rtol=0, atol=XTOL * np.abs(r["x"]).max())
    db = torch.tensor(b, device="cuda:0")
    dx = torch.zeros_like(db)
    assert S.bsr_solve_device(db.data_ptr(), dx.data_ptr()) == int(r["iters"])
    np.testing.assert_allclose(dx.cpu().numpy(), x, rtol=0, atol=1e-14 * np.abs(x).max())
    dz = torch.zeros_like(db)
    assert S.bsr_precond_device(db.data_ptr(), dz.data_ptr()) == 0
    np.testing.assert_allclose(dz.cpu().numpy(), v["z"], rtol=0,
                               atol=ZTOL * np.abs(v["z"]).max())
    st = S.stats()
    assert st.launches > 0 and st.condest > 1.0
    S.close()


def test_bsr_rejects_what_the_reference_rejects(golden):
    case, (ia, ja, val), b, v = load(golden, "kuhn/gs")
    x = np.zeros(len(b))
    # MINRES has no BSR version: solver_dbsr_linear_itsolver's default case
    it = hz.itsolver_param(linear_itsolver_type=hz.SOLVER_MinRes, linear_tol=1e-8,
                           linear_maxit=50)
    assert hz.linear_solver_dbsr_krylov_amg(NB[case], ia, ja, val, b, x, it,
                                            amg_of(v)) == hz.ERROR_SOLVER_TYPE
    # blocks larger than the kernels hold
    S = hz.Solver(amg_of(v), itparam("pcg"))
    n = 4
    bia = np.arange(n + 1, dtype=np.int32)
    bja = np.arange(n, dtype=np.int32)
    bval = np.tile(np.eye(9).reshape(-1), n)
    assert S.setup_bsr_host(9, bia, bja, bval) == hz.ERROR_INPUT_PAR
    # a zero diagonal block on a level that is smoothed
    big = matrix(golden, "kuhn")
    zval = big[2].copy().reshape(-1, 3, 3)
    rows = np.repeat(np.arange(len(big[0]) - 1), np.diff(big[0]))
    d0 = np.nonzero((big[1] == rows) & (rows == 5))[0][0]
    zval[d0] = 0.0
    assert S.setup_bsr_host(3, big[0], big[1], zval.reshape(-1)) == hz.ERROR_DATA_ZERODIAG
    S.close()
