"""CPU checks of the block (BSR) path: the fixture matrices are what
problems.block_system makes, the scalar expansion is the block matrix, the
oracle's restatement of amg_setup_ua_bsr gives the reference's hierarchies
bit for bit, the reference (where it is built here) still produces the
committed hierarchy, and linear_solver_dbsr_krylov_amg rejects malformed
input before it touches a device."""
import ctypes as C
import hashlib

import numpy as np
import pytest

import hazmath_b200 as hz
import oracle
from hazmath_b200 import problems as P
from conftest import small_case

NB = {"kuhn": 3, "fix": 2}
SEED = {"kuhn": 31, "fix": 32}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", ["kuhn", "fix"])
def test_block_system_reproduces_fixture(golden, case):
    g = small_case(golden("gmres.npz"), case)
    ia, ja, val = P.block_system(g["A_ia"], g["A_ja"], g["A_val"], NB[case], SEED[case])
    assert [sha(ia), sha(ja), sha(val)] == list(golden("bsr.npz")[f"{case}/A_sha"])
    # SPD blocks: symmetric pattern and values, positive diagonal blocks
    blocks = val.reshape(-1, NB[case], NB[case])
    rows = np.repeat(np.arange(len(ia) - 1), np.diff(ia))
    diag = blocks[ja == rows]
    assert np.all(np.linalg.eigvalsh(diag) > 0)


def test_bsr_to_csr_is_the_block_matrix():
    rng = np.random.default_rng(3)
    ia = np.array([0, 2, 3, 5], np.int32)
    ja = np.array([0, 2, 1, 0, 2], np.int32)
    val = rng.standard_normal(5 * 4)
    sia, sja, sval = P.bsr_to_csr(ia, ja, val, 2)
    dense = np.zeros((6, 6))
    for I in range(3):
        for k in range(ia[I], ia[I + 1]):
            dense[2 * I:2 * I + 2, 2 * ja[k]:2 * ja[k] + 2] = val[4 * k:4 * k + 4].reshape(2, 2)
    got = np.zeros((6, 6))
    for i in range(6):
        got[i, sja[sia[i]:sia[i + 1]]] = sval[sia[i]:sia[i + 1]]
    np.testing.assert_array_equal(got, dense)
    # row I nb + r lists the blocks of row I in order, columns in order
    assert list(sja[sia[0]:sia[1]]) == [0, 1, 4, 5]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_reference_still_gives_committed_hierarchy(golden):
    z = golden("bsr.npz")
    v = small_case(z, "kuhn/gs")
    g = small_case(golden("gmres.npz"), "kuhn")
    ia, ja, val = P.block_system(g["A_ia"], g["A_ja"], g["A_val"], 3, 31)
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    prm = oracle.AMGParams(max_levels=ip[0], coarse_dof=ip[1], cycle_type=ip[2],
                           smoother=ip[3], presmooth_iter=ip[4], postsmooth_iter=ip[5],
                           coarse_solver=ip[6], aggregation_type=ip[7], max_aggregation=ip[8],
                           coarse_scaling=ip[9], maxit=ip[11], strong_coupled=dp[0],
                           relaxation=dp[1], tol=dp[2])
    R = oracle.ref()
    assert R.bsr_setup(3, ia, ja, val, prm) == 0
    nl = R.bsr_num_levels()
    assert nl == len(v["info"])
    for l in range(nl):
        assert [sha(a) for a in R.bsr_level_A(l, 3)] == list(v[f"A{l}_sha"])
    np.testing.assert_array_equal(R.bsr_precond(z["kuhn/b"]), v["z"])
    R.bsr_free()


BSR_VARIANTS = ["kuhn/gs", "kuhn/jac", "kuhn/sgs", "kuhn/w", "kuhn/cs", "kuhn/m2", "kuhn/t",
                "kuhn/vmb", "fix/gs"]


@pytest.mark.parametrize("key", BSR_VARIANTS)
def test_oracle_bsr_hierarchy_matches_reference(golden, port, key):
    """The oracle's restatement of amg_setup_ua_bsr (condensation, HEM or
    VMB, dbsr_rap) against the reference's hierarchy digests."""
    case = key.split("/")[0]
    g = small_case(golden("gmres.npz"), case)
    ia, ja, val = P.block_system(g["A_ia"], g["A_ja"], g["A_val"], NB[case], SEED[case])
    v = small_case(golden("bsr.npz"), key)
    ip = [int(t) for t in v["params"]]
    levels, aggs = port.bsr_hierarchy(NB[case], ia, ja, val, theta=float(v["dparams"][0]),
                                      coarse_dof=ip[1], max_levels=ip[0],
                                      aggregation_type=ip[7], max_aggregation=ip[8])
    info = v["info"]
    assert len(levels) == len(info)
    for l, (lia, lja, lval) in enumerate(levels):
        assert (len(lia) - 1, len(lja)) == tuple(info[l]), l
        assert [sha(lia), sha(lja), sha(lval)] == list(v[f"A{l}_sha"]), l
    for l, agg in enumerate(aggs):
        np.testing.assert_array_equal(agg, v[f"agg{l}"])


def _mat(ia, ja, val, nb, manner=0, nnz=None):
    return hz.dBSRmat(len(ia) - 1, len(ia) - 1, int(ia[-1]) if nnz is None else nnz, nb, manner,
                      val.ctypes.data_as(C.POINTER(hz.REAL)), ia.ctypes.data_as(C.POINTER(hz.INT)),
                      ja.ctypes.data_as(C.POINTER(hz.INT)))


def test_drop_in_rejects_malformed_input_on_the_host():
    L = hz.lib()
    ia = np.array([0, 1, 2], np.int32)
    ja = np.array([0, 1], np.int32)
    val = np.tile(np.eye(2).reshape(-1), 2)
    b = np.ones(4)
    x = np.zeros(4)
    it = hz.itsolver_param(linear_itsolver_type=hz.SOLVER_CG)
    amg = hz.amg_param()

    def call(A, bb=b):
        return L.linear_solver_dbsr_krylov_amg(C.byref(A), C.byref(hz._dvec(bb)),
                                               C.byref(hz._dvec(x)), C.byref(it), C.byref(amg))

    assert call(_mat(ia, ja, val, 2, manner=1)) == hz.ERROR_INPUT_PAR
    assert call(_mat(ia, ja, val, 2, nnz=3)) == hz.ERROR_DATA_STRUCTURE
    assert call(_mat(ia, ja, val, 2), np.ones(3)) == hz.ERROR_MAT_SIZE
    assert L.linear_solver_dbsr_krylov_amg(None, None, None, None, None) == hz.ERROR_INPUT_PAR


@pytest.mark.parametrize("key", BSR_VARIANTS)
def test_oracle_bsr_precond_bit_exact(golden, port, key):
    """The oracle's restatement of precond_dbsr_amg / mgcycle_bsr (block
    smoothers, sequential residuals, the coarsest GMRES(25) without
    preconditioner, coarse scaling) gives the reference's z bit for bit."""
    case = key.split("/")[0]
    g = small_case(golden("gmres.npz"), case)
    ia, ja, val = P.block_system(g["A_ia"], g["A_ja"], g["A_val"], NB[case], SEED[case])
    z = golden("bsr.npz")
    v = small_case(z, key)
    ip = [int(t) for t in v["params"]]
    port.bsr_hierarchy(NB[case], ia, ja, val, theta=float(v["dparams"][0]), coarse_dof=ip[1],
                       max_levels=ip[0], aggregation_type=ip[7], max_aggregation=ip[8])
    got = port.bsr_precond(z[f"{case}/b"], cycle_type=ip[2], smoother=ip[3],
                           presmooth_iter=ip[4], coarse_scaling=ip[9], maxit=ip[11])
    assert got.tobytes() == v["z"].tobytes()
