"""The oracle's restatements of the reference's Krylov drivers (oracle/
hzoracle.c) against the reference's own runs: dcsr_pvgmres and
dcsr_pvfgmres with the V-cycle (tests/golden/gmres.npz) -- every restart
length 3-100 and the three stopping types give the same iteration counts
and the same number of preconditioner calls; the residual norms handed to
the preconditioner agree to 1e-9 of the largest (the coarsest solve is a
dense Cholesky here, the reference's sparse LDL^T there, and a restarted
flexible method carries that rounding through its restarts)."""
import numpy as np
import pytest

import oracle
from conftest import small_case

NAMES = ["max_levels", "coarse_dof", "cycle_type", "smoother", "presmooth_iter",
         "postsmooth_iter", "coarse_solver", "aggregation_type", "max_aggregation",
         "coarse_scaling", "print_level", "maxit"]
RUNS = [(flex, restart, stop) for flex in (0, 1) for restart in (3, 7, 25, 100)
        for stop in ((1, 2, 3) if restart == 25 else (1,))]


@pytest.mark.parametrize("case", ["fix", "kuhn"])
def test_oracle_gmres_matches_reference(golden, port, case):
    A = small_case(golden("gmres.npz"), case)
    ip = [int(t) for t in A["params"]]
    dp = [float(t) for t in A["dparams"]]
    kw = dict(zip(NAMES, ip[:12]))
    kw.update(strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])
    assert port.setup(A["A_ia"], A["A_ja"], A["A_val"], oracle.AMGParams(**kw)) == 0
    for flex, restart, stop in RUNS:
        key = f"{'f' if flex else 'v'}{restart}_s{stop}"
        it, x, hist = port.gmres_port(A["b"], tol=1e-8, maxit=300, restart=restart,
                                      flexible=bool(flex), stop_type=stop)
        rh = A[key + "/hist"]
        assert it == int(A[key + "/iters"]), key
        assert len(hist) == len(rh), key
        np.testing.assert_allclose(hist, rh, rtol=0, atol=1e-9 * rh.max(), err_msg=key)
        if key + "/x" in A:
            np.testing.assert_allclose(x, A[key + "/x"], rtol=0,
                                       atol=1e-9 * np.abs(A[key + "/x"]).max(), err_msg=key)


BASES = {"fix": {}, "kuhn": dict(smoother=10, presmooth_iter=2, postsmooth_iter=2,
                                 coarse_dof=100)}


@pytest.mark.parametrize("case", ["fix", "kuhn"])
def test_oracle_minres_matches_reference(golden, port, case):
    """dcsr_pminres restated (or_minres) against the reference's runs in
    tests/golden/minres.npz: the same iteration counts and preconditioner
    calls for the three stopping types with the V-cycle, histories and
    solutions to 1e-13; without a preconditioner (139 steps on the Kuhn
    matrix) the solution bit for bit."""
    A = small_case(golden("gmres.npz"), case)
    z = golden("minres.npz")
    assert port.setup(A["A_ia"], A["A_ja"], A["A_val"], oracle.AMGParams(**BASES[case])) == 0
    for stop in (1, 2, 3):
        v = small_case(z, f"{case}/s{stop}")
        it, x, hist = port.minres_port(A["b"], tol=1e-8, maxit=500, stop_type=stop)
        assert it == int(v["iters"]), stop
        assert len(hist) == len(v["hist"]), stop
        np.testing.assert_allclose(hist, v["hist"], rtol=0, atol=1e-13 * v["hist"].max())
        np.testing.assert_allclose(x, v["x"], rtol=0, atol=1e-13 * np.abs(v["x"]).max())
    if case == "kuhn":
        v = small_case(z, "kuhn/nopc")
        it, x, _ = port.minres_port(A["b"], tol=1e-6, maxit=2000, stop_type=1, use_pc=False)
        assert it == int(v["iters"])
        assert x.tobytes() == v["x"].tobytes()
